"""Repeated solves of moving solutes on one context (rism3d_ctx_set_solute):
the restart loop of a PES scan.  After a rebind, a solve warm-started from
the previous t reaches the root a fresh context finds for the new solute
(mu to 1e-9 kcal/mol, t to 1e-9 max-abs, both solved to |F|inf < 1e-12),
for a displaced site, a smaller solute and a larger one than the context
was created with.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from bgy3d_b200 import RismContext  # noqa: E402


def settings_of(meta, **kw):
    s = dict(meta["settings"])
    s["closure"] = int(s["closure"])
    s.update(kw)
    return s


def moved(solute, u, dx):
    out = [dict(a) for a in solute]
    x = list(out[u]["x"])
    x[0] += dx
    out[u]["x"] = tuple(x)
    return out


def fresh_solve(meta, arr, s, solute):
    ctx = RismContext(solute, meta["solvent"], s, arr["chi"])
    T, res = ctx.solve()
    obs = ctx.observables(T)
    out = (T.cpu().numpy(), obs["free-energy"], res)
    ctx.close()
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_rebind_matches_fresh_context(fixture_loader, precision):
    meta, arr = fixture_loader("synth6_kh_n32")
    s = settings_of(meta, **{"norm-tol": 1e-12, "precision": precision})
    sol = meta["solute"]
    scan = [moved(sol, 0, 0.1), sol[:4], sol + [dict(sol[0], x=(0.5, 0.5, 3.0), name="S9")]]
    ctx = RismContext(sol, meta["solvent"], s, arr["chi"])
    T, res = ctx.solve()
    for new in scan:
        ctx.set_solute(new)
        T, res = ctx.solve(T)  # warm start from the previous geometry's t
        assert res["status"] == 0
        mu = ctx.observables(T)["free-energy"]
        T_ref, mu_ref, res_ref = fresh_solve(meta, arr, s, new)
        assert abs(mu - mu_ref) < 1e-9
        assert np.max(np.abs(T.cpu().numpy() - T_ref)) < 1e-9
        assert res["newton-iters"] <= res_ref["newton-iters"]
    ctx.close()
