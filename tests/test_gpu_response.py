"""Linear-response derivatives (rism3d_response): the reference's
"free-energy-response" (hnc3d.c:1969-2135, response_t1 1366-1421) against
the oracle's restatement (oracle.hnc3d.response) at the same converged t,
and -- for an uncharged solute, where the response is the exact total
derivative -- against the adjoint gradient.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from bgy3d_b200 import RismContext  # noqa: E402
from bgy3d_b200._abi import RismError  # noqa: E402
from oracle import hnc3d  # noqa: E402


def settings_of(meta, **kw):
    s = dict(meta["settings"])
    s["closure"] = int(s["closure"])
    s.update(kw)
    return s


def oracle_problem(meta, arr, s, solute):
    N = (s["N"],) * 3
    L = (2 * s["L"],) * 3
    return hnc3d.Problem(N, L, s["beta"], s["rho"], s["closure"], meta["solvent"], solute, arr["chi"], s["rmax"],
                         renorm=not s.get("no-renorm", False))


@pytest.mark.parametrize("charged", [True, False])
def test_response_matches_oracle(fixture_loader, charged):
    meta, arr = fixture_loader("synth6_kh_n32")
    s = settings_of(meta, **{"norm-tol": 1e-12})
    sol = [dict(a) for a in meta["solute"]]
    if not charged:
        for a in sol:
            a["charge"] = 0.0
    ctx = RismContext(sol, meta["solvent"], s, arr["chi"])
    T, res = ctx.solve()
    assert res["status"] == 0
    r = ctx.response(T)
    assert r["resid"] < 1e-9
    assert r["krylov-jv"] > 0
    sites = [0, 3]
    ref = hnc3d.response(oracle_problem(meta, arr, s, sol), T.cpu().numpy(), rtol=1e-12, sites=sites)
    scale = np.max(np.abs(ref[sites]))
    assert np.max(np.abs(r["x"][sites] - ref[sites])) < 1e-7 * scale
    if not charged:
        # uncharged: field1 is the whole field's derivative and nothing
        # long-range moves, so the response is the exact dmu/dx
        g = ctx.gradient(T)
        assert np.max(np.abs(r["x"] - g["x"])) < 1e-7 * np.max(np.abs(g["x"]))
    ctx.close()


def test_response_rejects_py(fixture_loader):
    meta, arr = fixture_loader("synth6_kh_n32")
    s = settings_of(meta, closure=2)
    ctx = RismContext(meta["solute"], meta["solvent"], s, arr["chi"])
    with pytest.raises(RismError):
        ctx.response(ctx.zeros())
    ctx.close()
