"""Large results of rism3d_solute_solve cross to caller memory through two
alternating pinned chunks of 16 MB, the host side of each chunk copied out
by several threads.  At 128^3 (t and g are 50 MB each: three full chunks
and a partial one) the returned arrays must be the device arrays bit for
bit: g recomputed on the device from the returned t equals the returned g,
and the returned t is the converged state of a solve in a context."""
import numpy as np
import pytest
import torch

from bgy3d_b200 import RismContext, hnc3d_run_solute


@pytest.mark.gpu
def test_staged_copies_of_t_and_g(fixture_loader):
    meta, arr = fixture_loader("synth6_kh_n32")
    s = dict(meta["settings"])
    s["closure"] = int(s["closure"])
    s.update(N=128, L=24.0)
    ctx = RismContext(meta["solute"], meta["solvent"], s, arr["chi"])
    T_ref, res = ctx.solve()
    assert res["status"] == 0
    for _ in range(2):  # the second call takes its chunks from the free list
        out = hnc3d_run_solute(meta["solute"], meta["solvent"], s, arr["chi"], want_g=True, want_restart=True)
        t_host, g_host = out["RESTART"], out["GUV"]
        assert t_host.shape == tuple(ctx.shape) and g_host.shape == tuple(ctx.shape)
        g_dev = ctx.observables(torch.from_numpy(t_host).to("cuda"), want_g=True)["GUV"].cpu().numpy()
        assert np.array_equal(g_host, g_dev)
        assert np.max(np.abs(t_host - T_ref.cpu().numpy())) < 1e-9
    ctx.close()


@pytest.mark.gpu
def test_context_cache_rebinds_the_solute(fixture_loader):
    """rism3d_solute_solve keeps the device context of a finished call and
    rebinds the solute on the next call with equal settings, solvent and
    chi: solves on the rebound context equal solves on fresh contexts bit for
    bit, in either order, and a change of settings builds a new context."""
    from bgy3d_b200 import lib
    meta, arr = fixture_loader("synth6_kh_n32")
    s = dict(meta["settings"])
    s["closure"] = int(s["closure"])
    s["norm-tol"] = 1e-12
    moved = [dict(site) for site in meta["solute"]]
    moved[0]["x"] = [moved[0]["x"][0] + 0.3, moved[0]["x"][1], moved[0]["x"][2] - 0.2]

    def run(solute, settings=s):
        out = hnc3d_run_solute(solute, meta["solvent"], settings, arr["chi"], want_g=True, want_restart=True)
        assert out["status"] == 0
        return out

    lib().rism3d_cache_clear()
    a1 = run(meta["solute"])   # builds the context, kept afterwards
    b1 = run(moved)            # rebinds it
    a2 = run(meta["solute"])   # rebinds it back
    lib().rism3d_cache_clear()
    b0 = run(moved)            # a fresh context
    c0 = run(moved, dict(s, **{"norm-tol": 1e-11}))  # other settings: another context
    lib().rism3d_cache_clear()
    for x, y in ((a1, a2), (b0, b1)):
        assert x["free-energy"] == y["free-energy"]
        assert np.array_equal(x["GUV"], y["GUV"]) and np.array_equal(x["RESTART"], y["RESTART"])
    assert abs(a1["free-energy"] - b1["free-energy"]) > 1e-6
    assert abs(c0["free-energy"] - b0["free-energy"]) < 1e-8
