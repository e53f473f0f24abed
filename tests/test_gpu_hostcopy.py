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
