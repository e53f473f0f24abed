"""rism3d_jacobian_apply_noalloc: the Jacobian product for callers that
cannot allocate device memory, against rism3d_jacobian_t1.

The allocation-free entry point keeps its scratch in a file-scope device
array shared by all calls; it must give the same J dT as the context-based
entry point, call after call.  Tolerance as for the other FP64 Jacobian
tests: 1e-11 of the result's scale.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from bgy3d_b200 import RismContext, _abi  # noqa: E402
from bgy3d_b200.solver import problem_data  # noqa: E402
from tests.conftest import load_fixture  # noqa: E402


def _closure_slope(meta, v, T):
    """dc/dt of the fixture's closure at (v, T), computed with torch."""
    beta = meta["settings"]["beta"]
    x = -beta * v + T
    closure = int(meta["settings"]["closure"])
    if closure == 0:  # HNC
        return torch.expm1(x)
    if closure == 1:  # KH
        return torch.where(x <= 0, torch.expm1(torch.clamp(x, max=0.0)), torch.zeros_like(x))
    raise ValueError("fixture closure not handled here")


@pytest.mark.parametrize("name", ["water_hnc_n24", "na_kh_n32"])
def test_noalloc_jacobian_matches_context_entry_point(name):
    meta, arr = load_fixture(name)
    s = dict(meta["settings"])
    ctx = RismContext(meta["solute"], meta["solvent"], s, arr["chi"])
    rng = np.random.default_rng(17)
    pd = problem_data(s)
    chi = np.ascontiguousarray(arr["chi"], dtype=np.float64)
    v = ctx.field(0)
    L = _abi.lib()
    for call in range(2):  # two calls in a row share the scratch array
        T = torch.from_numpy(0.3 * rng.standard_normal(ctx.shape)).cuda()
        dT = torch.from_numpy(rng.standard_normal(ctx.shape)).cuda()
        ref = ctx.jacobian_t1(T, dT)
        d = _closure_slope(meta, v, T).contiguous()
        out = torch.full_like(dT, float("nan"))
        rc = L.rism3d_jacobian_apply_noalloc(
            ctypes.byref(pd), len(meta["solvent"]), chi.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(dT.data_ptr()), ctypes.c_void_p(out.data_ptr()))
        assert rc == _abi.OK, (call, rc)
        err = (out - ref).abs().max().item()
        assert err < 1e-11 * ref.abs().max().item(), (call, err)
    ctx.close()


def test_noalloc_rejects_grids_beyond_its_scratch():
    meta, arr = load_fixture("water_hnc_n24")
    s = dict(meta["settings"], N=256, L=24.0)
    pd = problem_data(s)
    pd.nrad = arr["chi"].shape[-1]
    pd.rmax = 10.0  # a 384-point table then reaches |k| = 120 / A: only the size check can fail
    chi = np.zeros((3, 3, pd.nrad))
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    rc = _abi.lib().rism3d_jacobian_apply_noalloc(
        ctypes.byref(pd), 3, chi.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), p, p, p)
    assert rc == _abi.ERR_ARG
