"""The pass-schedule autotuner (rism3d_tile_shapes): the timed tile shapes
only reschedule the same column transforms, so the residual and Jacobian
products are bitwise those of the register / occupancy rule when both run
the same pass family, and agree to rounding when the tuner swaps the
shape-specialised passes for the runtime-length ones."""
import os

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


def make(meta, arr, s, tuned):
    old = os.environ.get("RISM3D_AUTOTUNE")
    os.environ["RISM3D_AUTOTUNE"] = "1" if tuned else "0"
    try:
        return RismContext(meta["solute"], meta["solvent"], s, arr["chi"])
    finally:
        if old is None:
            del os.environ["RISM3D_AUTOTUNE"]
        else:
            os.environ["RISM3D_AUTOTUNE"] = old


@pytest.mark.parametrize("N", [32, 48, 64, 108])
def test_tuned_schedule_matches_rule(fixture_loader, N):
    meta, arr = fixture_loader("synth6_kh_n32")
    s = settings_of(meta, N=N, L=12.0, **{"coarse-h": 0})
    a, b = make(meta, arr, s, True), make(meta, arr, s, False)
    ta, tb = a.tile_shapes(), b.tile_shapes()
    for prec in ("f64", "f32"):
        assert all(k in (1, 2, 4, 8, 16, 32) for k in ta[prec][:3])
    g = torch.Generator(device="cuda").manual_seed(11)
    for dt in (torch.float64, torch.float32):
        T = (torch.randn(a.shape, generator=g, device="cuda", dtype=torch.float64) * 0.1).to(dt)
        dT = (torch.randn(a.shape, generator=g, device="cuda", dtype=torch.float64) * 0.1).to(dt)
        Fa, _ = a.iterate_t1(T)
        Fb, _ = b.iterate_t1(T)
        Ja, Jb = a.jacobian_t1(T, dT), b.jacobian_t1(T, dT)
        prec = "f64" if dt == torch.float64 else "f32"
        same_family = ta[prec][3] == tb[prec][3]
        for x, y in ((Fa, Fb), (Ja, Jb)):
            x, y = x.double().cpu().numpy(), y.double().cpu().numpy()
            if same_family:
                assert np.array_equal(x, y)
            else:
                tol = 1e-11 if dt == torch.float64 else 2e-5
                assert np.max(np.abs(x - y)) <= tol * max(1.0, np.max(np.abs(y)))
    a.close()
    b.close()


@pytest.mark.parametrize("N", [48, 96, 256])
def test_persistent_z_pass_is_bitwise(fixture_loader, N, monkeypatch):
    """The persistent double-buffered z pass computes the same tiles as the
    one-tile-per-CTA pass: identical F and J.v, FP64 and FP32."""
    meta, arr = fixture_loader("synth6_kh_n32")
    s = settings_of(meta, N=N, L=12.0 if N <= 128 else 36.0, **{"coarse-h": 0})  # |k| inside the chi table
    monkeypatch.setenv("RISM3D_Z_PERSISTENT", "1")
    a = RismContext(meta["solute"], meta["solvent"], s, arr["chi"])
    monkeypatch.setenv("RISM3D_Z_PERSISTENT", "0")
    b = RismContext(meta["solute"], meta["solvent"], s, arr["chi"])
    ta, tb = a.tile_shapes(), b.tile_shapes()
    assert ta["f32"][4] < 0 and ta["f64"][4] < 0 and tb["f32"][4] > 0
    g = torch.Generator(device="cuda").manual_seed(3)
    for dt in (torch.float64, torch.float32):
        T = (torch.randn(a.shape, generator=g, device="cuda", dtype=torch.float64) * 0.1).to(dt)
        dT = (torch.randn(a.shape, generator=g, device="cuda", dtype=torch.float64) * 0.1).to(dt)
        assert torch.equal(a.iterate_t1(T)[0], b.iterate_t1(T)[0])
        assert torch.equal(a.jacobian_t1(T, dT), b.jacobian_t1(T, dT))
    a.close()
    b.close()
