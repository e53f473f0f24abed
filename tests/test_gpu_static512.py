"""Shape-specialised passes for 512-point axes (y / z: 16 x 32 two-step
transforms, tiles moved as two 256-row TMA boxes) and 256-point x half
rows: F and J.v against the runtime-length passes on the same inputs."""
import os

import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from bgy3d_b200 import RismContext  # noqa: E402


def settings_of(meta, **kw):
    s = dict(meta["settings"])
    s["closure"] = int(s["closure"])
    s.update(kw)
    return s


def make(meta, arr, s, generic, monkeypatch):
    monkeypatch.setenv("RISM3D_AUTOTUNE", "0")
    if generic:
        monkeypatch.setenv("RISM3D_GENERIC_PASSES", "1")
    else:
        monkeypatch.delenv("RISM3D_GENERIC_PASSES", raising=False)
    return RismContext(meta["solute"], meta["solvent"], s, arr["chi"])


@pytest.mark.parametrize("N", [(512, 512, 512), (512, 256, 256), (256, 512, 512)])
def test_static_512_matches_generic(fixture_loader, N, monkeypatch):
    meta, arr = fixture_loader("synth6_kh_n32")
    s = settings_of(meta, N=list(N), L=48.0, **{"coarse-h": 0})
    a = make(meta, arr, s, False, monkeypatch)
    b = make(meta, arr, s, True, monkeypatch)
    assert a.tile_shapes()["f64"][3] and not b.tile_shapes()["f64"][3]
    g = torch.Generator(device="cuda").manual_seed(5)
    for dt, tol in ((torch.float64, 1e-12), (torch.float32, 2e-5)):
        T = (torch.randn(a.shape, generator=g, device="cuda", dtype=torch.float64) * 0.1).to(dt)
        dT = (torch.randn(a.shape, generator=g, device="cuda", dtype=torch.float64) * 0.1).to(dt)
        for x, y in ((a.iterate_t1(T)[0], b.iterate_t1(T)[0]), (a.jacobian_t1(T, dT), b.jacobian_t1(T, dT))):
            scale = float(y.double().abs().max())
            assert float((x.double() - y.double()).abs().max()) <= tol * max(1.0, scale)
        del T, dT
    a.close()
    b.close()
    torch.cuda.empty_cache()
