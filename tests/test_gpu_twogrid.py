"""Two-grid preconditioner of the Newton-Krylov solver (sm_100a path).

M^-1 v = P (J_H^-1 + I) R v - v with band-limited transfers R / P, the
coarse Jacobian J_H built from the restricted closure slope R c'(T), and a
fixed-step GMRES for J_H^-1.  The GPU result is checked against a NumPy
restatement on the oracle's operators at the coarse size; the coarse solve
runs in FP32 on the GPU, so the tolerance is 1e-4 of max|z|.  The
FFT passes at the coarse sizes and the many-solute grids (16^3 ... 192^3) are
checked against the oracle at the usual 1e-11 (FP64) / 2e-5 (FP32), and
solves with the preconditioner on, started from zero, reach the oracle's
root.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from bgy3d_b200 import RismContext, hnc3d_run_solute  # noqa: E402
from oracle import closures as cl  # noqa: E402
from oracle import hnc3d  # noqa: E402


def settings_of(meta, **kw):
    s = dict(meta["settings"])
    s["closure"] = int(s["closure"])
    s.update(kw)
    return s


def problem(meta, chi, n, L=None):
    s = meta["settings"]
    return hnc3d.Problem((n,) * 3, (2 * (L or s["L"]),) * 3, s["beta"], s["rho"], int(s["closure"]), meta["solvent"],
                         meta["solute"], chi, s["rmax"], renorm=not s["no-renorm"])


def to_dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def transfer(n, nc):
    """R [nc][n] and P [n][nc]: keep the modes |k| <= nc/2 (half weight at nc/2)."""
    x = np.arange(nc)[:, None] / nc - np.arange(n)[None, :] / n
    S = sum((0.5 if 2 * abs(k) == nc else 1.0) * np.cos(2 * np.pi * k * x) for k in range(-nc // 2, nc // 2 + 1))
    return S / n, (S / nc).T


def along(A, f):
    """Apply A along the three grid axes of f [m][z][y][x]."""
    f = np.einsum("ai,mzyi->mzya", A, f)
    f = np.einsum("ai,mziy->mzay", A, f)
    return np.einsum("ai,mizy->mazy", A, f)


def gmres_steps(A, b, k):
    """k steps of GMRES from 0 (classical Gram-Schmidt): the coarse solve."""
    beta = np.linalg.norm(b)
    V = [b / beta]
    H = np.zeros((k + 1, k))
    for j in range(k):
        w = A(V[j])
        h = np.array([np.sum(v * w) for v in V])
        w = w - sum(hi * v for hi, v in zip(h, V))
        H[:j + 1, j] = h
        H[j + 1, j] = np.linalg.norm(w)
        V.append(w / H[j + 1, j])
    e = np.zeros(k + 1)
    e[0] = beta
    y = np.linalg.lstsq(H, e, rcond=None)[0]
    return sum(yi * v for yi, v in zip(y, V))


@pytest.mark.parametrize("n", [16, 18, 48, 64, 72, 144, 192])
def test_coarse_sizes_match_oracle(fixture_loader, n):
    """Runtime-length passes (16, 18) and shape-specialised ones (the rest),
    in a 48 A box so that |k| stays inside the fixture's chi table."""
    meta, arr = fixture_loader("water_hnc_n24")
    ctx = RismContext(meta["solute"], meta["solvent"], settings_of(meta, N=n, L=24.0, **{"coarse-h": 0}), arr["chi"])
    P = problem(meta, arr["chi"], n, L=24.0)
    rng = np.random.default_rng(11)
    T = 0.3 * rng.standard_normal(ctx.shape)
    dT = rng.standard_normal(ctx.shape)
    F_ref, J_ref = P.iterate_t1(T), P.jacobian_t1(T, dT)
    for dt, tol in ((torch.float64, 1e-11), (torch.float32, 2e-5)):
        F = ctx.iterate_t1(to_dev(T, dt))[0].double().cpu().numpy()
        J = ctx.jacobian_t1(to_dev(T, dt), to_dev(dT, dt)).double().cpu().numpy()
        assert np.max(np.abs(F - F_ref)) < tol * np.max(np.abs(F_ref)), dt
        assert np.max(np.abs(J - J_ref)) < tol * np.max(np.abs(J_ref)), dt
    ctx.close()


@pytest.mark.parametrize("graph", ["1", "0"])
@pytest.mark.parametrize("name", ["water_hnc_n24", "synth6_kh_n32"])
def test_preconditioner_matches_numpy(fixture_loader, name, graph, monkeypatch):
    """Both coarse-solve drivers: the device-driven one replayed as a CUDA
    graph (default) and the host-driven GMRES (RISM3D_COARSE_GRAPH=0)."""
    monkeypatch.setenv("RISM3D_COARSE_GRAPH", graph)
    meta, arr = fixture_loader(name)
    steps = 12
    ctx = RismContext(meta["solute"], meta["solvent"], settings_of(meta, **{"coarse-steps": steps}), arr["chi"])
    s = meta["settings"]
    N = s["N"]
    nc = ctx.coarse_grid()
    assert nc is not None and nc[0] < N
    R, Pm = transfer(N, nc[0])
    Pc = problem(meta, arr["chi"], nc[0])
    rng = np.random.default_rng(3)
    for T in (arr["T"], 0.5 * rng.standard_normal(ctx.shape)):  # converged and far-off states
        v = rng.standard_normal(ctx.shape)
        z = ctx.precondition(to_dev(T), to_dev(v)).cpu().numpy()
        d = cl.closure1(int(s["closure"]), s["beta"], problem(meta, arr["chi"], N).v, T, np.ones_like(T))
        dH = along(R, d)

        def JH(u):
            return Pc.ifft(Pc.star(Pc.fft(dH * u) * Pc.h3)) * (1.0 / Pc.L3) - u

        rc = along(R, v)
        z_ref = along(Pm, gmres_steps(JH, rc, steps) + rc) - v
        assert np.max(np.abs(z - z_ref)) < 1e-4 * np.max(np.abs(z_ref))
    ctx.close()


@pytest.mark.parametrize("n, L", [(64, 9.0), (128, 24.0)])
def test_fft_transfers_match_dense(fixture_loader, n, L):
    """At row lengths with shape-specialised transforms the x-axis transfers
    run by FFT; the preconditioner still equals the dense restatement."""
    meta, arr = fixture_loader("synth6_kh_n32")
    steps = 12
    s = settings_of(meta, N=n, L=L, **{"coarse-steps": steps})
    ctx = RismContext(meta["solute"], meta["solvent"], s, arr["chi"])
    nc = ctx.coarse_grid()
    assert nc is not None and nc[0] < n
    R, Pm = transfer(n, nc[0])
    Pc = problem(meta, arr["chi"], nc[0], L=L)
    P = problem(meta, arr["chi"], n, L=L)
    rng = np.random.default_rng(8)
    T = 0.3 * rng.standard_normal(ctx.shape)
    v = rng.standard_normal(ctx.shape)
    z = ctx.precondition(to_dev(T), to_dev(v)).cpu().numpy()
    d = cl.closure1(int(meta["settings"]["closure"]), meta["settings"]["beta"], P.v, T, np.ones_like(T))
    dH = along(R, d)

    def JH(u):
        return Pc.ifft(Pc.star(Pc.fft(dH * u) * Pc.h3)) * (1.0 / Pc.L3) - u

    rc = along(R, v)
    z_ref = along(Pm, gmres_steps(JH, rc, steps) + rc) - v
    assert np.max(np.abs(z - z_ref)) < 1e-4 * np.max(np.abs(z_ref))
    ctx.close()


@pytest.mark.parametrize("name", ["water_hnc_n24", "synth6_kh_n32", "synth6_pse3_n32"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_preconditioned_solve_reaches_the_root(fixture_loader, name, precision):
    meta, arr = fixture_loader(name)
    out = hnc3d_run_solute(meta["solute"], meta["solvent"],
                           settings_of(meta, **{"norm-tol": 1e-12, "precision": precision}), arr["chi"])
    assert out["jv-evals-coarse"] > 0
    assert out["resid-inf"] < 1e-12
    assert abs(out["free-energy"] - meta["mu"]) < 1e-6
    assert np.max(np.abs(out["RESTART"] - arr["T"])) < 1e-10


@pytest.mark.parametrize("N, L", [((512, 48, 48), (48.0, 4.5, 4.5)), ((256, 48, 48), (24.0, 4.5, 4.5))])
def test_fft_transfers_match_dense_long_rows(fixture_loader, N, L, monkeypatch):
    """256- and 128-point half rows: the preconditioner with the FFT x
    transfers (both sides by FFT, and the coarse side by table product,
    RISM3D_DENSE_TRANSFERS=2) equals the one with the dense transfer tiles."""
    meta, arr = fixture_loader("synth6_kh_n32")
    s = settings_of(meta, N=list(N), L=list(L))
    rng = np.random.default_rng(9)
    out = []
    for dense in ("0", "2", "1"):
        monkeypatch.setenv("RISM3D_DENSE_TRANSFERS", dense)
        ctx = RismContext(meta["solute"], meta["solvent"], s, arr["chi"])
        assert ctx.coarse_grid() is not None
        if not out:
            T = to_dev(0.3 * rng.standard_normal(ctx.shape))
            v = to_dev(rng.standard_normal(ctx.shape))
        out.append(ctx.precondition(T, v).cpu().numpy())
        ctx.close()
    for z in out[:2]:
        assert np.max(np.abs(z - out[2])) < 1e-4 * np.max(np.abs(out[2]))


@pytest.mark.parametrize("N", [(256, 48, 48), (192, 48, 48), (128, 48, 48)])
def test_tensor_core_transfers(fixture_loader, N, monkeypatch):
    """x rows of 256, 192 and 128 points onto a 64-point coarse axis (a 48 A
    box): the FP32 preconditioner with the x transfers on the tensor cores
    (TF32 products in three terms, hi.hi + hi.lo + lo.hi) equals the one
    with the FFT x transfers (RISM3D_TC_TRANSFERS=0) to FP32 accuracy, and
    the FP64 preconditioner with the dense transfer tiles to the 1e-4 of the
    other preconditioner tests (the coarse solve is FP32 in both)."""
    meta, arr = fixture_loader("synth6_kh_n32")
    s = settings_of(meta, N=list(N), L=[24.0, 4.5, 4.5])
    rng = np.random.default_rng(12)
    out = {}
    for tc in ("1", "0"):
        monkeypatch.setenv("RISM3D_TC_TRANSFERS", tc)
        ctx = RismContext(meta["solute"], meta["solvent"], s, arr["chi"])
        assert ctx.coarse_grid()[0] == 64
        if not out:
            T = 0.3 * rng.standard_normal(ctx.shape)
            v = rng.standard_normal(ctx.shape)
        out[tc] = ctx.precondition(to_dev(T, torch.float32), to_dev(v, torch.float32)).double().cpu().numpy()
        ctx.close()
    monkeypatch.setenv("RISM3D_DENSE_TRANSFERS", "1")
    ctx = RismContext(meta["solute"], meta["solvent"], s, arr["chi"])
    ref = ctx.precondition(to_dev(T), to_dev(v)).cpu().numpy()
    ctx.close()
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(out["1"] - out["0"])) < 2e-5 * scale
    assert np.max(np.abs(out["1"] - ref)) < 1e-4 * scale
    assert np.max(np.abs(out["0"] - ref)) < 1e-4 * scale


@pytest.mark.parametrize("n", [96, 128])
def test_persistent_coarse_solve(fixture_loader, n, monkeypatch):
    """The coarse GMRES as one persistent cooperative kernel (coarse grids
    48^3 and 64^3 of a 48 A box) equals the NumPy restatement and the
    graph-replayed step-by-step kernels, and repeats bitwise."""
    meta, arr = fixture_loader("synth6_kh_n32")
    steps = 16
    s = settings_of(meta, N=n, L=24.0, **{"coarse-steps": steps})
    rng = np.random.default_rng(12)
    out = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("RISM3D_COARSE_PERSIST", mode)
        ctx = RismContext(meta["solute"], meta["solvent"], s, arr["chi"])
        nc = ctx.coarse_grid()
        if not out:
            T = 0.3 * rng.standard_normal(ctx.shape)
            v = rng.standard_normal(ctx.shape)
        z = ctx.precondition(to_dev(T), to_dev(v)).cpu().numpy()
        z2 = ctx.precondition(to_dev(T), to_dev(v)).cpu().numpy()
        out[mode] = (z, z2, ctx.coarse_driver(), nc)
        ctx.close()
    assert out["1"][2] == "persistent" and out["0"][2] == "graph"
    assert np.array_equal(out["1"][0], out["1"][1])
    nc = out["1"][3]
    assert nc[0] == (48 if n == 96 else 64)
    R, Pm = transfer(n, nc[0])
    Pc = problem(meta, arr["chi"], nc[0], L=24.0)
    P = problem(meta, arr["chi"], n, L=24.0)
    d = cl.closure1(int(meta["settings"]["closure"]), meta["settings"]["beta"], P.v, T, np.ones_like(T))
    dH = along(R, d)

    def JH(u):
        return Pc.ifft(Pc.star(Pc.fft(dH * u) * Pc.h3)) * (1.0 / Pc.L3) - u

    rc = along(R, v)
    z_ref = along(Pm, gmres_steps(JH, rc, steps) + rc) - v
    scale = np.max(np.abs(z_ref))
    for mode in ("1", "0"):
        assert np.max(np.abs(out[mode][0] - z_ref)) < 1e-4 * scale, mode


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_persistent_coarse_solve_reaches_the_root(fixture_loader, precision, monkeypatch):
    """Solves with the persistent coarse kernel (128^3, coarse 64^3) reach the
    same root as with the graph-replayed coarse solve."""
    meta, arr = fixture_loader("synth6_kh_n32")
    s = settings_of(meta, N=128, L=24.0, **{"norm-tol": 1e-11, "precision": precision})
    res = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("RISM3D_COARSE_PERSIST", mode)
        ctx = RismContext(meta["solute"], meta["solvent"], s, arr["chi"])
        T, r = ctx.solve()
        obs = ctx.observables(T)
        res[mode] = (T.cpu().numpy(), r, obs["free-energy"], ctx.coarse_driver())
        ctx.close()
    assert res["1"][3] == "persistent" and res["0"][3] == "graph"
    for mode in ("1", "0"):
        assert res[mode][1]["status"] == 0 and res[mode][1]["resid-inf"] < 1e-11
    assert abs(res["1"][2] - res["0"][2]) < 1e-8
    assert np.max(np.abs(res["1"][0] - res["0"][0])) < 1e-9
