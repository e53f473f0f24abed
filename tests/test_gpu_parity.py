"""Parity of the sm_100a path (through the C ABI) with the CPU oracle.

Tolerances: FP64 residual/Jacobian evaluations agree with the oracle to
1e-11 of their scale (FFT round-off only); converged FP64 solves agree in t
and g to 1e-10 max-abs and in mu to 1e-6 kcal/mol; FP32 evaluations to
2e-5 relative; the mixed-precision solve reaches the same FP64 residual
tolerance and its mu agrees with the FP64 one to 1e-4 kcal/mol.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from bgy3d_b200 import RismContext, hnc3d_run_solute  # noqa: E402
from bgy3d_b200 import _abi  # noqa: E402
from oracle import closures as cl  # noqa: E402
from oracle import hnc3d  # noqa: E402

CASES = ["water_hnc_n24", "water_hnc_norenorm_n24", "na_kh_n32", "synth6_kh_n32", "synth6_pse3_n32"]


def settings_of(meta, **kw):
    s = dict(meta["settings"])
    s["closure"] = int(s["closure"])
    s.update(kw)
    return s


def oracle_problem(meta, chi):
    s = meta["settings"]
    N = (s["N"],) * 3
    return hnc3d.Problem(N, (2 * s["L"],) * 3, s["beta"], s["rho"], int(s["closure"]), meta["solvent"],
                         meta["solute"], chi, s["rmax"], renorm=not s["no-renorm"])


def to_dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


@pytest.fixture(scope="module", params=CASES)
def case(request, fixture_loader):
    meta, arr = fixture_loader(request.param)
    ctx = RismContext(meta["solute"], meta["solvent"], settings_of(meta), arr["chi"])
    yield request.param, meta, arr, ctx
    ctx.close()


def test_solute_field_matches_oracle(case):
    name, meta, arr, ctx = case
    P = oracle_problem(meta, arr["chi"])
    v = ctx.field(0).cpu().numpy()
    assert np.max(np.abs(v - P.v) / np.maximum(1.0, np.abs(P.v))) < 1e-12


def test_iterate_t1_matches_oracle(case):
    name, meta, arr, ctx = case
    P = oracle_problem(meta, arr["chi"])
    rng = np.random.default_rng(7)
    T = 0.3 * rng.standard_normal(ctx.shape)
    F_ref = P.iterate_t1(T)
    F, (rinf, r2) = ctx.iterate_t1(to_dev(T))
    F = F.cpu().numpy()
    scale = np.max(np.abs(F_ref))
    assert np.max(np.abs(F - F_ref)) < 1e-11 * scale
    assert abs(rinf - np.max(np.abs(F_ref))) < 1e-11 * scale
    assert abs(r2 - np.linalg.norm(F_ref)) < 1e-10 * np.linalg.norm(F_ref)
    # FP32 form of the same evaluation
    F32, _ = ctx.iterate_t1(to_dev(T, torch.float32))
    assert np.max(np.abs(F32.cpu().numpy() - F_ref)) < 2e-5 * scale


def test_jacobian_t1_matches_oracle(case):
    name, meta, arr, ctx = case
    if int(meta["settings"]["closure"]) == cl.PY:
        pytest.skip("PY has no Jacobian")
    P = oracle_problem(meta, arr["chi"])
    rng = np.random.default_rng(11)
    T = 0.3 * rng.standard_normal(ctx.shape)
    dT = rng.standard_normal(ctx.shape)
    J_ref = P.jacobian_t1(T, dT)
    J = ctx.jacobian_t1(to_dev(T), to_dev(dT)).cpu().numpy()
    scale = np.max(np.abs(J_ref))
    assert np.max(np.abs(J - J_ref)) < 1e-11 * scale
    J32 = ctx.jacobian_t1(to_dev(T, torch.float32), to_dev(dT, torch.float32)).cpu().numpy()
    assert np.max(np.abs(J32 - J_ref)) < 2e-5 * scale


def test_jacobian_is_linear(case):
    name, meta, arr, ctx = case
    rng = np.random.default_rng(3)
    T = to_dev(0.2 * rng.standard_normal(ctx.shape))
    x = to_dev(rng.standard_normal(ctx.shape))
    y = to_dev(rng.standard_normal(ctx.shape))
    Jx = ctx.jacobian_t1(T, x)
    Jy = ctx.jacobian_t1(T, y)
    Jxy = ctx.jacobian_t1(T, (2.5 * x - 0.75 * y).contiguous())
    err = (Jxy - (2.5 * Jx - 0.75 * Jy)).abs().max().item()
    assert err < 1e-12 * Jxy.abs().max().item()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_matches_oracle(case, precision):
    name, meta, arr, ctx = case
    ctx2 = RismContext(meta["solute"], meta["solvent"],
                       settings_of(meta, **{"norm-tol": 1e-12, "precision": precision}), arr["chi"])
    T, res = ctx2.solve()
    assert res["status"] == 0, res
    assert res["resid-inf"] < 1e-12
    obs = ctx2.observables(T, want_g=True)
    assert abs(obs["free-energy"] - meta["mu"]) < 1e-6
    for k in ("HNC", "KH", "GF"):
        assert abs(obs["mu-" + k.lower()] - meta["mu_all"][k]) < 1e-6
    assert abs(obs["partial-molar-volume-factor"] - meta["pmv"]) < 1e-6
    Tn = T.cpu().numpy()
    assert np.max(np.abs(Tn - arr["T"])) < 1e-10
    # g = h + 1 = c(t) + t + 1 against the oracle's g from its own t
    P = oracle_problem(meta, arr["chi"])
    g_ref = P.observables(arr["T"])["g"]
    assert np.max(np.abs(obs["GUV"].cpu().numpy() - g_ref)) < 1e-10
    if precision == "mixed":
        assert res["jv-evals-fp32"] > 0
    ctx2.close()


@pytest.fixture(scope="module")
def static_cases(fixture_loader):
    """Grids served by the shape-specialised (TMA) passes: the README water
    case at 96^3 and a 5-site synthetic solute at 128^3."""
    from bgy3d_b200 import find_molecule, rism_solvent, synthetic_solute
    meta, arr = fixture_loader("water_readme_n96")
    out = [(meta["solute"], meta["solvent"], settings_of(meta), arr["chi"])]
    water = find_molecule("water, PR-SPC/E")
    s = {"L": 16.0, "N": 128, "rho": 0.0333295, "beta": 1.6889, "closure": "KH", "rmax": 40.0,
         "nrad": 1024, "dielectric": 78.4}
    chi = rism_solvent(water, dict(s, **{"norm-tol": 1e-12}))["susceptibility"]
    out.append((synthetic_solute(5, radius=3.0, seed=20261204), water, s, chi))
    return out


@pytest.mark.parametrize("which", [0, 1])
def test_static_passes_match_oracle(static_cases, which, monkeypatch):
    solute, solvent, s, chi = static_cases[which]
    ctx = RismContext(solute, solvent, s, chi)
    monkeypatch.setenv("RISM3D_GENERIC_PASSES", "1")
    gen = RismContext(solute, solvent, s, chi)
    monkeypatch.delenv("RISM3D_GENERIC_PASSES")
    N = s["N"]
    clo = cl.NAMES[s["closure"]] if isinstance(s["closure"], str) else int(s["closure"])
    P = hnc3d.Problem((N,) * 3, (2 * s["L"],) * 3, s["beta"], s["rho"], clo, solvent, solute, chi, s["rmax"])
    rng = np.random.default_rng(5)
    T = 0.3 * rng.standard_normal(ctx.shape)
    dT = rng.standard_normal(ctx.shape)
    F_ref = P.iterate_t1(T)
    J_ref = P.jacobian_t1(T, dT)
    for dt, tol in ((torch.float64, 1e-11), (torch.float32, 2e-5)):
        F = ctx.iterate_t1(to_dev(T, dt))[0].double().cpu().numpy()
        J = ctx.jacobian_t1(to_dev(T, dt), to_dev(dT, dt)).double().cpu().numpy()
        assert np.max(np.abs(F - F_ref)) < tol * np.max(np.abs(F_ref)), dt
        assert np.max(np.abs(J - J_ref)) < tol * np.max(np.abs(J_ref)), dt
        Fg = gen.iterate_t1(to_dev(T, dt))[0].double().cpu().numpy()
        assert np.max(np.abs(F - Fg)) < tol * np.max(np.abs(F_ref)), dt
    ctx.close()
    gen.close()


def test_host_entry_point_and_restart(fixture_loader):
    meta, arr = fixture_loader("water_hnc_n24")
    s = settings_of(meta, **{"norm-tol": 1e-12})
    out = hnc3d_run_solute(meta["solute"], meta["solvent"], s, arr["chi"])
    assert abs(out["free-energy"] - meta["mu"]) < 1e-6
    assert np.max(np.abs(out["RESTART"] - arr["T"])) < 1e-10
    again = hnc3d_run_solute(meta["solute"], meta["solvent"], s, arr["chi"], restart=out["RESTART"])
    assert again["newton-iters"] <= 1
    assert abs(again["free-energy"] - out["free-energy"]) < 1e-9


def test_readme_water_96(fixture_loader):
    meta, arr = fixture_loader("water_readme_n96")
    for precision in ("fp64", "mixed"):
        out = hnc3d_run_solute(meta["solute"], meta["solvent"],
                               settings_of(meta, **{"norm-tol": 1e-10, "precision": precision}),
                               arr["chi"], want_g=False)
        assert abs(out["free-energy"] - meta["mu"]) < 1e-6
        assert round(out["free-energy"], 6) == -6.349052


@pytest.mark.parametrize("opts", [{"coarse-h": 0, "ew-forcing": 0}, {"coarse-h": 0}, {"krylov-restart": 8},
                                  {"coarse-steps": 4, "precision": "mixed"}])
def test_krylov_options_reach_the_same_root(fixture_loader, opts):
    """The Krylov options change the path to the root, never the root."""
    meta, arr = fixture_loader("synth6_kh_n32")
    out = hnc3d_run_solute(meta["solute"], meta["solvent"],
                           settings_of(meta, **{"norm-tol": 1e-12, **opts}), arr["chi"])
    assert out["resid-inf"] < 1e-12
    assert abs(out["free-energy"] - meta["mu"]) < 1e-6
    assert np.max(np.abs(out["RESTART"] - arr["T"])) < 1e-10


def test_picard_and_trial_solvers(fixture_loader):
    meta, arr = fixture_loader("water_hnc_n24")
    for solver in ("trial",):
        out = hnc3d_run_solute(meta["solute"], meta["solvent"],
                               settings_of(meta, **{"norm-tol": 1e-11, "snes-solver": solver}), arr["chi"])
        assert abs(out["free-energy"] - meta["mu"]) < 1e-6


def test_jager_mixing_follows_the_reference_rule(fixture_loader):
    """60 iterations of the adaptive mixing (bgy3d_snes_jager) from t = 0
    land on the oracle's iterate of the same rule."""
    from oracle import hnc3d, newton
    meta, arr = fixture_loader("water_hnc_n24")
    s = settings_of(meta, **{"snes-solver": "jager", "lambda": 0.1, "max-iter": 60, "norm-tol": 1e-14})
    ctx = RismContext(meta["solute"], meta["solvent"], s, arr["chi"])
    T, res = ctx.solve(ctx.zeros())
    ctx.close()
    assert res["newton-iters"] == 60 and res["status"] == _abi.ERR_NOT_CONVERGED
    N, L = (s["N"],) * 3, (2 * s["L"],) * 3
    P = hnc3d.Problem(N, L, s["beta"], s["rho"], s["closure"], meta["solvent"], meta["solute"], arr["chi"],
                      s["rmax"])
    x, its, norm = newton.jager(P.iterate_t1, np.zeros((3,) + N), 0.1, 60, 1e-14)
    assert its == 60
    assert np.max(np.abs(T.cpu().numpy() - x)) < 1e-10 * max(1.0, np.max(np.abs(x)))


def test_errors_are_status_codes(fixture_loader):
    meta, arr = fixture_loader("water_hnc_n24")
    # not converged: max-iter = 1
    with pytest.raises(_abi.RismError) as e:
        hnc3d_run_solute(meta["solute"], meta["solvent"],
                         settings_of(meta, **{"norm-tol": 1e-12, "max-iter": 1}), arr["chi"])
    assert e.value.code == _abi.ERR_NOT_CONVERGED
    # NaN in the initial guess
    bad = np.zeros((3, 24, 24, 24))
    bad[1, 3, 4, 5] = np.nan
    ctx = RismContext(meta["solute"], meta["solvent"], settings_of(meta), arr["chi"])
    T, res = ctx.solve(to_dev(bad))
    assert res["status"] == _abi.ERR_NAN
    ctx.close()
    # the device context is still usable afterwards
    out = hnc3d_run_solute(meta["solute"], meta["solvent"], settings_of(meta, **{"norm-tol": 1e-10}),
                           arr["chi"], want_g=False)
    assert abs(out["free-energy"] - meta["mu"]) < 1e-6
