"""The 3D pure-solvent solve (rism3d_solvent_solve, hnc3d_solvent_solve) and
the solute solve on its k-grid susceptibility (rism3d_solute_solve_chi3,
the reference's --solvent-3d).

Parity: the residual iterate_t2 and its Jacobian against the oracle's
restatement (oracle.solvent3d) on the same pair fields; the converged free
energies against the reference's regression outputs test/out/water.hnc3d.g2
(pure water) and test/out/*.hnc3d.g1 (six solutes in it), all printed
digits, and against the oracle's values of the same runs.  The settings
are those of test/Makefile:19-31 (--N 96 --L 10 --rho 0.033427745 --beta
1.6889 --norm-tol 1e-12 --closure KH --solvent water --solvent-3d).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from bgy3d_b200 import RismContext, find_molecule, hnc3d_run_solute, hnc3d_run_solvent  # noqa: E402
from oracle import solvent3d  # noqa: E402

SETTINGS = {"N": 96, "L": 10.0, "rho": 0.033427745, "beta": 1.6889, "norm-tol": 1e-12, "closure": "KH",
            "max-iter": 100}

# test/out/water.hnc3d.g2 (print_chempot of the pure solvent: HNC, KH*, GF)
GOLDEN_SOLVENT = (-4.161039, -5.793348, -9.595354)
# test/out/<solute>.hnc3d.g1
GOLDEN_SOLUTE = {
    "water": (-2.284209, -3.894980, -5.870259),
    "hydrogen chloride": (7.330353, 5.998107, 3.375364),
    "carbon disulfide": (13.646542, 11.493160, 6.983352),
    "methanol": (3.284694, 0.958059, -2.553333),
    "butanoic acid": (21.182314, 17.406944, 9.765351),
    "hexane": (33.090555, 29.070619, 20.420020),
}
# The oracle's values of the same runs (more digits than the goldens print).
ORACLE_SOLVENT = (-4.161039019635813, -5.7933482100063625, -9.595354314186249)
ORACLE_WATER = (-2.284209312055313, -3.894979905403376, -5.8702593428357925)


@pytest.fixture(scope="module")
def solvent_run():
    w = find_molecule("water")
    return w, hnc3d_run_solvent(w, SETTINGS)


def test_iterate_t2_and_jacobian_match_oracle():
    w = find_molecule("water")
    s = dict(SETTINGS, N=32)
    P = solvent3d.SolventProblem((32,) * 3, (20.0,) * 3, s["beta"], s["rho"], 1, w)
    T = P.initial_guess()
    rng = np.random.default_rng(5)
    dT = rng.standard_normal(T.shape) * 0.01
    F_ref = P.iterate_t2(T)
    J_ref = P.jacobian_t2(T, dT)
    ctx = RismContext(None, w, s, None)
    assert ctx.shape == T.shape
    Td = torch.tensor(T, device="cuda")
    F, (rinf, r2) = ctx.iterate_t1(Td)
    F = F.cpu().numpy()
    assert np.max(np.abs(F - F_ref)) < 1e-10 * max(1.0, np.max(np.abs(F_ref)))
    assert abs(rinf - np.max(np.abs(F_ref))) < 1e-10 * max(1.0, rinf)
    J = ctx.jacobian_t1(Td, torch.tensor(dT, device="cuda")).cpu().numpy()
    assert np.max(np.abs(J - J_ref)) < 1e-10 * np.max(np.abs(J_ref))
    ctx.close()


def test_pure_water_matches_goldens(solvent_run):
    _, r = solvent_run
    assert r["status"] == 0 and r["resid-inf"] < 1e-12
    mu = (r["free-energy-all"]["HNC"], r["free-energy-all"]["KH"], r["free-energy-all"]["GF"])
    assert r["free-energy"] == mu[1]  # KH is the native closure
    for got, gold, orc in zip(mu, GOLDEN_SOLVENT, ORACLE_SOLVENT):
        assert abs(got - gold) <= 5e-7 + 1e-12
        assert abs(got - orc) < 1e-8
    chi = r["susceptibility-3d"]
    assert chi.shape == (6, 96, 96, 49)
    assert np.max(np.abs(chi.imag)) < 1e-10  # a symmetric distribution: real up to rounding
    assert np.all(np.isfinite(r["GVV"])) and r["compressibility"] > 0


def regression():
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "hnc3d_regression.json")) as f:
        return json.load(f)


def check_moments(got, gold):
    """4 printed digits: within half a unit of the last one."""
    q, d, Q = got
    assert abs(q - gold["q"]) <= 5e-5 + 1e-9
    assert np.max(np.abs(d - np.array(gold["d"]))) <= 5e-5 + 1e-9
    assert np.max(np.abs(Q - np.array(gold["Q"]))) <= 5e-5 + 1e-9


def test_pure_water_g_moments(solvent_run):
    w, r = solvent_run
    ctx = RismContext(None, w, SETTINGS, None)
    mom = ctx.moments(torch.tensor(r["GVV"], device="cuda"))
    ctx.close()
    pair = {"g00.bin": 0, "g01.bin": 1, "g11.bin": 2, "g02.bin": 3, "g12.bin": 4, "g22.bin": 5}
    gold = regression()["solvent"]["moments"]
    assert len(gold) == 6
    for gm in gold:
        check_moments(mom[pair[gm["file"]]], gm)


@pytest.mark.parametrize("name", list(GOLDEN_SOLUTE))
def test_solutes_in_3d_solvent_match_goldens(solvent_run, name):
    w, r = solvent_run
    out = hnc3d_run_solute(find_molecule(name), w, SETTINGS, r["susceptibility-3d"], want_g=False,
                           want_restart=False)
    assert out["status"] == 0
    mu = (out["mu-hnc"], out["mu-kh"], out["mu-gf"])
    for got, gold in zip(mu, GOLDEN_SOLUTE[name]):
        assert abs(got - gold) <= 5e-7 + 1e-12, (name, mu)
    if name == "water":
        for got, orc in zip(mu, ORACLE_WATER):
            assert abs(got - orc) < 1e-8


@pytest.mark.parametrize("name", list(GOLDEN_SOLUTE))
def test_solute_observables_match_goldens(solvent_run, name):
    """print_info's observables and the moments of 1 - g of the same runs."""
    w, r = solvent_run
    gold = regression()["solutes"][name]
    ctx = RismContext(find_molecule(name), w, SETTINGS, r["susceptibility-3d"])
    T, res = ctx.solve()
    assert res["status"] == 0
    inf = ctx.info(T)
    g = ctx.observables(T, want_g=True)["GUV"]
    mom = ctx.moments(g)
    ctx.close()
    gi = gold["info"]
    tol = 5e-7 + 1e-9  # 6 printed digits
    assert abs(inf["q_u"]) <= tol and abs(inf["q_v"]) <= tol
    for key in ("d_n", "d_u", "d_v"):
        assert np.max(np.abs(inf[key] - np.array(gi[key]))) <= tol, (name, key, inf[key])
    assert abs(inf["U_v_rho_N_trilinear"] - gi["U_v_rho_N"]) <= tol, (name, inf["U_v_rho_N_trilinear"])
    assert abs(inf["U_v_rho_u"] - gi["U_v_rho_u"]) <= tol, (name, inf["U_v_rho_u"])
    assert abs(inf["rho_v_U_u"] - gi["rho_v_U_u"]) <= tol, (name, inf["rho_v_U_u"])
    files = {m["file"]: m for m in gold["moments"]}
    for i in range(3):
        check_moments(mom[i], files["g%d.bin" % i])
    if name == "water":
        # the trigonometric value (the shipped bgy3d_pot_interp) and the rest
        # against the oracle on the same g
        from oracle import info as oinfo
        ref = oinfo.info((96,) * 3, (20.0,) * 3, SETTINGS["rho"], w, find_molecule(name), g.cpu().numpy())
        for key in ("U_v_rho_N", "U_v_rho_N_trilinear", "U_v_rho_u", "rho_v_U_u", "q_v"):
            assert abs(inf[key] - ref[key]) < 1e-9 * max(1.0, abs(ref[key])), key
        assert np.max(np.abs(inf["Q_v"] - ref["Q_v"])) < 1e-9
        assert np.max(np.abs(inf["site_potential"] - ref["site_potential"])) < 1e-9
