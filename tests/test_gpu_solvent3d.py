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
