"""The library's 1D RISM/DRISM chi producer (rism1d_solvent_chi, CPU code)
against the oracle restatement of rism_vv (rism.f90:310-583)."""
import numpy as np
import pytest

from bgy3d_b200 import find_molecule, rism_solvent
from oracle import closures as cl
from oracle import rism1d

WATER = find_molecule("water, PR-SPC/E")


@pytest.mark.parametrize("rmax,nrad,closure,eps", [
    (10.0, 96, cl.HNC, 78.4),      # the README 3D example's default radial grid
    (40.0, 1536, cl.HNC, 78.4),    # the grid hnc3d_solute_solve upscales to
    (32.0, 512, cl.KH, 78.4),
    (20.0, 256, cl.HNC, 0.0),      # plain RISM, no dielectric correction
    (160.0, 4096, cl.HNC, 78.4),   # the grid every benchmark configuration uses (README:16 solvent)
    (160.0, 4096, cl.KH, 78.4),    # the chi of the benched 256^3 KH workload
])
def test_chi_matches_oracle(rmax, nrad, closure, eps):
    s = {"rmax": rmax, "nrad": nrad, "rho": 0.0333295, "beta": 1.6889, "dielectric": eps,
         "closure": closure, "norm-tol": 1e-12}
    got = rism_solvent(WATER, s)
    ref = rism1d.rism_vv(closure, nrad, rmax, 1.6889, 0.0333295, WATER, eps=eps, tol=1e-12)
    assert np.max(np.abs(got["susceptibility"] - ref["chi"])) < 1e-9
    assert abs(got["free-energy"] - ref["mu"]) < 1e-8


def test_single_site_solvent():
    lj = [dict(name="A", x=(0.0, 0.0, 0.0), sigma=3.0, epsilon=0.2, charge=0.0)]
    s = {"rmax": 20.0, "nrad": 256, "rho": 0.02, "beta": 1.6889, "closure": cl.HNC, "norm-tol": 1e-12}
    got = rism_solvent(lj, s)
    ref = rism1d.rism_vv(cl.HNC, 256, 20.0, 1.6889, 0.02, lj, tol=1e-12)
    assert np.max(np.abs(got["susceptibility"] - ref["chi"])) < 1e-9
