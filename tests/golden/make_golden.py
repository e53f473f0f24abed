"""Generate the golden fixtures under tests/golden/ from the CPU oracle.

    python tests/golden/make_golden.py

Each fixture holds the inputs of one solute solve (sites, settings, the 1D
chi) and the oracle's outputs: the converged t (small grids only), the
chemical potentials by the native/HNC/KH/GF functionals and the PMV factor.
The oracle itself is pinned to the reference's published values by
tests/test_oracle_goldens.py.
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from bgy3d_b200.sites import find_molecule, synthetic_solute  # noqa: E402
from oracle import closures as cl  # noqa: E402
from oracle import hnc3d, rism1d  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def chi_1d(solvent, closure, rmax, nrad, beta, rho, eps):
    return rism1d.rism_vv(closure, nrad, rmax, beta, rho, solvent, eps=eps, tol=1e-12)["chi"]


def case(name, solute, solvent, N, Lhalf, closure, rmax, nrad, beta=1.6889, rho=0.0333295, eps=78.4,
         renorm=True, keep_t=True, tol=1e-12, picard=0):
    chi = chi_1d(solvent, closure, rmax, nrad, beta, rho, eps)
    out = hnc3d.solute_solve((N,) * 3, (2.0 * Lhalf,) * 3, beta, rho, closure, solvent, solute, chi,
                             rmax, renorm=renorm, tol=tol, picard_steps=picard)
    settings = {"L": Lhalf, "N": N, "rho": rho, "beta": beta, "closure": closure, "rmax": rmax,
                "nrad": nrad, "no-renorm": not renorm, "dielectric": eps}
    meta = {"settings": settings, "solute": solute, "solvent": solvent,
            "mu": out["mu"], "mu_all": out["mu_all"], "pmv": out["pmv"], "iters": out["iters"]}
    arrays = {"chi": chi}
    if keep_t:
        arrays["T"] = out["T"]
    T = out["T"]
    arrays["T_checksums"] = np.array([T.sum(), (T ** 2).sum(), np.abs(T).max()])
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **arrays)
    with open(os.path.join(OUT, name + ".json"), "w") as f:
        json.dump(meta, f, indent=1, default=float)
    print(name, out["mu"], out["mu_all"], out["pmv"])


if __name__ == "__main__":
    only = set(sys.argv[1:])  # fixture names to (re)generate; none: all
    if only:
        _case = case

        def case(name, *a, **k):
            if name in only:
                _case(name, *a, **k)
    water = find_molecule("water, PR-SPC/E")
    cspce = find_molecule("water, cSPC/E")
    # water in water, HNC, renorm and no-renorm, 24^3 in a 16 A box
    case("water_hnc_n24", water, water, 24, 8.0, cl.HNC, 32.0, 384)
    case("water_hnc_norenorm_n24", water, water, 24, 8.0, cl.HNC, 32.0, 384, renorm=False)
    # charged solute (renormalised long range with net charge), KH
    case("na_kh_n32", find_molecule("Na+, JC08, SPC/E"), cspce, 32, 8.0, cl.KH, 32.0, 512)
    # synthetic 6-site neutral solute, KH and PSE3, non-trivial geometry
    syn = synthetic_solute(6, radius=3.0, seed=20261203)
    case("synth6_kh_n32", syn, water, 32, 9.0, cl.KH, 36.0, 512)
    case("synth6_pse3_n32", syn, water, 32, 9.0, cl.PSE0 + 3, 36.0, 512)
    # the README 3D example (--L 10 --N 96, chi from the upscaled 1D grid):
    # mu only, t is too large to commit
    case("water_readme_n96", water, water, 96, 10.0, cl.HNC, 40.0, 1536, keep_t=False, tol=1e-11)
    # configuration 0 as written: chi from 1D DRISM/HNC at rmax 160 / nrad
    # 4096, 96^3 in a 20 A box, to the tightest FP64 residual both sides
    # reach (mu and checksums only; the GPU test re-runs this oracle solve)
    case("water_config0_n96", water, water, 96, 10.0, cl.HNC, 160.0, 4096, keep_t=False, tol=1e-13)
