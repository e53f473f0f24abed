"""Generate tests/golden/ions_regression.json: the reference's charged-ion
regression (test/run-ions.scm with its output test/out/run-ions-out) and the
oracle's values at the same settings.

    python tests/golden/make_ion_goldens.py [REFERENCE_ROOT]

Settings of test/run-ions.scm:16-30: cSPC/E water, rho 0.0333295, beta
1.6889, DRISM eps_r 78.4, chi per closure from 1D RISM at rmax 160 A / nrad
4096; 3D on 64^3 in a 20 A box (--L 10) with the renormalised long-range
term, solver "trial" (100 Picard steps at lambda 0.02, then Newton),
norm-tol 1e-14.  Nine JC08 ions x six closures (KH, PSE1, PSE2, PSE3,
PSE7, HNC), 1D and 3D.  The reference's printed values (4 decimals) are
parsed from run-ions-out; the oracle's come from oracle.rism1d.rism_uv and
an oracle 3D solve (residual ||F||_inf below TOL3D, the tightest FP64
reaches for these charged solutes); the chi of every closure goes to
tests/golden/ions_chi.npz.
"""
import json
import os
import re
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from bgy3d_b200.sites import find_molecule  # noqa: E402
from oracle import closures as cl  # noqa: E402
from oracle import hnc3d, newton, rism1d  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ions_regression.json")
# The oracle's chi per closure: the 3D mu of a charged solute moves by up to
# 1e-2 kcal/mol when chi changes by 1e-10 near k = 0 (the renormalised
# long-range term divides by k^2), so parity tests solve on exactly this chi.
OUT_CHI = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ions_chi.npz")
NAMES = ["Li+, JC08, SPC/E", "Na+, JC08, SPC/E", "K+, JC08, SPC/E", "Rb+, JC08, SPC/E", "Cs+, JC08, SPC/E",
         "F-, JC08, SPC/E", "Cl-, JC08, SPC/E", "Br-, JC08, SPC/E", "I-, JC08, SPC/E"]
CLOSURES = ["KH", "PSE1", "PSE2", "PSE3", "PSE7", "HNC"]
SETTINGS = {"rmax": 160.0, "nrad": 4096, "L": 10.0, "N": 64, "rho": 0.0333295, "beta": 1.6889,
            "dielectric": 78.4, "lambda": 0.02, "picard-steps": 100}
TOL3D = 1e-12


def parse_run_ions_out(path):
    """{"RISM-1D": {closure: {ion: value}}, "RISM-3D": {...}} from the
    pretty-printed alist of run-ions.scm."""
    text = open(path).read()
    out = {}
    i1, i3 = text.index("(RISM-1D:"), text.index("(RISM-3D:")
    for key, chunk in (("RISM-1D", text[i1:i3]), ("RISM-3D", text[i3:])):
        table = {}
        # a closure symbol opens a list of ("ion" "value") pairs
        for m in re.finditer(r"\((\w+)\s+((?:\(\"[^\"]+\"\s+\"[-0-9.]+\"\)\s*)+)\)", chunk):
            table[m.group(1)] = {n: float(v) for n, v in re.findall(r"\(\"([^\"]+)\"\s+\"([-0-9.]+)\"\)", m.group(2))}
        out[key] = table
    return out


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    ref = parse_run_ions_out(os.path.join(ref_root, "test", "out", "run-ions-out"))
    s = SETTINGS
    solvent = find_molecule("water, cSPC/E")
    threads = max(1, min(16, os.cpu_count() or 1))
    res = {"settings": s, "tol3d": TOL3D, "solvent": "water, cSPC/E", "names": NAMES, "closures": CLOSURES,
           "reference": ref, "oracle": {"RISM-1D": {}, "RISM-3D": {}}}
    N = (s["N"],) * 3
    L = (2 * s["L"],) * 3
    chis = {}
    for clo in CLOSURES:
        c = cl.NAMES[clo]
        chi = rism1d.rism_vv(c, s["nrad"], s["rmax"], s["beta"], s["rho"], solvent, eps=s["dielectric"],
                             tol=1e-12)["chi"]
        chis[clo] = chi
        res["oracle"]["RISM-1D"][clo] = {}
        res["oracle"]["RISM-3D"][clo] = {}
        for name in NAMES:
            ion = find_molecule(name)
            t0 = time.perf_counter()
            uv = rism1d.rism_uv(c, s["nrad"], s["rmax"], s["beta"], s["rho"], solvent, chi, ion, tol=1e-12)
            P = hnc3d.Problem(N, L, s["beta"], s["rho"], c, solvent, ion, chi, s["rmax"], threads=threads)
            T, _ = newton.solve(P.iterate_t1, np.zeros((3,) + N), jv=P.jacobian_t1, tol=TOL3D,
                                picard_steps=s["picard-steps"], picard_lambda=s["lambda"])
            mu3 = float(P.observables(T)["mu"])
            res["oracle"]["RISM-1D"][clo][name] = float(uv["mu"])
            res["oracle"]["RISM-3D"][clo][name] = mu3
            print(f"{clo:5s} {name:18s} 1D {uv['mu']:.6f} (ref {ref['RISM-1D'][clo][name]:.4f})  "
                  f"3D {mu3:.6f} (ref {ref['RISM-3D'][clo][name]:.4f})  {time.perf_counter() - t0:.1f} s",
                  flush=True)
    with open(OUT, "w") as f:
        json.dump(res, f, indent=1)
    np.savez_compressed(OUT_CHI, **chis)


if __name__ == "__main__":
    main()
