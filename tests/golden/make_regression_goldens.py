"""Parse the reference's 3D-RISM regression outputs (test/out/*.hnc3d.g1 and
water.hnc3d.g2) into tests/golden/hnc3d_regression.json.

Each output holds, for a run of test/Makefile:19-31 (--N 96 --L 10 --rho
0.033427745 --beta 1.6889 --norm-tol 1e-12 --closure KH --solvent water
--solvent-3d): the moments of 1 - g for every distribution (the
``moments`` command, guile/bgy3d.scm:1136-1155, 4 digits), the observables
of print_info (bgy3d-potential.c:316-458, 6 digits) and the free energies
of print_chempot (hnc3d.c:674-694).

    python tests/golden/make_regression_goldens.py /path/to/reference
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def parse(path):
    text = open(path, encoding="utf-8").read()
    out = {"moments": [], "mu": {}, "info": {}}
    for block in re.finditer(r';;; Moments from (\S+)\n(\(.*?\)\)\))', text, re.S):
        nums = [float(x) for x in re.findall(r'"(-?[0-9.]+)"', block.group(2))]
        out["moments"].append({"file": block.group(1), "q": nums[0], "d": nums[1:4],
                               "Q": [nums[4:7], nums[7:10], nums[10:13]]})
    for name, val in re.findall(r'# mu = (-?[0-9.]+) kcal \((\w+)\)', text):
        out["mu"][val] = float(name)
    pats = {
        "q_v": r'q_v = (-?[0-9.]+)', "q_u": r'q_u = (-?[0-9.]+)',
        "d_n": r'\|<x\|ρ_n>\| = \|\s*(-?[0-9.]+),\s*(-?[0-9.]+),\s*(-?[0-9.]+)\|',
        "d_u": r'\|<x\|ρ_u>\| = \|\s*(-?[0-9.]+),\s*(-?[0-9.]+),\s*(-?[0-9.]+)\|',
        "d_v": r'\|<x\|ρ_v>\| = \|\s*(-?[0-9.]+),\s*(-?[0-9.]+),\s*(-?[0-9.]+)\|',
        "U_v_rho_N": r'<U_v\|ρ_N> = (-?[0-9.]+)', "U_v_rho_u": r'<U_v\|ρ_u> = (-?[0-9.]+)',
        "rho_v_U_u": r'<ρ_v\|U_u> = (-?[0-9.]+)',
    }
    for key, pat in pats.items():
        m = re.search(pat, text)
        if m:
            vals = [float(x) for x in m.groups()]
            out["info"][key] = vals if len(vals) > 1 else vals[0]
    return out


def main(ref):
    outdir = os.path.join(ref, "test", "out")
    result = {"settings": {"N": 96, "L": 10.0, "rho": 0.033427745, "beta": 1.6889, "closure": "KH",
                           "norm-tol": 1e-12, "solvent": "water"},
              "solvent": parse(os.path.join(outdir, "water.hnc3d.g2")), "solutes": {}}
    for f in sorted(os.listdir(outdir)):
        if f.endswith(".hnc3d.g1"):
            result["solutes"][f[: -len(".hnc3d.g1")].replace("_", " ")] = parse(os.path.join(outdir, f))
    with open(os.path.join(HERE, "hnc3d_regression.json"), "w") as fh:
        json.dump(result, fh, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
