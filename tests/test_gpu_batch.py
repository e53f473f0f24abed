"""Batched solves (rism3d_solve_batch): solutes of uneven site counts, grids,
boxes and closures solved concurrently by several host workers, each on its
own stream.  Every job reaches the oracle's root as its single solve does
(mu to 1e-6 kcal/mol, t to 1e-10 max-abs), and one job's failure is
reported in its own status without disturbing the others.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from bgy3d_b200 import hnc3d_run_batch  # noqa: E402
from oracle import hnc3d  # noqa: E402

CASES = ["water_hnc_n24", "water_hnc_norenorm_n24", "na_kh_n32", "synth6_kh_n32", "synth6_pse3_n32"]


def settings_of(meta, **kw):
    s = dict(meta["settings"])
    s["closure"] = int(s["closure"])
    s.update(kw)
    return s


def test_batch_matches_oracle(fixture_loader):
    # one batch has one solvent: the fixtures in PR-SPC/E water (na_kh_n32's
    # is cSPC/E)
    cases = [fixture_loader(n) for n in CASES]
    solvent = cases[0][0]["solvent"]
    cases = [(meta, arr) for meta, arr in cases if meta["solvent"] == solvent]
    assert len(cases) == 4
    jobs = [(meta, arr, prec) for prec in ("fp64", "mixed") for meta, arr in cases]
    res = hnc3d_run_batch([meta["solute"] for meta, _, _ in jobs], solvent,
                          [settings_of(meta, **{"norm-tol": 1e-12, "precision": p}) for meta, _, p in jobs],
                          [arr["chi"] for _, arr, _ in jobs], workers=4, want_g=True,
                          restarts=[np.zeros_like(arr["T"]) for _, arr, _ in jobs])
    assert len(res) == len(jobs)
    for (meta, arr, prec), r in zip(jobs, res):
        assert r["status"] == 0, (meta["settings"], prec)
        assert r["resid-inf"] < 1e-12
        assert abs(r["free-energy"] - meta["mu"]) < 1e-6
        assert np.max(np.abs(r["RESTART"] - arr["T"])) < 1e-10
    meta, arr, _ = jobs[0]
    s = meta["settings"]
    P = hnc3d.Problem((s["N"],) * 3, (2 * s["L"],) * 3, s["beta"], s["rho"], int(s["closure"]), meta["solvent"],
                      meta["solute"], arr["chi"], s["rmax"], renorm=not s["no-renorm"])
    assert np.max(np.abs(res[0]["GUV"] - P.observables(arr["T"])["g"])) < 1e-10


def test_batch_reports_each_job(fixture_loader):
    meta, arr = fixture_loader("synth6_kh_n32")
    good = settings_of(meta, **{"norm-tol": 1e-10})
    bad = settings_of(meta, **{"norm-tol": 1e-12, "max-iter": 1})
    res = hnc3d_run_batch([meta["solute"]] * 3, meta["solvent"], [good, bad, good], arr["chi"], workers=3)
    assert [r["status"] for r in res] == [0, -5, 0]
    assert abs(res[0]["free-energy"] - meta["mu"]) < 1e-6
    assert abs(res[2]["free-energy"] - meta["mu"]) < 1e-6
