"""The C-ABI library builds, loads and exports what include/rism3d.h declares
(no GPU needed; no compute call reaches the device)."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from bgy3d_b200 import _abi, build, problem_data

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rism3d.h")


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _abi.lib()


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rism[13]d_[a-z0-9_]+)\s*\(", src)))


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert names, "no declarations parsed"
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(set(_abi.EXPORTS)) == sorted(set(names))


def test_struct_layout_matches_header(lib):
    prog = r"""
    #include <stdio.h>
    #include <stddef.h>
    #include "rism3d.h"
    int main(void) {
      printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(rism3d_site), sizeof(rism3d_problem),
             sizeof(rism3d_result), offsetof(rism3d_problem, precision),
             offsetof(rism3d_result, seconds), offsetof(rism3d_site, charge),
             offsetof(rism3d_problem, coarse_h), offsetof(rism3d_problem, coarse_steps),
             sizeof(rism3d_job), offsetof(rism3d_job, chi), offsetof(rism3d_job, result));
      return 0;
    }
    """
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(prog)
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        got = [int(x) for x in subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()]
    want = [ctypes.sizeof(_abi.Site), ctypes.sizeof(_abi.Problem), ctypes.sizeof(_abi.Result),
            _abi.Problem.precision.offset, _abi.Result.seconds.offset, _abi.Site.charge.offset,
            _abi.Problem.coarse_h.offset, _abi.Problem.coarse_steps.offset,
            ctypes.sizeof(_abi.Job), _abi.Job.chi.offset, _abi.Job.result.offset]
    assert got == want


def test_problem_defaults_mirror_reference(lib):
    pd = _abi.Problem()
    lib.rism3d_problem_defaults(ctypes.byref(pd), 10.0, 96)
    assert list(pd.N) == [96, 96, 96] and list(pd.L) == [20.0, 20.0, 20.0]
    assert pd.rmax == 10.0 and pd.nrad == 96          # bgy3d-guile.c:328-331
    assert pd.beta == 1.6889 and pd.rho == 0.033427745  # guile/bgy3d.scm:327-328
    assert pd.max_iter == 1500 and pd.norm_tol == 1e-7
    py = problem_data({"L": 10.0, "N": 96})
    assert (py.rmax, py.nrad, py.beta, py.rho) == (pd.rmax, pd.nrad, pd.beta, pd.rho)


def test_bad_arguments_fail_before_the_device(lib):
    site = (_abi.Site * 1)()
    site[0].sigma, site[0].epsilon, site[0].charge = 3.0, 0.1, 0.0
    chi = (ctypes.c_double * (1 * 1 * 64))()
    h = ctypes.c_void_p()
    pd = _abi.Problem()
    lib.rism3d_problem_defaults(ctypes.byref(pd), 10.0, 100)  # 100 is not 2^a 3^b
    pd.nrad = 64
    assert lib.rism3d_ctx_create(ctypes.byref(pd), 1, site, 1, site, chi, ctypes.byref(h)) == _abi.ERR_ARG
    lib.rism3d_problem_defaults(ctypes.byref(pd), 10.0, 32)
    pd.nrad = 64
    assert lib.rism3d_ctx_create(ctypes.byref(pd), 7, site, 1, site, chi, ctypes.byref(h)) == _abi.ERR_ARG
    # the |k| of a 32^3 / 20 A grid reaches 9.4 / A; a 64-point table at
    # rmax = 10 ends at 19.9 / A, one at rmax = 40 ends at 5.0 / A
    pd.rmax, pd.nrad = 40.0, 64
    assert lib.rism3d_ctx_create(ctypes.byref(pd), 1, site, 1, site, chi, ctypes.byref(h)) == _abi.ERR_TABLE
    assert not h.value
    assert lib.rism3d_iterate_t1(None, None, None, None) == _abi.ERR_ARG
