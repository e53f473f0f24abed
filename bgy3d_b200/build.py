"""Build librism3d.so (the C-ABI library of include/rism3d.h) in-tree for sm_100a.

    python -m bgy3d_b200.build [--verbose-ptxas]

nvcc cross-compiles without a GPU; the .so lands next to this file so it
travels with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "librism3d.so")
SOURCES = ["rism3d.cu", "twogrid_fx2.cu", "twogrid_yz.cu", "twogrid_tc.cu", "coarse_pk.cu", "rism1d.cpp", "noalloc.cu"]
HEADERS = ["fft_core.cuh", "kernels.cuh", "fft_static.cuh", "kernels_static.cuh", "krylov.cuh", "twogrid.cuh",
           "twogrid_fft.cuh", "grad.cuh", "solvent.cuh", "info.cuh", "coarse_pk.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "rism3d.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose_ptxas=False):
    if not force and not _stale() and not verbose_ptxas:
        return LIB
    # per-thread default streams: host threads of the batch driver issue
    # independently; each still orders against torch's legacy stream
    flags = ["-O3", "-std=c++17", "-lineinfo", "--default-stream", "per-thread",
             "-gencode", "arch=compute_100a,code=sm_100a",
             "-Xcompiler", "-fPIC,-O3",
             "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    if verbose_ptxas:
        flags.insert(0, "-Xptxas=-v")
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = [os.path.join(objdir, os.path.splitext(s)[0] + ".o") for s in SOURCES]
    # one nvcc per source, concurrently (the translation units share no device code)
    procs = [subprocess.Popen([NVCC] + flags + ["-c", "-o", o, os.path.join(CSRC, s)])
             for s, o in zip(SOURCES, objs)]
    codes = [p.wait() for p in procs]
    if any(codes):
        raise subprocess.CalledProcessError(max(codes), "nvcc")
    subprocess.run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB + ".tmp"] + objs, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose_ptxas="--verbose-ptxas" in sys.argv)
    print(LIB)
