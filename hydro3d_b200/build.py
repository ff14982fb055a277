"""Build the in-tree CUDA library hydro3d_b200/libh3dmg.so for sm_100a.

    python -m hydro3d_b200.build        (or __graft_entry__.build())

nvcc cross-compiles without a GPU.  The library is built with --fmad=false:
the FP64 path reproduces the reference's arithmetic (no contraction into
fused multiply-adds), which the parity tests check bit for bit.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libh3dmg.so")
BUILD = os.path.join(ROOT, "_build")

SOURCES = ["h3d_halo.cpp", "h3d_kernels.cu", "h3d_mg.cu", "h3d_noalloc.cu"]
HEADERS = ["h3d_internal.h", "h3d_kernels.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-Wall", "-Xcompiler", "-Wno-unused-function"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _host_cxx():
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    return None


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile (incrementally) and link libh3dmg.so.  H3D_BOUNDS_CHECK=1 in the
    environment builds the bounds-checked debug variant."""
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    ccbin = _host_cxx()
    base = [nvcc] + ARCH + NVFLAGS + (["-ccbin", ccbin] if ccbin else [])
    if ptxas_info:
        base += ["-Xptxas", "-v"]
    debug = os.environ.get("H3D_BOUNDS_CHECK") == "1"
    if debug:
        base += ["-DH3D_BOUNDS_CHECK"]
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "h3d_mg.h")]
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + (".dbg.o" if debug else ".o"))
        objs.append(o)
        if ptxas_info or debug or _stale(o, [s, __file__] + hdrs):
            cmd = base + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    stamp = os.path.join(BUILD, "flavor")
    flavor = "debug" if debug else "release"
    last = open(stamp).read() if os.path.exists(stamp) else ""
    if last != flavor or _stale(OUT, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", OUT] + objs + (["-ccbin", ccbin] if ccbin else []) + \
            ["-cudart", "static"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        with open(stamp, "w") as f:
            f.write(flavor)
    return OUT


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
