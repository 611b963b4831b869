"""Build libm3dgpu.so in-tree for sm_100a with nvcc.

The library is compiled with -fmad=false: every fused multiply-add in the
kernels is an explicit fmaf()/fma(), which fixes the evaluation order of the
FP32 path.  The host compiler gets -ffp-contract=off for the same reason (the
QLG tables and the rotation/stencil coefficients are formed on the host).
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libm3dgpu.so")
SOURCES = ["m3d_api.cu"]


def _deps() -> list[str]:
    """Every file the library is built from: all of csrc/ and the public header."""
    files = [f for f in glob.glob(os.path.join(CSRC, "*")) if os.path.isfile(f)]
    return sorted(files) + [os.path.join(ROOT, "include", "m3dgpu.h")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
           "-fmad=false", "--shared", "-Xcompiler", "-fPIC,-ffp-contract=off", "-cudart", "static",
           "-I", os.path.join(ROOT, "include"), "-o", LIB + ".tmp"]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
