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
TORCH_LIB = os.path.join(HERE, "libm3d_torch.so")
SOURCES = ["m3d_api.cu"]
TORCH_SOURCE = "m3d_torch.cpp"


def _deps() -> list[str]:
    """Every file the library is built from: all of csrc/ and the public header."""
    files = [f for f in glob.glob(os.path.join(CSRC, "*")) if os.path.isfile(f) and not f.endswith(TORCH_SOURCE)]
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


def build_torch(force: bool = False) -> str:
    """libm3d_torch.so: the torch.ops.m3d operators (csrc/m3d_torch.cpp) over the C ABI,
    linked against libm3dgpu.so beside it (rpath $ORIGIN), with torch's own headers,
    libraries and C++ ABI."""
    src = os.path.join(CSRC, TORCH_SOURCE)
    lib = build(force=force)
    if not force and os.path.exists(TORCH_LIB) and os.path.getmtime(TORCH_LIB) >= max(
            os.path.getmtime(src), os.path.getmtime(lib), os.path.getmtime(os.path.join(ROOT, "include", "m3dgpu.h"))):
        return TORCH_LIB
    import torch
    from torch.utils import cpp_extension as ce
    cuda_home = ce.CUDA_HOME or "/usr/local/cuda"
    cmd = [os.environ.get("CXX", "g++"), "-shared", "-fPIC", "-O2", "-std=c++17",
           f"-D_GLIBCXX_USE_CXX11_ABI={int(torch._C._GLIBCXX_USE_CXX11_ABI)}", src, "-o", TORCH_LIB + ".tmp"]
    cmd += [f"-I{p}" for p in ce.include_paths()] + [f"-I{os.path.join(cuda_home, 'include')}",
                                                     f"-I{os.path.join(ROOT, 'include')}"]
    cmd += [f"-L{p}" for p in ce.library_paths()] + ["-lc10", "-lc10_cuda", "-ltorch_cpu", "-ltorch_cuda", "-ltorch",
                                                     f"-L{HERE}", "-lm3dgpu", "-Wl,-rpath,$ORIGIN"]
    subprocess.run(cmd, check=True)
    os.replace(TORCH_LIB + ".tmp", TORCH_LIB)
    return TORCH_LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
    if "--torch" in sys.argv:
        print(build_torch(force="--force" in sys.argv))
