"""Build the in-tree CUDA library ``model_mosaic_b200/libmosaic.so`` for sm_100a.

    python -m model_mosaic_b200.build          # or: python model_mosaic_b200/build.py

The library is a plain C-ABI shared object (include/mosaic.h) compiled with
nvcc for ``arch=compute_100a,code=sm_100a`` and linked against cuFFT.  It is
built in place so that it travels with the source tree.
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
LIB = os.path.join(HERE, "libmosaic.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(ROOT, "include", "mosaic.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = True, extra=None) -> str:
    if not force and not needs_build():
        return LIB
    cuda_lib = os.path.join(os.path.dirname(os.path.dirname(nvcc())), "lib64")
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
           "-Xcompiler", "-fPIC", "-shared", "-o", LIB + ".tmp", *sources(),
           "-lcufft", f"-L{cuda_lib}", f"-Xlinker=-rpath={cuda_lib}", *(extra or [])]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=ROOT)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, extra=[a for a in sys.argv[1:] if a != "--force"])
