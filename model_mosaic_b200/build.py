"""Build the in-tree CUDA library ``model_mosaic_b200/libmosaic.so`` for sm_100a.

    python -m model_mosaic_b200.build          # or: python model_mosaic_b200/build.py

The library is a plain C-ABI shared object (include/mosaic.h) compiled with
nvcc for ``arch=compute_100a,code=sm_100a`` and linked against cuFFT.  It is
built in place so that it travels with the source tree.  Each ``.cu`` file is
compiled to its own object under ``model_mosaic_b200/_build/`` in parallel
(only the files whose sources or headers changed), then the objects are
linked.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmosaic.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(ROOT, "include", "mosaic.h")]


def _obj(src: str) -> str:
    return os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")


def _stale(src: str) -> bool:
    o = _obj(src)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    return any(os.path.getmtime(d) > t for d in [src, *headers()])


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in sources() + headers())


def build(force: bool = False, verbose: bool = True, extra=None) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    cc = nvcc()
    todo = [s for s in sources() if force or _stale(s)]

    def compile_one(src):
        cmd = [cc, *ARCH, *FLAGS, "-c", "-o", _obj(src) + ".tmp", src, *(extra or [])]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr.strip():
            print(r.stderr, flush=True)
        os.replace(_obj(src) + ".tmp", _obj(src))

    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 4))) as ex:
        list(ex.map(compile_one, todo))
    cuda_lib = os.path.join(os.path.dirname(os.path.dirname(cc)), "lib64")
    cmd = [cc, *ARCH, "-shared", "-o", LIB + ".tmp", *[_obj(s) for s in sources()],
           "-lcufft", f"-L{cuda_lib}", f"-Xlinker=-rpath={cuda_lib}"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=ROOT)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, extra=[a for a in sys.argv[1:] if a != "--force"])
