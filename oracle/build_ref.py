"""Build recipe: compile the reference's own CUDA kernel source for the HOST.

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.

The reference keeps all of its kernels as CUDA C source strings inside
``processing/kernels.py`` (cupy.RawKernel), so its hot-path kernels can be
built here from its own source without cupy or a GPU.  This script

1. parses ``<reference>/processing/kernels.py`` with ``ast`` (nothing is
   executed) and takes the source string and entry name of every
   ``cp.RawKernel(src, name)`` call;
2. writes a translation unit into ``oracle/_ref/`` that puts those strings
   after a small host shim (``float2``, ``__expf`` -> ``expf``,
   ``__cosf``/``__sinf``, ``atomicAdd`` -> an OpenMP atomic add, the
   ``threadIdx``/``blockIdx``/``blockDim`` built-ins as thread-local
   variables) and adds one launch driver per kernel that walks the grid;
3. compiles it with ``g++ -fopenmp`` into ``oracle/_ref/libref_kernels.so``
   and deletes the generated source;
4. writes a second translation unit with the same kernel strings, verbatim,
   behind ``#include <math.h>`` / ``#undef M_PI`` (the kernels declare their
   own ``const float M_PI``) and one ``extern "C"`` launcher per kernel
   (grid, block and stream as arguments), compiles it with nvcc for sm_100a
   into ``oracle/_ref/libref_gpu.so`` and deletes the source.  That library
   is the reference's GPU kernels as cupy would run them, for the GPU
   reference harness (``oracle/refgpu.py``).

Only ``oracle/_ref/`` is written; it is git-ignored (the reference source
never enters the repository) but travels with the tree to the GPU box.
Each library is rebuilt only when ``kernels.py`` is newer.  Exit status 0
with a message when the reference tree is absent.
"""
from __future__ import annotations

import ast
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libref_kernels.so")
LIB_GPU = os.path.join(OUT_DIR, "libref_gpu.so")
DEFAULT_REF = "/root/reference"

SHIM = r"""
#include <math.h>
#include <stdint.h>
#undef M_PI
struct float2 { float x, y; };
static inline float2 make_float2(float a, float b) { float2 r; r.x = a; r.y = b; return r; }
struct mm_dim3 { unsigned x, y, z; };
static thread_local mm_dim3 threadIdx, blockIdx, blockDim;
#define __global__
#define __device__
#define __restrict__ __restrict
#define __expf expf
#define __cosf cosf
#define __sinf sinf
static inline float atomicAdd(float* p, float v) {
    float old;
    #pragma omp atomic capture
    { old = *p; *p += v; }
    return old;
}
"""

# One driver per kernel: grid (gx, gy, gz) of single-thread blocks; the
# kernels compute their indices from blockDim*blockIdx+threadIdx and return
# when out of range, so this visits every thread position exactly once.
DRIVER = r"""
extern "C" void ref_launch_%(name)s(long gx, long gy, long gz %(params)s) {
    #pragma omp parallel for collapse(2) schedule(dynamic, 16)
    for (long z = 0; z < gz; ++z)
    for (long y = 0; y < gy; ++y)
    for (long x = 0; x < gx; ++x) {
        blockDim.x = blockDim.y = blockDim.z = 1;
        threadIdx.x = threadIdx.y = threadIdx.z = 0;
        blockIdx.x = (unsigned)x; blockIdx.y = (unsigned)y; blockIdx.z = (unsigned)z;
        %(name)s(%(args)s);
    }
}
"""


GPU_PRELUDE = r"""
#include <math.h>
#include <cuda_runtime.h>
#undef M_PI
"""

GPU_LAUNCHER = r"""
extern "C" int refgpu_%(name)s(unsigned gx, unsigned gy, unsigned gz, unsigned bx, unsigned by, unsigned bz,
                               void* stream %(params)s) {
    %(name)s<<<dim3(gx, gy, gz), dim3(bx, by, bz), 0, (cudaStream_t)stream>>>(%(args)s);
    return (int)cudaGetLastError();
}
"""


def _fresh(lib: str, src: str) -> bool:
    return os.path.exists(lib) and os.path.getmtime(lib) >= os.path.getmtime(src)


def extract_kernels(kernels_py: str):
    """Return [(entry_name, source)] for every cp.RawKernel(src, name) call."""
    tree = ast.parse(open(kernels_py).read())
    found = []
    for node in ast.walk(tree):
        if isinstance(node, ast.Call) and getattr(node.func, "attr", None) == "RawKernel":
            if len(node.args) >= 2 and all(isinstance(a, ast.Constant) for a in node.args[:2]):
                found.append((node.args[1].value, node.args[0].value))
    return found


def _signature(src: str, name: str):
    """Parameter list text of `name(...)` in the kernel source."""
    i = src.index(name + "(")
    j = i + len(name) + 1
    depth = 1
    k = j
    while depth:
        if src[k] == "(":
            depth += 1
        elif src[k] == ")":
            depth -= 1
        k += 1
    params = " ".join(src[j:k - 1].split())
    parts = [p.strip() for p in params.split(",") if p.strip()]
    names = [p.replace("*", " ").split()[-1] for p in parts]
    return parts, names


def build_gpu(ref_root: str = DEFAULT_REF, verbose: bool = True, force: bool = False) -> str | None:
    """The reference's kernel strings compiled for sm_100a with launchers."""
    kp = os.path.join(ref_root, "processing", "kernels.py")
    if not os.path.exists(kp):
        return None
    if not force and _fresh(LIB_GPU, kp):
        return LIB_GPU
    kernels = extract_kernels(kp)
    os.makedirs(OUT_DIR, exist_ok=True)
    tu = [GPU_PRELUDE]
    for name, src in kernels:
        tu.append(f"// ---- kernel source: processing/kernels.py entry '{name}' ----\n")
        tu.append(src)
    for name, src in kernels:
        parts, names = _signature(src, name)
        params = "".join(", " + p for p in parts)
        tu.append(GPU_LAUNCHER % {"name": name, "params": params, "args": ", ".join(names)})
    cu = os.path.join(OUT_DIR, "ref_kernels_gpu.cu")
    with open(cu, "w") as f:
        f.write("\n".join(tu))
    nvcc = "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc"
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-Xcompiler", "-fPIC", "-shared", "-w",
           cu, "-o", LIB_GPU]
    try:
        subprocess.run(cmd, check=True)
    finally:
        os.remove(cu)
    if verbose:
        print(f"build_ref: {len(kernels)} kernels for sm_100a -> {LIB_GPU}")
    return LIB_GPU


def build(ref_root: str = DEFAULT_REF, verbose: bool = True, force: bool = False) -> str | None:
    kp = os.path.join(ref_root, "processing", "kernels.py")
    if not os.path.exists(kp):
        if verbose:
            print(f"build_ref: {kp} not found; oracle/_ref not rebuilt")
        return None
    build_gpu(ref_root, verbose, force)
    if not force and _fresh(LIB, kp):
        return LIB
    kernels = extract_kernels(kp)
    os.makedirs(OUT_DIR, exist_ok=True)
    tu = [SHIM]
    for name, src in kernels:
        tu.append(f"// ---- kernel source: processing/kernels.py entry '{name}' ----\n")
        tu.append(src)
    for name, src in kernels:
        parts, names = _signature(src, name)
        params = "".join(", " + p for p in parts)
        tu.append(DRIVER % {"name": name, "params": params, "args": ", ".join(names)})
    cpp = os.path.join(OUT_DIR, "ref_kernels_host.cpp")
    with open(cpp, "w") as f:
        f.write("\n".join(tu))
    cmd = ["g++", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c++17", "-w", cpp, "-o", LIB]
    try:
        subprocess.run(cmd, check=True)
    finally:
        os.remove(cpp)
    if verbose:
        print(f"build_ref: {len(kernels)} kernels -> {LIB}: {[k for k, _ in kernels]}")
    return LIB


if __name__ == "__main__":
    build(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_REF)
