"""Generate the committed golden fixtures from the reference's own kernels.

The reference publishes no golden vectors; its tests pin only
self-consistency (tests/test_large_variants.py).  These fixtures are made by
running the reference's kernel source (processing/kernels.py, compiled for
the host by ``oracle/build_ref.py``) with the host glue of
processing/tomo.py and processing/propagation.py restated in NumPy
(``oracle/refkernels.py``), on the shapes and seeds of
tests/test_large_variants.py.

Run from the repository root (needs the reference tree for build_ref):

    python oracle/build_ref.py && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.refkernels import RefTomoReal, RefTomoLargeReal, RefPropagation  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def tomo_fixtures():
    # test_tomo_R_vs_large: n=64, nz=16, ntheta=24, theta in [0, 2pi), seed 0
    n, nz, T = 64, 16, 24
    theta = np.linspace(0, 2 * np.pi, T, endpoint=False).astype("float32")
    np.random.seed(0)
    obj = np.random.randn(nz, n, n).astype(np.float32)
    sino = RefTomoReal(n, nz, theta).R(obj)
    sino_l = RefTomoLargeReal(n, nz, theta).R(obj)
    np.savez_compressed(os.path.join(OUT, "tomo_R_n64_nz16_t24.npz"),
                        theta=theta, obj=obj, sino=sino, sino_large=sino_l)

    # test_tomo_RT_vs_large: n=64, nz=8, ntheta=24, complex64 then float32 sinos
    n, nz, T = 64, 8, 24
    theta = np.linspace(0, 2 * np.pi, T, endpoint=False).astype("float32")
    np.random.seed(0)
    sc = (np.random.randn(T, nz, n) + 1j * np.random.randn(T, nz, n)).astype(np.complex64)
    sr = np.random.randn(T, nz, n).astype(np.float32)
    tomo = RefTomoReal(n, nz, theta)
    np.savez_compressed(os.path.join(OUT, "tomo_RT_n64_nz8_t24.npz"),
                        theta=theta, sino_c=sc, obj_c=tomo.RT(sc), sino_r=sr, obj_r=tomo.RT(sr))

    # test_tomo_R_RT_adjoint: n=64, nz=8, ntheta=24
    np.random.seed(0)
    x = np.random.randn(nz, n, n).astype(np.float32)
    y = np.random.randn(T, nz, n).astype(np.float32)
    np.savez_compressed(os.path.join(OUT, "tomo_adjoint_n64_nz8_t24.npz"),
                        theta=theta, x=x, y=y, Rx=tomo.R(x), RTy=tomo.RT(y))

    # half-angle range, non-square slice count, n=48 (n % 4 == 0, not 2^k)
    n, nz, T = 48, 3, 30
    theta = np.linspace(0, np.pi, T, endpoint=False).astype("float32")
    rng = np.random.default_rng(7)
    obj = rng.standard_normal((nz, n, n)).astype(np.float32)
    tomo = RefTomoReal(n, nz, theta)
    ys = rng.standard_normal((T, nz, n)).astype(np.float32)
    np.savez_compressed(os.path.join(OUT, "tomo_n48_nz3_t30.npz"),
                        theta=theta, obj=obj, sino=tomo.R(obj), y=ys, RTy=tomo.RT(ys))


def prop_fixtures():
    # test_propagation_vs_large: n=64, nz=32, ntheta=3, three distances, seed 0
    n, nz, T = 64, 32, 3
    wl, vs, dist = 4.13e-11, 1.4e-6, [0.0, 0.02, 0.1]
    np.random.seed(0)
    psi = (np.random.randn(T, nz, n) + 1j * np.random.randn(T, nz, n)).astype(np.complex64)
    prop = RefPropagation(n, nz, T, len(dist), wl, vs, dist)
    D = np.stack([prop.D(psi, j) for j in range(len(dist))])
    np.savez_compressed(os.path.join(OUT, "prop_D_n64_nz32_t3.npz"),
                        psi=psi, D=D, wavelength=wl, voxelsize=vs, distance=np.array(dist))


if __name__ == "__main__":
    tomo_fixtures()
    prop_fixtures()
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))
