"""Oracle calls packaged as top-level functions for a process pool.

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.  The full-size parity
tests run several FP64 oracle slices at once in a ``spawn`` pool (NumPy's FFT
is single-threaded); each function here builds its oracle object inside the
worker, so only arrays and scalars cross the process boundary.
"""
from __future__ import annotations

import multiprocessing as mp

import numpy as np


def pool(workers: int = 4):
    """A spawn-context pool: safe to start after the parent has used a GPU."""
    return mp.get_context("spawn").Pool(workers)


def tomo_R(n, theta, obj, dtype=np.float64, eps=1e-3):
    """TomoReal.R (processing/tomo.py:121-151) of `obj` (nz, n, n)."""
    from .usfft import TomoRealOracle
    return TomoRealOracle(n, obj.shape[0], theta, dtype=dtype, eps=eps).R(obj)


def tomo_RT(n, theta, data, dtype=np.float64, eps=1e-3):
    """TomoReal.RT (processing/tomo.py:153-188) of `data` (ntheta, nz, n)."""
    from .usfft import TomoRealOracle
    return TomoRealOracle(n, data.shape[1], theta, dtype=dtype, eps=eps).RT(data)


def ref_tomo_R(n, theta, obj):
    """TomoReal.R with the reference's own gather kernel (host build)."""
    from .refkernels import RefTomoReal
    return RefTomoReal(n, obj.shape[0], theta).R(obj)


def model_grad(n, theta, wavelength, voxelsize, distance, s, delta, d, dtype=np.float64):
    """Loss and gradient of the L2 misfit of |D psi(R delta)|^2 (FP64, or the
    float32 floor with dtype=np.float32)."""
    from .model import ModelOracle
    o = ModelOracle(n, delta.shape[0], theta, wavelength, voxelsize, distance, s=s, dtype=dtype)
    return o.loss(delta, d), o.grad(delta, d)


def model_forward(n, theta, wavelength, voxelsize, distance, s, delta):
    from .model import ModelOracle
    return ModelOracle(n, delta.shape[0], theta, wavelength, voxelsize, distance, s=s).forward(delta)
