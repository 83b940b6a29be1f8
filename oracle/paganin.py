"""FP64 NumPy restatement of the reference's Paganin retrieval -- test infrastructure.

Only tests/ and bench.py's CPU legs use this module, as the checker; the
product is model_mosaic_b200/csrc/paganin.cu.

processing/paganin.py:38-91: per (nz, n) intensity frame I,
    H(ky, kx) = alpha / (lambda z (kx^2 + ky^2) / (4 pi) + alpha)   (float32 table
        on the fftfreq(nz) x rfftfreq(n) grid, :46-53)
    phase = -log(clip(irfft2(H * rfft2(I)), 1e-6))                   (:80-90)
"""
from __future__ import annotations

import numpy as np


def paganin_filter(n, nz, wavelength, voxelsize, distance, alpha) -> np.ndarray:
    """The reference's float32 (nz, n//2 + 1) filter table (processing/paganin.py:46-53)."""
    fy = np.fft.fftfreq(nz, d=voxelsize).astype("float32")
    fx = np.fft.rfftfreq(n, d=voxelsize).astype("float32")
    w2 = fy[:, None] ** 2 + fx[None, :] ** 2
    return (alpha / (wavelength * distance * w2 / (4.0 * np.pi) + alpha)).astype("float32")


def retrieve(intensity, filt) -> np.ndarray:
    """-log(clip(irfft2(filt * rfft2(I)), 1e-6)) per frame, FP64 (processing/paganin.py:64-91)."""
    x = np.asarray(intensity, dtype=np.float64)
    nz, n = x.shape[-2:]
    y = np.fft.irfft2(np.fft.rfft2(x, axes=(-2, -1)) * np.asarray(filt, np.float64), s=(nz, n), axes=(-2, -1))
    return -np.log(np.clip(y, 1e-6, None))
