"""Paganin -- single-distance phase retrieval on one B200 (drop-in for processing/paganin.py).

Same constructor and method as the reference class (processing/paganin.py:28-91):

    pgn = Paganin(n, nz, ntheta, wavelength, voxelsize, distance, alpha)
    phase = pgn.retrieve(intensity)     # (ntheta', nz, n) or (nz, n) float32 -> same shape, new array

phase = -log(clip(irfft2(H * rfft2(I)), 1e-6)) per frame with
H = alpha / (lambda z (kx^2 + ky^2) / (4 pi) + alpha).  The filter table is
built here exactly as the reference builds it (float32 arithmetic on the
fftfreq x rfftfreq grid, :46-53); the transform runs in ``libmosaic.so`` (three
fused passes for sizes 2^k up to 4096 and 3 * 2^k in [96, 3072], cuFFT
otherwise).  Inputs may
be torch CUDA tensors, ``__cuda_array_interface__`` arrays or numpy arrays;
the result comes back as the same kind.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from model_mosaic_b200 import _ffi
from model_mosaic_b200._interop import from_device, require_cuda, stream_ptr, to_device


def paganin_table(n, nz, wavelength, voxelsize, distance, alpha) -> np.ndarray:
    """float32 (nz, n//2 + 1) filter on the (fftfreq(nz), rfftfreq(n)) grid (processing/paganin.py:46-53)."""
    fy = np.fft.fftfreq(nz, d=voxelsize).astype("float32")
    fx = np.fft.rfftfreq(n, d=voxelsize).astype("float32")
    w2 = fy[:, None] ** 2 + fx[None, :] ** 2
    return (alpha / (wavelength * distance * w2 / (4.0 * np.pi) + alpha)).astype("float32")


class Paganin:
    """Single-distance Paganin phase retrieval (processing/paganin.py:28)."""

    def __init__(self, n, nz, ntheta, wavelength, voxelsize, distance, alpha):
        require_cuda()
        self.n, self.nz, self._ntheta = int(n), int(nz), int(ntheta)
        self.filt = np.ascontiguousarray(paganin_table(self.n, self.nz, wavelength, voxelsize, distance, alpha))
        h = C.c_void_p()
        _ffi.check(_ffi.lib().mm_pgn_create(self.n, self.nz, self._ntheta, self.filt.ctypes.data_as(C.c_void_p),
                                            C.byref(h)), "mm_pgn_create")
        self._h = h

    def free(self):
        if getattr(self, "_h", None):
            _ffi.lib().mm_pgn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def retrieve(self, intensity):
        """(ntheta', nz, n) or (nz, n) real float32 intensity -> phase of the same shape."""
        x, kind = to_device(intensity, torch.float32)
        added = x.dim() == 2
        if added:
            x = x.unsqueeze(0)
        b = x.shape[0]
        assert b <= self._ntheta, f"batch {b} > cached ntheta {self._ntheta}"
        if x.shape[1:] != (self.nz, self.n):
            raise ValueError(f"intensity shape {tuple(x.shape)} is not (batch, {self.nz}, {self.n})")
        out = torch.empty_like(x)
        self.retrieve_into(x, out)
        return from_device(out[0] if added else out, kind)

    def retrieve_into(self, x: torch.Tensor, out: torch.Tensor):
        """Device-to-device form (no copies): x, out (batch, nz, n) float32 CUDA tensors."""
        if self._h is None:
            raise RuntimeError("Paganin used after free()")
        _ffi.check(_ffi.lib().mm_pgn_retrieve(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()),
                                              x.shape[0], C.c_void_p(stream_ptr(x.device))), "mm_pgn_retrieve")
        return out
