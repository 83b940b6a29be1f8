"""Propagation -- Fresnel propagator on one B200 (drop-in for processing/propagation.py).

    prop = Propagation(n, nz, ntheta, ndist, wavelength, voxelsize, distance)
    out  = prop.D(psi, j)     # (ntheta', nz, n) or (nz, n) complex64, ntheta' <= ntheta
    back = prop.DT(out, j)    # adjoint of D (new: the reference has no DT)
    I    = prop.intensity(proj, inv_norm, inv_beta_ratio, j)   # fused step3 stage

Inputs may be torch CUDA tensors, cupy arrays or host numpy arrays; results
come back as the same kind, freshly allocated (propagation.py:61-64).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from model_mosaic_b200 import _ffi
from model_mosaic_b200._interop import require_cuda, to_device, from_device, stream_ptr


class Propagation:
    """Fresnel forward propagator sized for (ntheta x nz x n) (propagation.py:15)."""

    def __init__(self, n, nz, ntheta, ndist, wavelength, voxelsize, distance):
        require_cuda()
        L = _ffi.lib()
        self.n, self.nz, self.ntheta, self.ndist = int(n), int(nz), int(ntheta), int(ndist)
        dist = np.ascontiguousarray(np.atleast_1d(np.asarray(distance, dtype=np.float64))[:self.ndist])
        if dist.size < self.ndist:
            raise ValueError(f"need {self.ndist} distances, got {dist.size}")
        self.wavelength, self.voxelsize, self.distance = float(wavelength), float(voxelsize), dist
        h = C.c_void_p()
        _ffi.check(L.mm_prop_create(self.n, self.nz, self.ntheta, self.ndist, self.wavelength, self.voxelsize,
                                    dist.ctypes.data_as(C.c_void_p), C.byref(h)), "mm_prop_create")
        self._h = h

    def free(self):
        if getattr(self, "_h", None):
            _ffi.lib().mm_prop_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def _handle(self):
        if not self._h:
            raise RuntimeError("Propagation used after free()")
        return self._h

    def _apply(self, fn, psi, j):
        x, kind = to_device(psi, torch.complex64)
        added = x.dim() == 2
        if added:
            x = x.unsqueeze(0)
        if x.dim() != 3 or x.shape[1] != self.nz or x.shape[2] != self.n:
            raise ValueError(f"psi shape {tuple(x.shape)} is not (ntheta, {self.nz}, {self.n})")
        out = torch.empty_like(x)
        _ffi.check(fn(self._handle(), C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), x.shape[0], int(j),
                      C.c_void_p(stream_ptr(x.device))))
        if added:
            out = out[0]
        return from_device(out, kind)

    def D(self, psi, j):
        """Forward Fresnel propagation with the j-th kernel (propagation.py:47-64)."""
        return self._apply(_ffi.lib().mm_prop_D, psi, j)

    def DT(self, g, j):
        """Adjoint of D: <D a, b> = <a, DT b> (complex inner product)."""
        return self._apply(_ffi.lib().mm_prop_DT, g, j)

    def intensity(self, proj, inv_norm, inv_beta_ratio, j=0):
        """|D(psi(proj))|^2 with psi = exp(-p s/beta_r)(cos p s, sin p s), the
        step3_propagation.py:220-225 stage chain in two passes over HBM."""
        x, kind = to_device(proj, torch.float32)
        added = x.dim() == 2
        if added:
            x = x.unsqueeze(0)
        if x.dim() != 3 or x.shape[1] != self.nz or x.shape[2] != self.n:
            raise ValueError(f"proj shape {tuple(x.shape)} is not (ntheta, {self.nz}, {self.n})")
        out = torch.empty_like(x)
        _ffi.check(_ffi.lib().mm_prop_intensity(self._handle(), C.c_void_p(x.data_ptr()), float(inv_norm),
                                                float(inv_beta_ratio), C.c_void_p(out.data_ptr()), x.shape[0],
                                                int(j), C.c_void_p(stream_ptr(x.device))))
        if added:
            out = out[0]
        return from_device(out, kind)

    # -- per-stage CUDA-event timing ---------------------------------------------
    def set_timing(self, on: bool = True):
        _ffi.check(_ffi.lib().mm_prop_set_timing(self._handle(), int(bool(on))))

    def timing(self):
        """({stage: (ms, calls)}, own kernel launches) since set_timing(True)."""
        return _ffi.read_timing(_ffi.lib().mm_prop_get_timing, self._handle(), _ffi.PROP_STAGES)

    # torch-native entry points (no copies, caller-provided outputs)
    def D_into(self, x: torch.Tensor, out: torch.Tensor, j=0):
        _ffi.check(_ffi.lib().mm_prop_D(self._handle(), C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()),
                                        x.shape[0], int(j), C.c_void_p(stream_ptr(x.device))))
        return out

    def DT_into(self, x: torch.Tensor, out: torch.Tensor, j=0):
        _ffi.check(_ffi.lib().mm_prop_DT(self._handle(), C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()),
                                         x.shape[0], int(j), C.c_void_p(stream_ptr(x.device))))
        return out

    def intensity_into(self, x: torch.Tensor, out: torch.Tensor, inv_norm, inv_beta_ratio, j=0):
        _ffi.check(_ffi.lib().mm_prop_intensity(self._handle(), C.c_void_p(x.data_ptr()), float(inv_norm),
                                                float(inv_beta_ratio), C.c_void_p(out.data_ptr()), x.shape[0],
                                                int(j), C.c_void_p(stream_ptr(x.device))))
        return out
