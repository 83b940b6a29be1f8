"""TomoReal -- USFFT Radon transform on one B200 (drop-in for processing/tomo.py).

Same constructor and methods as the reference class (processing/tomo.py:17-188):

    tomo = TomoReal(n, nz, theta)
    sino = tomo.R(obj)      # (nz', n, n) float32 -> (ntheta, nz', n) float32, nz' <= nz
    rec  = tomo.RT(sino)    # (ntheta, nz', n) float32|complex64 -> (nz', n, n) same dtype
    tomo.free()

Inputs may be torch CUDA tensors, cupy (``__cuda_array_interface__``) arrays
or host numpy arrays; results come back as the same kind, freshly allocated
(the reference returns a new contiguous device array, tomo.py:151,188).
All arithmetic runs in the CUDA library (``libmosaic.so``) through the C-ABI.

Keyword-only extras (not in the reference): ``eps`` and ``m`` override the
Gaussian accuracy / half-width (defaults 1e-3 and 4, processing/tomo.py:39-42);
``clamp_xy`` selects TomoLargeReal's clamped sample coordinates
(processing/kernels.py:478-481); ``compensated`` makes the adjoint's sums
Kahan-compensated; ``max_table_angles`` caps the angles per block of the
adjoint's scatter table (0: sized by free device memory).  bfloat16 torch tensors are accepted as storage (the
arithmetic stays float32): ``R`` of a bfloat16 volume returns a bfloat16
sinogram unless ``out_dtype`` says otherwise, ``RT`` of a bfloat16 sinogram
returns a bfloat16 volume.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from model_mosaic_b200 import _ffi
from model_mosaic_b200._interop import (require_cuda, to_device, from_device, stream_ptr, is_complex)


class _TomoOpts(C.Structure):
    _fields_ = [("eps", C.c_double), ("m", C.c_int), ("clamp_xy", C.c_int), ("compensated", C.c_int),
                ("max_table_angles", C.c_int), ("reserved", C.c_int * 3)]


def _storage(dt: torch.dtype) -> int:
    return _ffi.MM_BF16 if dt == torch.bfloat16 else _ffi.MM_F32


class TomoReal:
    """Radon transform via USFFT for REAL float32 objects (processing/tomo.py:17)."""

    def __init__(self, n, nz, theta, *, eps: float = 1e-3, m: int | None = None, clamp_xy: bool = False,
                 compensated: bool = False, max_table_angles: int = 0):
        require_cuda()
        L = _ffi.lib()
        self.n = int(n)
        self._nz = int(nz)
        th = np.ascontiguousarray(np.asarray(theta).astype("float32"))   # tomo.py:57
        self.ntheta = len(th)
        self.theta = th
        opts = _TomoOpts(eps=float(eps), m=int(m or 0), clamp_xy=int(bool(clamp_xy)),
                         compensated=int(bool(compensated)), max_table_angles=int(max_table_angles))
        h = C.c_void_p()
        _ffi.check(L.mm_tomo_create(self.n, self._nz, self.ntheta, th.ctypes.data_as(C.c_void_p),
                                    C.byref(opts), C.byref(h)), "mm_tomo_create")
        self._h = h
        self.device = torch.cuda.current_device()

    # -- lifetime ------------------------------------------------------------
    def free(self):
        """Release the device workspace (processing/tomo.py:109-119)."""
        if getattr(self, "_h", None):
            _ffi.lib().mm_tomo_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def _handle(self):
        if not self._h:
            raise RuntimeError("TomoReal used after free()")
        return self._h

    def workspace_bytes(self) -> int:
        return int(_ffi.lib().mm_tomo_workspace_bytes(self._handle()))

    def prepare_rt(self):
        """Build the adjoint's scatter table now (otherwise on the first RT)."""
        _ffi.check(_ffi.lib().mm_tomo_prepare_rt(self._handle(), C.c_void_p(stream_ptr())))

    # -- operators -------------------------------------------------------------
    def R(self, obj, out_dtype=None):
        """(nz, n, n) REAL float32 obj -> (ntheta, nz, n) float32 sinogram.
        A bfloat16 torch tensor is read as bfloat16; the sinogram is stored
        as ``out_dtype`` (torch.float32 or torch.bfloat16, default: the
        input's)."""
        bf = isinstance(obj, torch.Tensor) and obj.dtype == torch.bfloat16
        x, kind = to_device(obj, torch.bfloat16 if bf else torch.float32)
        if x.dim() != 3 or x.shape[1] != self.n or x.shape[2] != self.n:
            raise ValueError(f"R: obj shape {tuple(x.shape)} is not (nz, {self.n}, {self.n})")
        odt = out_dtype or x.dtype
        if odt not in (torch.float32, torch.bfloat16):
            raise ValueError(f"R: out_dtype {odt} is not float32 or bfloat16")
        nz = x.shape[0]
        out = torch.empty((self.ntheta, nz, self.n), dtype=odt, device=x.device)
        _ffi.check(_ffi.lib().mm_tomo_R_ex(self._handle(), C.c_void_p(x.data_ptr()), _storage(x.dtype),
                                           C.c_void_p(out.data_ptr()), _storage(odt), nz,
                                           C.c_void_p(stream_ptr(x.device))), "mm_tomo_R")
        return from_device(out, kind)

    def RT(self, data):
        """Adjoint: (ntheta, nz, n) sinogram -> (nz, n, n) object; float32 in
        gives float32 out, complex64 in gives complex64 out (tomo.py:153-188)."""
        cplx = is_complex(data)
        bf = isinstance(data, torch.Tensor) and data.dtype == torch.bfloat16
        dt = torch.complex64 if cplx else (torch.bfloat16 if bf else torch.float32)
        y, kind = to_device(data, dt)
        if y.dim() != 3 or y.shape[0] != self.ntheta or y.shape[2] != self.n:
            raise ValueError(f"RT: sinogram shape {tuple(y.shape)} is not ({self.ntheta}, nz, {self.n})")
        nz = y.shape[1]
        out = torch.empty((nz, self.n, self.n), dtype=dt, device=y.device)
        _ffi.check(_ffi.lib().mm_tomo_RT(self._handle(), C.c_void_p(y.data_ptr()),
                                         _ffi.MM_C64 if cplx else _storage(dt), C.c_void_p(out.data_ptr()), nz,
                                         C.c_void_p(stream_ptr(y.device))), "mm_tomo_RT")
        return from_device(out, kind)

    # -- per-stage CUDA-event timing ---------------------------------------------
    def set_timing(self, on: bool = True):
        _ffi.check(_ffi.lib().mm_tomo_set_timing(self._handle(), int(bool(on))))

    def timing(self):
        """({stage: (ms, calls)}, own kernel launches) since set_timing(True)."""
        return _ffi.read_timing(_ffi.lib().mm_tomo_get_timing, self._handle(), _ffi.TOMO_STAGES)

    # torch-native entry points used by the differentiable model (no copies)
    def R_into(self, x: torch.Tensor, out: torch.Tensor):
        _ffi.check(_ffi.lib().mm_tomo_R(self._handle(), C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()),
                                        x.shape[0], C.c_void_p(stream_ptr(x.device))), "mm_tomo_R")
        return out

    def RT_into(self, y: torch.Tensor, out: torch.Tensor):
        """float32 or complex64 sinogram y -> out of the same dtype."""
        dt = _ffi.MM_C64 if y.is_complex() else _ffi.MM_F32
        _ffi.check(_ffi.lib().mm_tomo_RT(self._handle(), C.c_void_p(y.data_ptr()), dt,
                                         C.c_void_p(out.data_ptr()), y.shape[1],
                                         C.c_void_p(stream_ptr(y.device))), "mm_tomo_RT")
        return out
