"""Run the reference's own kernels (compiled for the host by
``oracle/build_ref.py``) with the reference's host glue restated in NumPy.

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.  This is the
strongest pin available without cupy: the gather/scatter/pad arithmetic is
the reference's own source (processing/kernels.py), only the FFT calls
(cuFFT in the reference, pocketfft here) and the elementwise glue of
processing/tomo.py / processing/propagation.py are restated.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .usfft import usfft_params, phi_table, c1dfftshift
from .fresnel import fresnel_kernel

_LIB = None
_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libref_kernels.so")


def available() -> bool:
    return os.path.exists(_PATH)


def lib():
    global _LIB
    if _LIB is None:
        if not available():
            raise FileNotFoundError(f"{_PATH} missing: run python oracle/build_ref.py")
        L = C.CDLL(_PATH)
        p, i, l, f = C.c_void_p, C.c_int, C.c_long, C.c_float
        L.ref_launch_gather.argtypes = [l, l, l, p, p, p, i, p, i, i, i, C.c_bool]
        L.ref_launch_gather_rfft_full.argtypes = [l, l, l, p, p, p, i, p, i, i, i]
        L.ref_launch_gather_compact.argtypes = [l, l, l, p, p, p, p, p, p, i, p, i, i, i, i]
        L.ref_launch_pad_fwd.argtypes = [l, l, l, p, p, i, i, i]
        _LIB = L
    return _LIB


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _fft_backend(workers):
    """numpy.fft (single thread) or scipy.fft with `workers` threads."""
    if workers:
        import functools
        import scipy.fft as sf
        class _F:
            rfft2 = functools.partial(sf.rfft2, workers=workers)
            ifft = functools.partial(sf.ifft, workers=workers)
            fft = functools.partial(sf.fft, workers=workers)
            ifft2 = functools.partial(sf.ifft2, workers=workers)
            fft2 = functools.partial(sf.fft2, workers=workers)
        return _F
    return np.fft


class RefTomoReal:
    """TomoReal (processing/tomo.py) with the reference gather kernels."""

    def __init__(self, n, nz, theta, workers=0):
        self.fft = _fft_backend(workers)
        self.n, self.nz = n, nz
        self.theta = np.ascontiguousarray(np.asarray(theta).astype(np.float32))
        self.ntheta = len(self.theta)
        self.mu, self.m = usfft_params(n)
        self.mua = np.array([self.mu], dtype=np.float32)
        self.phi = phi_table(n, self.ntheta, self.mu, np.float32)
        self.c1d = c1dfftshift(n)
        c2 = (1 - 2 * (np.arange(1, 2 * n + 1) % 2)).astype(np.int8)
        self.c2d = np.outer(c2, c2)

    def R(self, obj):
        """processing/tomo.py:121-151 around gather_rfft_full."""
        n, T = self.n, self.ntheta
        nz = obj.shape[0]
        padded = np.zeros((nz, 2 * n, 2 * n), np.float32)
        padded[:, n // 2:3 * n // 2, n // 2:3 * n // 2] = obj.astype(np.float32) * self.phi
        fde = np.ascontiguousarray(self.fft.rfft2(padded, axes=(-2, -1)).astype(np.complex64))
        sino = np.zeros((T, nz, n), np.complex64)
        lib().ref_launch_gather_rfft_full(n, T, nz, _ptr(sino), _ptr(fde), _ptr(self.theta),
                                          self.m, _ptr(self.mua), n, T, nz)
        sino *= self.c1d
        sino = self.fft.ifft(sino, axis=-1).astype(np.complex64) * self.c1d
        return np.ascontiguousarray(sino.real / 4).astype(np.float32)

    def RT(self, data):
        """processing/tomo.py:153-188 around the dir=1 scatter."""
        n, T = self.n, self.ntheta
        nz = data.shape[1]
        s = np.ascontiguousarray((data * self.c1d).astype(np.complex64))
        s = np.fft.fft(s, axis=-1).astype(np.complex64) * self.c1d
        s = np.ascontiguousarray(s)
        fde = np.zeros((nz, 2 * n, 2 * n), np.complex64)
        lib().ref_launch_gather(n, T, nz, _ptr(s), _ptr(fde), _ptr(self.theta),
                                self.m, _ptr(self.mua), n, T, nz, True)
        fde *= self.c2d
        fde = np.fft.ifft2(fde, axes=(-2, -1)).astype(np.complex64) * self.c2d
        res = fde[:, n // 2:3 * n // 2, n // 2:3 * n // 2] * self.phi
        if np.dtype(data.dtype) == np.float32:
            res = res.real
        return np.ascontiguousarray(res)


class RefTomoLargeReal(RefTomoReal):
    """TomoLargeReal.R math with the reference's compact gather kernel run
    over one bin that holds every sample (tomo_large.py:459-579): the x0/y0
    clamp and the scale placement of the host-chunked class."""

    def R(self, obj, chunks=None):
        n, T = self.n, self.ntheta
        nz = obj.shape[0]
        t = np.linspace(-0.5, 0.5, n, endpoint=False).astype(np.float32)
        phi1d = np.exp(np.float32(self.mu * n * n) * (t * t)).astype(np.float32)
        phi_scale = np.float32(1 - n % 4)
        padded = np.zeros((nz, 2 * n, 2 * n), np.float32)
        padded[:, n // 2:3 * n // 2, n // 2:3 * n // 2] = (
            phi_scale * phi1d[None, :, None] * phi1d[None, None, :] * obj.astype(np.float32))
        fde = np.fft.rfft2(padded, axes=(-2, -1)).astype(np.complex64)
        cos_t = np.cos(self.theta).astype(np.float32)
        sin_t = np.sin(self.theta).astype(np.float32)
        k, j = np.meshgrid(np.arange(T, dtype=np.int32), np.arange(n, dtype=np.int32), indexing="ij")
        ti, xi = np.ascontiguousarray(k.ravel()), np.ascontiguousarray(j.ravel())
        nel = T * n
        sino = np.zeros((T, nz, n), np.complex64)
        out = np.zeros(nel, np.complex64)
        for z in range(nz):
            f = np.ascontiguousarray(fde[z])
            lib().ref_launch_gather_compact(nel, 1, 1, _ptr(out), _ptr(f), _ptr(xi), _ptr(ti),
                                            _ptr(cos_t), _ptr(sin_t), self.m, _ptr(self.mua),
                                            nel, 0, n + 1, n)
            sino[:, z, :] = out.reshape(T, n)
        sino *= self.c1d
        sino = np.fft.ifft(sino, axis=-1).astype(np.complex64) * self.c1d
        scale = np.float32(1.0 / (4 * n * np.sqrt(n * T)))
        return np.ascontiguousarray((sino * scale).real).astype(np.float32)


class RefPropagation:
    """Propagation.D (processing/propagation.py:47-64) with pad_fwd."""

    def __init__(self, n, nz, ntheta, ndist, wavelength, voxelsize, distance, workers=0):
        self.fft = _fft_backend(workers)
        self.n, self.nz = n, nz
        self.fker = fresnel_kernel(n, nz, wavelength, voxelsize, list(distance)[:ndist], np.float32)

    def D(self, psi, j):
        added = psi.ndim == 2
        if added:
            psi = psi[None]
        n, nz = self.n, self.nz
        T = psi.shape[0]
        src = np.ascontiguousarray(psi.astype(np.complex64))
        pad = np.zeros((T, 2 * nz, 2 * n), np.complex64)
        lib().ref_launch_pad_fwd(2 * n, 2 * nz, T, _ptr(pad), _ptr(src), n, nz, T)
        f = self.fft.fft2(pad, axes=(-2, -1)).astype(np.complex64) * self.fker[j]
        f = self.fft.ifft2(f, axes=(-2, -1), norm="forward").astype(np.complex64)
        res = np.ascontiguousarray(f[:, nz // 2:nz // 2 + nz, n // 2:n // 2 + n])
        return res[0] if added else res
