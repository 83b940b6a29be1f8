"""FBPFilter -- the step8_fbp filter on one B200 (drop-in for processing/fbp_filter.py).

Same constructor and methods as the reference class (processing/fbp_filter.py:38-247):

    f = FBPFilter(n, batch_chunk=256)
    w = f.calc_filter("shepp")          # (2n + 1,) float32 weights on the GPU, cached per name
    f.filter(sino, w)                   # (..., n) float32 device array, filtered in place, returned
    f.filter_host(sino_h, w)            # host array, chunked host <-> device round trips

Each row of n samples is edge-replicated to 4n, multiplied in frequency by the
weights and cropped back to n (processing/fbp_filter.py:182-191).  The work
runs in ``libmosaic.so``: for 4n a power of two up to 8192 or 3 * 2^k up to
12288 one fused kernel per two rows, in place and without scratch; other n
through cuFFT, batch_chunk rows at a time.  The weights are host-side FP64 arithmetic, as in the reference
(NumPy here), copied to the device once per filter name.  Inputs may be torch
CUDA tensors or ``__cuda_array_interface__`` arrays (cupy); `filter` writes
into the caller's array as the reference does.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from model_mosaic_b200 import _ffi
from model_mosaic_b200._interop import require_cuda, stream_ptr

FILTERS = ("none", "ramp", "shepp", "cosine", "cosine2", "hamming", "hann", "parzen")


def _quadrature(q: int, t: np.ndarray) -> np.ndarray:
    """Order-q quadrature weights on the grid t (processing/fbp_filter.py:90-126):
    polynomial integration weights from the inverse Vandermonde matrix of q
    nodes in (0, 1], summed over the overlapping short intervals, the last 40
    replaced by a linear taper.  The 12x12 Vandermonde matrix has a condition
    number near 1e9, so the weights depend on the inverse's algorithm at the
    1e-5 level; NumPy's (LAPACK) inverse is used, as the reference's host code
    does when run on NumPy."""
    N = len(t)
    s = np.linspace(1e-40, 1, q)
    iv = np.linalg.inv(np.exp(np.outer(np.arange(q), np.log(s))))
    a = np.arange(1, q + 2)
    u = np.diff(np.exp(np.outer(a, np.log(s))) * np.tile(1.0 / a[..., np.newaxis], [1, q]))
    w1 = iv @ u[1:q + 1, :]
    w2 = iv @ u[0:q, :]
    p = 1 / np.concatenate((np.arange(1, q), (q - 1) * np.ones(N - 2 * (q - 1) - 1), np.arange(q - 1, 0, -1)))
    w = np.zeros(N)
    for j in range(N - q + 1):
        dt = t[j + q - 1] - t[j]
        W = (dt ** 2) * w1 + dt * t[j] * w2
        for k in range(q - 1):
            w[j:j + q] = w[j:j + q] + p[j + k] * W[:, k]
    if N > 40:
        w[-40:] = (w[-40]) / (N - 40) * np.arange(N - 40, N)
    return w


def filter_weights(n: int, name: str) -> np.ndarray:
    """Host float32 (2n + 1,) weights of filter `name` (processing/fbp_filter.py:49-88)."""
    d = 0.5
    ne = 4 * n
    t = np.arange(0, ne // 2 + 1) / ne
    if name == "none":
        wfa = ne * 0.5 + t * 0
        wfa[0] *= 2
    else:
        if name not in FILTERS:
            raise ValueError(f"unknown FBP filter '{name}'; expected one of {', '.join(FILTERS)}")
        if len(t) < 23:
            raise ValueError(f"n={n} too small for the 12-point quadrature of filter '{name}'")
        base = ne * 0.5 * _quadrature(12, t)
        shape = {
            "ramp": 1.0,
            "shepp": np.sinc(t / (2 * d)) * (t / d <= 2),
            "cosine": np.cos(np.pi * t / (2 * d)) * (t / d <= 1),
            "cosine2": (np.cos(np.pi * t / (2 * d))) ** 2 * (t / d <= 1),
            "hamming": (.54 + .46 * np.cos(np.pi * t / d)) * (t / d <= 1),
            "hann": (1 + np.cos(np.pi * t / d)) / 2.0 * (t / d <= 1),
            "parzen": (1 - t / d) ** 3 * (t / d <= 1),
        }[name]
        wfa = base * shape
    wfa = 2 * wfa * (wfa >= 0)
    wfa[0] *= 2
    return (3 * n * wfa).astype(np.float32)


def _device_tensor(x):
    """A CUDA torch tensor sharing memory with `x` (torch or __cuda_array_interface__)."""
    if isinstance(x, torch.Tensor):
        if not x.is_cuda:
            raise ValueError("filter: sino must be on the GPU (use filter_host for host arrays)")
        return x
    if hasattr(x, "__cuda_array_interface__"):
        return torch.as_tensor(x, device="cuda")
    raise ValueError("filter: sino must be a CUDA array (use filter_host for host arrays)")


class FBPFilter:
    """FBP 1-D filter with edge-replicated 4x padding (processing/fbp_filter.py:38)."""

    def __init__(self, n: int, batch_chunk: int = 256):
        require_cuda()
        self.n = int(n)
        self.ne = 4 * self.n
        self.pad = (self.ne - self.n) // 2
        self.batch_chunk = int(batch_chunk)
        self._cache: dict[str, torch.Tensor] = {}
        h = C.c_void_p()
        _ffi.check(_ffi.lib().mm_fbp_create(self.n, self.batch_chunk, C.byref(h)), "mm_fbp_create")
        self._h = h

    def free(self):
        if getattr(self, "_h", None):
            _ffi.lib().mm_fbp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def calc_filter(self, name: str) -> torch.Tensor:
        """(ne//2 + 1,) float32 weights of the named filter on the GPU (cached)."""
        if name not in self._cache:
            self._cache[name] = torch.from_numpy(filter_weights(self.n, name)).cuda()
        return self._cache[name]

    def filter(self, sino, w, batch_chunk: int | None = None):
        """Filter `sino` (..., n) float32 on the GPU in place along its last
        axis and return it (processing/fbp_filter.py:128-192)."""
        t = _device_tensor(sino)
        if t.shape[-1] != self.n:
            raise ValueError(f"sino last-axis {t.shape[-1]} != filter n={self.n}")
        if not t.is_contiguous():
            raise ValueError("sino must be C-contiguous (reshape view for chunk loop)")
        if t.dtype != torch.float32:
            raise ValueError(f"sino must be float32, got {t.dtype}")
        wt = _device_tensor(w)
        if wt.dtype != torch.float32 or wt.numel() != self.ne // 2 + 1:
            raise ValueError(f"w must be float32 of length {self.ne // 2 + 1}")
        rows = t.numel() // self.n
        _ffi.check(_ffi.lib().mm_fbp_filter(self._h, C.c_void_p(t.data_ptr()), rows,
                                            C.c_void_p(wt.contiguous().data_ptr()),
                                            C.c_void_p(stream_ptr(t.device))), "mm_fbp_filter")
        return sino

    def filter_host(self, sino_h, w, batch_chunk: int | None = None):
        """Filter a host sinogram in place, batch_chunk rows per host <->
        device round trip (processing/fbp_filter.py:196-247)."""
        if sino_h.shape[-1] != self.n:
            raise ValueError(f"sino_h last-axis {sino_h.shape[-1]} != filter n={self.n}")
        if not sino_h.flags.c_contiguous:
            raise ValueError("sino_h must be C-contiguous (reshape view for chunk loop)")
        flat = sino_h.reshape(-1, self.n)
        chunk = min(int(batch_chunk or self.batch_chunk), flat.shape[0])
        for i0 in range(0, flat.shape[0], chunk):
            i1 = min(i0 + chunk, flat.shape[0])
            d = torch.from_numpy(np.ascontiguousarray(flat[i0:i1], dtype=np.float32)).cuda()
            self.filter(d, w)
            flat[i0:i1] = d.cpu().numpy()
        return sino_h
