"""TomoLargeReal -- drop-in for processing/tomo_large.py on one B200.

The reference stages its (nz, 2n, n+1) spectrum through pinned host memory
because it did not fit on the GPUs it targeted (processing/tomo_large.py:1-19).
A B200 holds every configuration of the forward model in HBM, so this class
keeps the reference's host-array API -- numpy in, numpy out, results in
internal pinned buffers that the next call reuses (tomo_large.py:545-555,
611) -- and runs the same device-resident USFFT as ``TomoReal`` in between.

    tomo = TomoLargeReal(n, theta, chunk_xy)
    sino = tomo.R(obj_host, [chunk_n, chunk_theta, chunk_xy])
    rec  = tomo.RT(sino_host, [chunk_n, chunk_theta, chunk_xy])
    buf  = tomo.obj_buffer(nz)      # pinned (nz, n, n) float32
    tomo.free()

The chunk sizes are validated like the reference (chunk_n must divide n,
tomo_large.py:438-440) and otherwise only bound the slab size moved per call.
"""
from __future__ import annotations

import numpy as np
import torch

from model_mosaic_b200._interop import pinned_empty, require_cuda
from model_mosaic_b200.processing.tomo import TomoReal


class TomoLargeReal:
    def __init__(self, n, theta, chunk_xy, *, eps: float = 1e-3, m: int | None = None, max_nz: int = 64):
        require_cuda()
        self.n = int(n)
        self.theta = np.asarray(theta).astype("float32")
        self.ntheta = len(self.theta)
        self.chunk_xy = int(chunk_xy)
        self._eps, self._m = eps, m
        self._max_nz = int(max_nz)
        self._tomo = None
        self._tomo_nz = 0
        self._sino = None
        self._obj = None
        self._obj_rt = None

    def _engine(self, nz):
        if self._tomo is None or self._tomo_nz < nz:
            if self._tomo is not None:
                self._tomo.free()
            self._tomo_nz = max(nz, 1)
            self._tomo = TomoReal(self.n, self._tomo_nz, self.theta, eps=self._eps, m=self._m, clamp_xy=True)
        return self._tomo

    def _check_chunks(self, chunks):
        chunk_n, chunk_theta, chunk_xy = (int(c) for c in chunks)
        assert self.n % chunk_n == 0, f"CHUNK_N={chunk_n} must divide n={self.n} (rfft x-axis strips)"
        assert self.ntheta % chunk_theta == 0, f"CHUNK_THETA={chunk_theta} must divide ntheta={self.ntheta}"
        assert chunk_xy > 0, f"CHUNK_XY={chunk_xy} must be positive"

    def free(self):
        if self._tomo is not None:
            self._tomo.free()
        self._tomo = None
        self._sino = self._obj = self._obj_rt = None

    def obj_buffer(self, nz):
        """Pinned (nz, n, n) float32 buffer for the caller to fill
        (tomo_large.py:327-341); cached across calls."""
        shape = (nz, self.n, self.n)
        if self._obj is None or self._obj.shape != shape:
            self._obj = pinned_empty(shape, np.float32)
        return self._obj

    def R(self, obj, chunks):
        """(nz, n, n) float32 host obj -> (ntheta, nz, n) float32 host sino,
        returned in an internal buffer valid until the next R()."""
        self._check_chunks(chunks)
        obj = np.asarray(obj)
        nz = obj.shape[0]
        shape = (self.ntheta, nz, self.n)
        if self._sino is None or self._sino.shape != shape:
            self._sino = pinned_empty(shape, np.float32)
        tomo = self._engine(min(nz, self._max_nz) if nz > self._max_nz else nz)
        step = tomo._nz
        for z0 in range(0, nz, step):
            z1 = min(nz, z0 + step)
            x = torch.from_numpy(np.ascontiguousarray(obj[z0:z1], dtype=np.float32)).cuda()
            out = torch.empty((self.ntheta, z1 - z0, self.n), dtype=torch.float32, device="cuda")
            tomo.R_into(x, out)
            self._sino[:, z0:z1, :] = out.cpu().numpy()
        return self._sino

    def RT(self, sino, chunks):
        """(ntheta, nz, n) host sino (float32 or complex64) -> (nz, n, n) host
        obj of the matching dtype, in an internal buffer (tomo_large.py:582-630)."""
        self._check_chunks(chunks)
        sino = np.asarray(sino)
        nz = sino.shape[1]
        dt = np.complex64 if np.iscomplexobj(sino) else np.float32
        shape = (nz, self.n, self.n)
        if self._obj_rt is None or self._obj_rt.shape != shape or self._obj_rt.dtype != dt:
            self._obj_rt = pinned_empty(shape, dt)
        tomo = self._engine(min(nz, self._max_nz) if nz > self._max_nz else nz)
        step = tomo._nz
        for z0 in range(0, nz, step):
            z1 = min(nz, z0 + step)
            part = np.ascontiguousarray(sino[:, z0:z1, :], dtype=dt)
            self._obj_rt[z0:z1] = tomo.RT(part)
        return self._obj_rt
