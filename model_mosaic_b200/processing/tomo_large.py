"""TomoLargeReal -- drop-in for processing/tomo_large.py on one B200.

The reference stages its (nz, 2n, n+1) spectrum through pinned host memory
because it did not fit on the GPUs it targeted (processing/tomo_large.py:1-19).
A B200 holds a slab of slices of the forward model in HBM, so this class
keeps the reference's host-array API -- numpy in, numpy out, results in
internal pinned buffers that the next call reuses (tomo_large.py:545-555,
611) -- and runs the same device-resident USFFT as ``TomoReal`` on slabs of
slices, streamed: the copy-in of slab i+1, the transform of slab i and the
copy-out of slab i-1 overlap on three streams (``staging.ChunkStream``, as
the reference's StreamPipe, processing/pipeline.py:255-359).  The slab is
sized from the free device memory (a 24576^2 slice, the reference scripts'
ups = 8 size, takes about 30 GB of workspace).

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
from model_mosaic_b200.staging import ChunkStream


def slab_slices(n, ntheta, nz, max_nz, free_bytes):
    """Slices per slab: a power of two (the handle pads slabs to one) whose
    workspace -- the two (2n, n+1) spectra, the cuFFT x-side rows, the polar
    lines, the scatter table share and the streamed buffers -- fits in
    about half of the free device memory."""
    per_slice = 8.0 * 2 * n * (n + 1) * 2 + 4.0 * n * 2 * n + 8.0 * n * (n + 1) + 12.0 * ntheta * n * 2 + 16.0 * n * n
    fit = max(1, int(0.5 * free_bytes / per_slice))
    z = 1
    while z * 2 <= min(max_nz, nz, fit):
        z *= 2
    return z


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
        self._stream = None

    def _engine(self, nz):
        """A TomoReal handle for slabs of up to `nz` slices, sized by memory."""
        want = slab_slices(self.n, self.ntheta, nz, self._max_nz, torch.cuda.mem_get_info()[0]
                           + (self._tomo.workspace_bytes() if self._tomo is not None else 0))
        if self._tomo is None or self._tomo_nz != want:
            if self._tomo is not None:
                self._tomo.free()
                self._tomo = None
            self._tomo_nz = want
            self._tomo = TomoReal(self.n, want, self.theta, eps=self._eps, m=self._m, clamp_xy=True)
        if self._stream is None:
            self._stream = ChunkStream()
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
        if self._stream is not None:
            self._stream.free()
        self._stream = None
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
        nz, n, T = obj.shape[0], self.n, self.ntheta
        shape = (T, nz, n)
        if self._sino is None or self._sino.shape != shape:
            self._sino = pinned_empty(shape, np.float32)
        tomo = self._engine(nz)
        step = tomo._nz
        slabs = [(z0, min(nz, z0 + step)) for z0 in range(0, nz, step)]
        sino = self._sino

        def load(k, dst):
            dst[...] = obj[k[0]:k[1]]

        def store(k, src):
            sino[:, k[0]:k[1], :] = src

        self._stream.run(slabs, lambda k: (k[1] - k[0], n, n), np.float32, lambda k: (T, k[1] - k[0], n),
                         np.float32, load, lambda k, x, y: tomo.R_into(x, y), store)
        return self._sino

    def RT(self, sino, chunks):
        """(ntheta, nz, n) host sino (float32 or complex64) -> (nz, n, n) host
        obj of the matching dtype, in an internal buffer (tomo_large.py:582-630)."""
        self._check_chunks(chunks)
        sino = np.asarray(sino)
        T, nz, n = sino.shape[0], sino.shape[1], self.n
        dt = np.complex64 if np.iscomplexobj(sino) else np.float32
        shape = (nz, n, n)
        if self._obj_rt is None or self._obj_rt.shape != shape or self._obj_rt.dtype != dt:
            self._obj_rt = pinned_empty(shape, dt)
        tomo = self._engine(nz)
        step = tomo._nz
        slabs = [(z0, min(nz, z0 + step)) for z0 in range(0, nz, step)]
        out = self._obj_rt

        def load(k, dst):
            dst[...] = sino[:, k[0]:k[1], :]

        def store(k, src):
            out[k[0]:k[1]] = src

        self._stream.run(slabs, lambda k: (T, k[1] - k[0], n), dt, lambda k: (k[1] - k[0], n, n), dt, load,
                         lambda k, x, y: tomo.RT_into(x, y), store)
        return self._obj_rt
