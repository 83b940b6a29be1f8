"""PropagationLarge -- drop-in for processing/propagation_large.py on one B200.

The reference streams the padded (ntheta, 2nz, 2n) work buffer through pinned
host memory in three separable passes (propagation_large.py:36-53).  On a
B200 the propagator's kernels run device-resident on chunks of frames, so
this class keeps the host-array API -- numpy (or a banded pinned object with
``copy_to``) in, an internal pinned numpy buffer out, reused by the next call
(propagation_large.py:226-236) -- and validates the chunk sizes with the same
assertions (:216-223).  Frames are streamed: the copy-in of chunk i+1, D of
chunk i and the copy-out of chunk i-1 overlap on three streams
(``staging.ChunkStream``); the chunk is sized from the free device memory
(a 24576^2 frame, the reference scripts' ups = 8 size, is 4.8 GB).
"""
from __future__ import annotations

import numpy as np
import torch

from model_mosaic_b200._interop import pinned_empty, require_cuda
from model_mosaic_b200.processing.propagation import Propagation
from model_mosaic_b200.staging import ChunkStream


def chunk_frames(n, nz, ntheta, free_bytes):
    """Frames per chunk: two device buffers per side plus the handle's two
    work frames within about 40% of the free device memory."""
    per = 8.0 * n * nz * 6
    return max(1, min(ntheta, int(0.4 * free_bytes / per)))


class PropagationLarge:
    def __init__(self, n, nz, wavelength, voxelsize, distance):
        require_cuda()
        self.n, self.nz = int(n), int(nz)
        self.wavelength, self.voxelsize = float(wavelength), float(voxelsize)
        self.distance = np.atleast_1d(np.asarray(distance, dtype=np.float64))
        self._prop = None
        self._prop_nt = 0
        self._out = None
        self._psi = None
        self._stream = None

    def _engine(self, ntheta):
        """A handle for chunks of frames (at most ntheta), sized by memory."""
        free = torch.cuda.mem_get_info()[0] + (8 * self.n * self.nz * 2 * self._prop_nt if self._prop else 0)
        want = chunk_frames(self.n, self.nz, ntheta, free)
        if self._prop is None or self._prop_nt != want:
            if self._prop is not None:
                self._prop.free()
                self._prop = None
            self._prop_nt = want
            self._prop = Propagation(self.n, self.nz, want, self.distance.size, self.wavelength,
                                     self.voxelsize, self.distance)
        if self._stream is None:
            self._stream = ChunkStream()
        return self._prop

    def free(self):
        if self._prop is not None:
            self._prop.free()
        self._prop = None
        if self._stream is not None:
            self._stream.free()
        self._stream = None
        self._out = self._psi = None

    def psi_buffer(self, ntheta):
        """Pinned (ntheta, nz, n) complex64 buffer (propagation_large.py:177-199)."""
        shape = (ntheta, self.nz, self.n)
        if self._psi is None or self._psi.shape != shape:
            self._psi = pinned_empty(shape, np.complex64)
        return self._psi

    def _run(self, psi, j, chunks, adjoint):
        added = psi.ndim == 2
        if added:
            psi = psi[np.newaxis]
        ntheta, nz_in, n_in = psi.shape
        assert nz_in == self.nz and n_in == self.n, \
            f"psi shape (…, {nz_in}, {n_in}) mismatches propagator ({self.nz}, {self.n})"
        chunk_nz, chunk_2n = chunks
        assert self.nz % chunk_nz == 0, f"CHUNK_NZ={chunk_nz} must divide nz={self.nz}"
        assert (2 * self.n) % chunk_2n == 0, f"CHUNK_2N={chunk_2n} must divide 2n={2*self.n}"
        if hasattr(psi, "copy_to"):
            host = np.empty(psi.shape, np.complex64)
            psi.copy_to(host, np.s_[:, :, :])
            psi = host
        shape = (ntheta, self.nz, self.n)
        if self._out is None or self._out.shape != shape:
            self._out = pinned_empty(shape, np.complex64)
        prop = self._engine(ntheta)
        step = self._prop_nt
        chunks_t = [(t0, min(ntheta, t0 + step)) for t0 in range(0, ntheta, step)]
        out = self._out
        run = prop.DT_into if adjoint else prop.D_into

        def load(k, dst):
            dst[...] = psi[k[0]:k[1]]

        def store(k, src):
            out[k[0]:k[1]] = src

        fshape = lambda k: (k[1] - k[0], self.nz, self.n)  # noqa: E731
        self._stream.run(chunks_t, fshape, np.complex64, fshape, np.complex64, load,
                         lambda k, x, y: run(x, y, j), store)
        return self._out[0] if added else self._out

    def D(self, psi, j, chunks):
        """Forward Fresnel propagation with the j-th distance (propagation_large.py:202-236)."""
        return self._run(psi, j, chunks, False)

    def DT(self, g, j, chunks):
        """Adjoint of D (no reference counterpart)."""
        return self._run(g, j, chunks, True)
