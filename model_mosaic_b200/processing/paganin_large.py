"""PaganinLarge -- drop-in for processing/paganin_large.py on one B200.

The reference streams its (ntheta, nz, n//2+1) spectrum through pinned host
memory in three chunked passes (processing/paganin_large.py:42-145) because it
did not fit its GPUs.  On a B200 the three passes run device-resident
(``Paganin``), so this class keeps the host-array API -- numpy in, an internal
pinned numpy buffer out that the next call reuses -- and validates the chunk
sizes with the reference's assertions (:130-135).
"""
from __future__ import annotations

import numpy as np
import torch

from model_mosaic_b200._interop import pinned_empty, require_cuda
from model_mosaic_b200.processing.paganin import Paganin


class PaganinLarge:
    def __init__(self, n, nz, wavelength, voxelsize, distance, alpha):
        require_cuda()
        self.n, self.nz = int(n), int(nz)
        self.wavelength, self.voxelsize = float(wavelength), float(voxelsize)
        self.distance, self.alpha = float(distance), float(alpha)
        self._pgn = None
        self._pgn_nt = 0
        self._out = None

    def _engine(self, ntheta):
        if self._pgn is None or self._pgn_nt < ntheta:
            if self._pgn is not None:
                self._pgn.free()
            self._pgn_nt = ntheta
            self._pgn = Paganin(self.n, self.nz, ntheta, self.wavelength, self.voxelsize, self.distance,
                                self.alpha)
        return self._pgn

    def free(self):
        if self._pgn is not None:
            self._pgn.free()
        self._pgn = None
        self._out = None

    def retrieve(self, intensity, chunks):
        """(ntheta, nz, n) or (nz, n) host float32 intensity -> host phase of the
        same shape in an internal pinned buffer (reused by the next call)."""
        added = intensity.ndim == 2
        if added:
            intensity = intensity[np.newaxis]
        ntheta, nz_in, n_in = intensity.shape
        assert nz_in == self.nz and n_in == self.n, \
            f"intensity shape (…, {nz_in}, {n_in}) mismatches ({self.nz}, {self.n})"
        chunk_nz, chunk_n = chunks
        assert self.nz % chunk_nz == 0, f"CHUNK_NZ={chunk_nz} must divide nz={self.nz}"
        assert self.n % chunk_n == 0, f"CHUNK_N={chunk_n} must divide n={self.n}"
        pgn = self._engine(ntheta)
        x = torch.from_numpy(np.ascontiguousarray(intensity, dtype=np.float32)).cuda()
        y = torch.empty_like(x)
        pgn.retrieve_into(x, y)
        if self._out is None or self._out.shape != intensity.shape:
            self._out = pinned_empty(intensity.shape, np.float32)
        self._out[...] = y.cpu().numpy()
        return self._out[0] if added else self._out
