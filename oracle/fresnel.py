"""NumPy restatement of the reference's Fresnel propagator and the two
elementwise stages around it.

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.

* fker = exp(-i pi lambda z (fx^2 + fy^2)) / (4 n nz) .. processing/propagation.py:23-31
* symmetric mirror pad (pad_fwd) ....................... processing/kernels.py:530-550
* D = crop(ifft2_unnormalised(fker * fft2(pad(psi)))) ... processing/propagation.py:47-64
* separable three-pass D (PropagationLarge) ............ processing/propagation_large.py:202-348
* psi = exp(-p s / beta_r) (cos p s, sin p s) ......... step3_propagation.py:94-103
* |u|^2 ................................................ step3_propagation.py:105-110

``DT`` has no reference counterpart (the reference ships only the forward
operator, processing/propagation_large.py:15); it is the exact adjoint
fold(ifft2_unnormalised(conj(fker) * fft2(embed(g)))) of ``D``.
"""
from __future__ import annotations

import numpy as np


def _ctype(dtype):
    return np.complex128 if np.dtype(dtype) == np.float64 else np.complex64


def mirror_index(n: int):
    """Source index of each of the 2n padded positions (kernels.py:541-544)."""
    t = np.arange(2 * n)
    return np.where(t < n // 2, n // 2 - t - 1,
                    np.where(t >= n + n // 2, 2 * n - t + n // 2 - 1, t - n // 2))


def fresnel_kernel(n, nz, wavelength, voxelsize, distance, dtype=np.float64):
    """fker[j] (ndist, 2nz, 2n) -- propagation.py:23-31.  The frequency grids
    are float32 as in the reference; the phase is evaluated in ``dtype``."""
    fx = np.fft.fftfreq(2 * n, d=voxelsize).astype(np.float32).astype(dtype)
    fy = np.fft.fftfreq(2 * nz, d=voxelsize).astype(np.float32).astype(dtype)
    fx, fy = np.meshgrid(fx, fy)
    f2 = fx ** 2 + fy ** 2
    norm = float(4 * n * nz)
    out = np.empty((len(distance), 2 * nz, 2 * n), dtype=_ctype(dtype))
    for j, z in enumerate(distance):
        out[j] = np.exp(-1j * np.pi * wavelength * z * f2) / norm
    return out


class PropagationOracle:
    """Restatement of Propagation (processing/propagation.py:15-64) plus DT."""

    def __init__(self, n, nz, ntheta, ndist, wavelength, voxelsize, distance, dtype=np.float64):
        self.n, self.nz, self.dtype = n, nz, dtype
        self.fker = fresnel_kernel(n, nz, wavelength, voxelsize, list(distance)[:ndist], dtype)
        self.ix = mirror_index(n)
        self.iy = mirror_index(nz)

    def _pad(self, psi):
        return psi[:, self.iy][:, :, self.ix]

    def D(self, psi, j):
        """propagation.py:47-64: 2-D input gives 2-D output."""
        ct = _ctype(self.dtype)
        added = psi.ndim == 2
        if added:
            psi = psi[None]
        f = self._pad(psi.astype(ct))
        f = np.fft.fft2(f, axes=(-2, -1)).astype(ct)
        f = f * self.fker[j]
        f = np.fft.ifft2(f, axes=(-2, -1), norm="forward").astype(ct)
        n, nz = self.n, self.nz
        res = f[:, nz // 2:nz // 2 + nz, n // 2:n // 2 + n]
        return res[0] if added else res

    def DT(self, g, j):
        """Adjoint of D: zero-embed, fft2, * conj(fker), unnormalised ifft2,
        fold the mirrored borders back onto their source pixels."""
        ct = _ctype(self.dtype)
        added = g.ndim == 2
        if added:
            g = g[None]
        n, nz = self.n, self.nz
        nt = g.shape[0]
        f = np.zeros((nt, 2 * nz, 2 * n), dtype=ct)
        f[:, nz // 2:nz // 2 + nz, n // 2:n // 2 + n] = g
        f = np.fft.fft2(f, axes=(-2, -1)).astype(ct)
        f = f * np.conj(self.fker[j])
        f = np.fft.ifft2(f, axes=(-2, -1), norm="forward").astype(ct)
        # fold along x then y (adjoint of the gather psi[:, iy][:, :, ix])
        fx = np.zeros((nt, 2 * nz, n), dtype=ct)
        for t in range(2 * n):
            fx[:, :, self.ix[t]] += f[:, :, t]
        out = np.zeros((nt, nz, n), dtype=ct)
        for t in range(2 * nz):
            out[:, self.iy[t], :] += fx[:, t, :]
        return out[0] if added else out


class PropagationLargeOracle:
    """Restatement of PropagationLarge.D's separable passes
    (processing/propagation_large.py:55-79, 239-348): x-pad, FFT_x, *K_x;
    y-pad, FFT_y, *K_y, IFFT_y (/2nz), crop y; IFFT_x (/2n), crop x."""

    def __init__(self, n, nz, wavelength, voxelsize, distance, dtype=np.float64):
        self.n, self.nz, self.dtype = n, nz, dtype
        ct = _ctype(dtype)
        dist = np.atleast_1d(np.asarray(distance, dtype=np.float64))
        fx = np.fft.fftfreq(2 * n, d=voxelsize).astype(np.float32).astype(dtype)
        fy = np.fft.fftfreq(2 * nz, d=voxelsize).astype(np.float32).astype(dtype)
        self.Kx = np.stack([np.exp(-1j * np.pi * wavelength * L * fx * fx) for L in dist]).astype(ct)
        self.Ky = np.stack([np.exp(-1j * np.pi * wavelength * L * fy * fy) for L in dist]).astype(ct)
        self.ix = mirror_index(n)
        self.iy = mirror_index(nz)

    def D(self, psi, j, chunks=None):
        ct = _ctype(self.dtype)
        added = psi.ndim == 2
        if added:
            psi = psi[None]
        n, nz = self.n, self.nz
        f = psi.astype(ct)[:, :, self.ix]
        f = np.fft.fft(f, axis=-1) * self.Kx[j]
        f = f[:, self.iy, :]
        f = np.fft.fft(f, axis=1) * self.Ky[j][:, None]
        f = np.fft.ifft(f, axis=1)[:, nz // 2:nz // 2 + nz, :]
        f = np.fft.ifft(f, axis=-1)[:, :, n // 2:n // 2 + n]
        res = f.astype(ct)
        return res[0] if added else res


def psi_from_proj(p, inv_norm, inv_beta_ratio, dtype=np.float64):
    """step3_propagation.py:94-103."""
    phase = p.astype(dtype) * dtype(inv_norm)
    atten = np.exp(-phase * dtype(inv_beta_ratio))
    return (atten * np.cos(phase) + 1j * atten * np.sin(phase)).astype(_ctype(dtype))


def abs2(u):
    """step3_propagation.py:105-110."""
    return (u.real * u.real + u.imag * u.imag)
