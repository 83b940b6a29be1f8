"""NumPy restatement of the reference's USFFT Radon transform pair.

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.  Every function
follows a reference file:line and keeps its arithmetic and conventions:

* parameters (eps=1e-3, mu, m) ............ processing/tomo.py:39-42
* phi deapodisation incl. (1 - n%4) ....... processing/tomo.py:46-49,59
* c1dfftshift / c2dfftshift ............... processing/tomo.py:51, 98-99
* R: pad, rfft2, gather, r-IFFT, .real/4 .. processing/tomo.py:121-151
* gather from the rfft half spectrum ...... processing/kernels.py:274-349
* RT: r-FFT, scatter, ifft2, crop*phi ..... processing/tomo.py:153-188
* scatter (gather kernel, dir=1) .......... processing/kernels.py:16-93
* TomoLargeReal R (x0/y0 clamp) ........... processing/tomo_large.py:344-579,
                                            processing/kernels.py:451-526

``dtype`` selects the arithmetic: ``np.float64`` gives the FP64 oracle,
``np.float32`` mimics the reference's float32/complex64 storage.
"""
from __future__ import annotations

import math

import numpy as np


def usfft_params(n: int, eps: float = 1e-3):
    """(mu, m) exactly as processing/tomo.py:39-42."""
    mu = -math.log(eps) / (2 * n * n)
    m = math.ceil(2 * n / math.pi * math.sqrt(-mu * math.log(eps) + (mu * n) ** 2 / 4))
    return mu, m


def _ctype(dtype):
    return np.complex128 if np.dtype(dtype) == np.float64 else np.complex64


def phi_table(n: int, ntheta: int, mu: float, dtype=np.float64):
    """Deapodisation factor phi(y, x) -- processing/tomo.py:46-49,59."""
    t = np.linspace(-0.5, 0.5, n, endpoint=False).astype(dtype)
    dx, dy = np.meshgrid(t, t)
    phi = np.exp((dtype(mu * (n * n)) * (dx * dx + dy * dy)).astype(dtype)) * dtype(1 - n % 4)
    phi = phi * dtype(1.0 / (n * np.sqrt(n * ntheta)))
    return phi.astype(dtype)


def c1dfftshift(n: int):
    """(-1)^(i+1) sign table -- processing/tomo.py:51."""
    return (1 - 2 * (np.arange(1, n + 1) % 2)).astype(np.int8)


def _mu32(mu):
    # The kernels receive mu as a float32 device scalar (tomo.py:53).
    return float(np.float32(mu))


def _polar(n, theta, dtype, clamp=False):
    """Sample coordinates of the gather kernels (kernels.py:293-295 and the
    clamped variant kernels.py:475-481)."""
    tx = np.arange(n, dtype=dtype)
    r = (tx - dtype(n * 0.5)) / dtype(n)
    th = theta.astype(np.float32).astype(dtype)
    x0 = r[None, :] * np.cos(th)[:, None]
    y0 = -r[None, :] * np.sin(th)[:, None]
    if clamp:
        x0 = np.clip(x0, dtype(-0.5), dtype(0.5 - 1e-5))
        y0 = np.clip(y0, dtype(-0.5), dtype(0.5 - 1e-5))
    return x0.astype(dtype), y0.astype(dtype)


def _window(n, m, mu, x0, y0, dtype):
    """Symmetric (2m+1) window centred with rint and its separable Gaussian
    weights (kernels.py:298-315).  Returns ell0, ell1 (T,n,L) and ex, ey."""
    twon = 2 * n
    mu = dtype(_mu32(mu))
    coeff0 = dtype(np.pi) / mu
    coeff1 = -dtype(np.pi) * dtype(np.pi) / mu
    inv_twon = dtype(1.0) / dtype(twon)
    bx = np.rint(dtype(twon) * x0).astype(np.int64) - m
    by = np.rint(dtype(twon) * y0).astype(np.int64) - m
    i = np.arange(2 * m + 1)
    ell0 = bx[..., None] + i
    ell1 = by[..., None] + i
    w0 = (ell0 * inv_twon).astype(dtype) - x0[..., None]
    w1 = (ell1 * inv_twon).astype(dtype) - y0[..., None]
    ex = np.exp(coeff1 * w0 * w0).astype(dtype)
    ey = (coeff0 * np.exp(coeff1 * w1 * w1)).astype(dtype)
    return ell0, ell1, ex, ey


def gather_rfft_full(fde, theta, n, m, mu, dtype=np.float64, clamp=False, zchunk=8, tchunk=None):
    """Polar gather from the (nz, 2n, n+1) raw-order rfft2 half spectrum with
    conjugate reflection for k0 > n and the (-1)^(k0+k1) sign; divides by n.
    processing/kernels.py:274-349 (clamp=True: kernels.py:451-526).
    Returns g with shape (ntheta, nz, n).  Angles are taken `tchunk` at a
    time (default: enough to keep each index array near 2^23 taps), which
    bounds the memory at production sizes; the arithmetic per sample is the
    same whatever the chunking."""
    ct = _ctype(dtype)
    nz = fde.shape[0]
    T = len(theta)
    L = 2 * m + 1
    if tchunk is None:
        tchunk = max(1, (1 << 23) // (n * L * L))
    g = np.empty((T, nz, n), dtype=ct)
    fde = fde.astype(ct, copy=False)
    for t0 in range(0, T, tchunk):
        t1 = min(T, t0 + tchunk)
        g[t0:t1] = _gather_angles(fde, np.asarray(theta)[t0:t1], n, m, mu, dtype, clamp, zchunk)
    return g


def _gather_angles(fde, theta, n, m, mu, dtype, clamp, zchunk):
    ct = _ctype(dtype)
    nz = fde.shape[0]
    T = len(theta)
    twon = 2 * n
    x0, y0 = _polar(n, theta, dtype, clamp)
    ell0, ell1, ex, ey = _window(n, m, mu, x0, y0, dtype)
    k0 = np.mod(ell0, twon)[:, :, None, :]
    ky = np.mod(ell1, twon)[:, :, :, None]
    w = ey[:, :, :, None] * ex[:, :, None, :]
    sign = np.where(((k0 + ky) & 1) == 1, -1.0, 1.0).astype(dtype)
    refl = np.broadcast_to(k0 > n, w.shape)
    rkx = np.where(refl, twon - k0, k0)
    rky = np.where(refl, np.mod(twon - ky, twon), ky)
    sw = (sign * w).astype(dtype)
    g = np.empty((T, nz, n), dtype=ct)
    for z0 in range(0, nz, zchunk):
        z1 = min(nz, z0 + zchunk)
        v = fde[z0:z1][:, rky, rkx]                      # (zc, T, n, L, L)
        v = np.where(refl[None], np.conj(v), v)
        acc = np.sum(sw[None] * v, axis=(-2, -1))
        g[:, z0:z1, :] = (acc / dtype(n)).astype(ct).transpose(1, 0, 2)
    return g


def scatter_full(g, theta, n, m, mu, dtype=np.float64, tchunk=None):
    """Adjoint scatter of the full-complex gather kernel (dir=1): every
    sample adds w * g into f[(n + ell1) % 2n, (n + ell0) % 2n]; no divide by n.
    processing/kernels.py:16-93.  g: (ntheta, nz, n) -> f: (nz, 2n, 2n).
    Angles are summed `tchunk` at a time into float64 accumulators (the
    reference's float atomics have no fixed order, so neither does this)."""
    ct = _ctype(dtype)
    T, nz, _ = g.shape
    twon = 2 * n
    L = 2 * m + 1
    if tchunk is None:
        tchunk = max(1, (1 << 23) // (n * L * L))
    re = np.zeros((nz, twon * twon), dtype=np.float64)
    im = np.zeros((nz, twon * twon), dtype=np.float64)
    th = np.asarray(theta)
    for t0 in range(0, T, tchunk):
        t1 = min(T, t0 + tchunk)
        x0, y0 = _polar(n, th[t0:t1], dtype)
        ell0, ell1, ex, ey = _window(n, m, mu, x0, y0, dtype)
        w = (ex[:, :, None, :] * ey[:, :, :, None]).astype(dtype)   # ex[i0]*ey (kernels.py:68)
        fy = np.mod(n + ell1, twon)[:, :, :, None]
        fx = np.mod(n + ell0, twon)[:, :, None, :]
        idx = np.broadcast_to(fy * twon + fx, w.shape).reshape(-1)
        wf = w.reshape(t1 - t0, n, -1)
        for z in range(nz):
            val = (wf * g[t0:t1, z, :, None]).reshape(-1)
            re[z] += np.bincount(idx, weights=val.real.astype(np.float64), minlength=twon * twon)
            im[z] += np.bincount(idx, weights=val.imag.astype(np.float64), minlength=twon * twon)
    return (re + 1j * im).reshape(nz, twon, twon).astype(ct)


class TomoRealOracle:
    """Restatement of TomoReal (processing/tomo.py:17-188)."""

    def __init__(self, n, nz, theta, dtype=np.float64, eps=1e-3):
        self.n, self.nz = n, nz
        self.theta = np.asarray(theta, dtype=np.float32)
        self.ntheta = len(self.theta)
        self.dtype = dtype
        self.mu, self.m = usfft_params(n, eps)
        self.phi = phi_table(n, self.ntheta, self.mu, dtype)
        self.c1d = c1dfftshift(n)
        c2 = (1 - 2 * (np.arange(1, 2 * n + 1) % 2)).astype(np.int8)
        self.c2d = np.outer(c2, c2)

    def R(self, obj, clamp=False):
        """tomo.py:121-151 -> (ntheta, nz, n) real."""
        d, n = self.dtype, self.n
        ct = _ctype(d)
        nz = obj.shape[0]
        padded = np.zeros((nz, 2 * n, 2 * n), dtype=d)
        padded[:, n // 2:3 * n // 2, n // 2:3 * n // 2] = obj.astype(d) * self.phi
        fde = np.fft.rfft2(padded, axes=(-2, -1)).astype(ct)
        g = gather_rfft_full(fde, self.theta, n, self.m, self.mu, d, clamp)
        g = g * self.c1d
        g = np.fft.ifft(g, axis=-1).astype(ct)
        g = g * self.c1d
        return (g.real / d(4)).astype(d)

    def RT(self, data):
        """tomo.py:153-188 -> (nz, n, n); real output for real input."""
        d, n = self.dtype, self.n
        ct = _ctype(d)
        real_in = not np.iscomplexobj(data)
        s = (data * self.c1d).astype(ct)
        s = np.fft.fft(s, axis=-1).astype(ct)
        s = s * self.c1d
        f = scatter_full(s, self.theta, n, self.m, self.mu, d)
        f = f * self.c2d
        f = np.fft.ifft2(f, axes=(-2, -1)).astype(ct)
        f = f * self.c2d
        res = f[:, n // 2:3 * n // 2, n // 2:3 * n // 2] * self.phi
        return (res.real.astype(d) if real_in else res.astype(ct))


class TomoLargeRealOracle(TomoRealOracle):
    """Restatement of TomoLargeReal's math (processing/tomo_large.py:46-838).

    Forward: the same pipeline with the gather's x0/y0 clamp
    (kernels.py:478-481) and the 1/(4 n sqrt(n ntheta)) scale applied after
    the r-IFFT instead of inside phi (tomo_large.py:543,576).  The adjoint
    passes (tomo_large.py:632-838) compute the same operator as TomoReal.RT.
    """

    def R(self, obj, chunks=None):
        return super().R(obj, clamp=True)

    def RT(self, data, chunks=None):
        return super().RT(data)


def radon_direct(obj, theta, dtype=np.float64):
    """Exact non-uniform DFT version of the same operator (method check, not a
    parity gate): TomoReal.R with the Gaussian gridding replaced by a direct
    sum over the image pixels, then the same r-IFFT, shifts and scale.  The
    difference to R is the USFFT approximation error at eps=1e-3."""
    nz, n, _ = obj.shape
    th = np.asarray(theta, np.float32).astype(np.float64)
    T = len(th)
    r = (np.arange(n) - n * 0.5) / n
    xs = np.arange(n) - n // 2                           # pixel coordinates (centred)
    out = np.empty((T, nz, n), dtype=np.float64)
    c1 = c1dfftshift(n)
    # The 2-D Gaussian (pi/mu) exp(-pi^2 |d|^2/mu) integrates to 1 and its
    # transform exp(-mu |X|^2) is undone by phi; summed on the (2n)^2 grid and
    # divided by n in the gather, the continuous limit of the gathered sample
    # is 4n (1 - n%4) / (n sqrt(n T)) * sum_X obj(X) exp(-2 pi i x.X).
    scale = 4.0 * (1 - n % 4) / np.sqrt(n * T)
    for t in range(T):
        kx = r * np.cos(th[t]) * 2 * np.pi
        ky = -r * np.sin(th[t]) * 2 * np.pi
        ex = np.exp(-1j * np.outer(kx, xs))              # (n_r, n_x)
        ey = np.exp(-1j * np.outer(ky, xs))              # (n_r, n_y)
        for z in range(nz):
            g = np.einsum('ry,yx,rx->r', ey, obj[z].astype(np.float64), ex) * scale
            g = g * c1
            g = np.fft.ifft(g) * c1
            out[t, z] = g.real / 4
    return out.astype(dtype)
