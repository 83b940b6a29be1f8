"""FP64 NumPy restatement of the reference's FBP filter -- test infrastructure.

Only tests/, smoke() and bench.py's CPU legs use this module, as the checker;
the product filter is the CUDA kernel in model_mosaic_b200/csrc/fbp.cu.

processing/fbp_filter.py (vendored from tomocupy): a 1-D filter along the last
axis of a real sinogram row of length n, edge-replicated to ne = 4n
(:142-150,182-186), rfft -> multiply by the real weights w (ne/2 + 1) ->
irfft (numpy/cupy 'backward' norm, i.e. the inverse divides by ne) -> crop the
centre n (:187-191).  Weights (:49-88): t = k/ne; a shape factor per filter
name times ne/2 times the 12-point quadrature weights _wint(12, t)
(:90-126), clipped at zero, doubled, w[0] doubled again, times 3n, cast to
float32.
"""
from __future__ import annotations

import numpy as np

FILTERS = ("none", "ramp", "shepp", "cosine", "cosine2", "hamming", "hann", "parzen")


def wint(n: int, t: np.ndarray) -> np.ndarray:
    """Quadrature weights of processing/fbp_filter.py:90-126 (FP64)."""
    N = len(t)
    s = np.linspace(1e-40, 1, n)
    tmp1 = np.arange(n)
    tmp2 = np.arange(1, n + 2)
    iv = np.linalg.inv(np.exp(np.outer(tmp1, np.log(s))))
    u = np.diff(np.exp(np.outer(tmp2, np.log(s))) * np.tile(1.0 / tmp2[..., np.newaxis], [1, n]))
    W1 = iv @ u[1:n + 1, :]
    W2 = iv @ u[0:n, :]
    p = 1 / np.concatenate((np.arange(1, n), (n - 1) * np.ones(N - 2 * (n - 1) - 1), np.arange(n - 1, 0, -1)))
    w = np.zeros(N)
    for j in range(N - n + 1):
        W = ((t[j + n - 1] - t[j]) ** 2) * W1 + (t[j + n - 1] - t[j]) * t[j] * W2
        for k in range(n - 1):
            w[j:j + n] = w[j:j + n] + p[j + k] * W[:, k]
    if N > 40:
        w[-40:] = (w[-40]) / (N - 40) * np.arange(N - 40, N)
    return w


def calc_filter(n: int, name: str) -> np.ndarray:
    """(2n + 1,) float32 weights, processing/fbp_filter.py:49-88."""
    d = 0.5
    ne = 4 * n
    t = np.arange(0, ne // 2 + 1) / ne
    if name == "none":
        wfa = ne * 0.5 + t * 0
        wfa[0] *= 2
    elif name == "ramp":
        wfa = ne * 0.5 * wint(12, t)
    elif name == "shepp":
        wfa = ne * 0.5 * wint(12, t) * np.sinc(t / (2 * d)) * (t / d <= 2)
    elif name == "cosine":
        wfa = ne * 0.5 * wint(12, t) * np.cos(np.pi * t / (2 * d)) * (t / d <= 1)
    elif name == "cosine2":
        wfa = ne * 0.5 * wint(12, t) * (np.cos(np.pi * t / (2 * d))) ** 2 * (t / d <= 1)
    elif name == "hamming":
        wfa = ne * 0.5 * wint(12, t) * (.54 + .46 * np.cos(np.pi * t / d)) * (t / d <= 1)
    elif name == "hann":
        wfa = ne * 0.5 * wint(12, t) * (1 + np.cos(np.pi * t / d)) / 2.0 * (t / d <= 1)
    elif name == "parzen":
        wfa = ne * 0.5 * wint(12, t) * (1 - t / d) ** 3 * (t / d <= 1)
    else:
        raise ValueError(f"unknown FBP filter '{name}'")
    wfa = 2 * wfa * (wfa >= 0)
    wfa[0] *= 2
    return (3 * n * wfa).astype(np.float32)


def filter_rows(sino: np.ndarray, w: np.ndarray) -> np.ndarray:
    """Filtered copy of `sino` (..., n) in FP64, processing/fbp_filter.py:182-191."""
    n = sino.shape[-1]
    ne = 4 * n
    pad = (ne - n) // 2
    x = np.asarray(sino, dtype=np.float64).reshape(-1, n)
    t = np.empty((x.shape[0], ne))
    t[:, pad:pad + n] = x
    t[:, :pad] = x[:, :1]
    t[:, pad + n:] = x[:, -1:]
    y = np.fft.irfft(np.fft.rfft(t, axis=-1) * np.asarray(w, dtype=np.float64), n=ne, axis=-1)
    return y[:, pad:pad + n].reshape(sino.shape)
