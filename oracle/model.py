"""FP64 oracle of the differentiable forward model and its gradient.

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.  Composes the
restated reference operators: p = R delta (processing/tomo.py:121-151),
psi = exp(-p s/beta_r)(cos p s, sin p s) (step3_propagation.py:94-103),
u = D psi (processing/propagation.py:47-64), data = |u|^2 (:105-110); the
L2 loss sum (|u|^2 - d)^2 and its gradient through the exact adjoints
(D^H = PropagationOracle.DT, R^T = TomoRealOracle.RT, the reference's RT).
"""
from __future__ import annotations

import numpy as np

from .usfft import TomoRealOracle
from .fresnel import PropagationOracle


class ModelOracle:
    """``dtype`` np.float64 is the oracle; np.float32 runs the same composition
    in the reference's float32/complex64 arithmetic (its rounding floor)."""

    def __init__(self, n, nz, theta, wavelength, voxelsize, distance, s, beta_ratio=100.0, dtype=np.float64):
        self.dtype = dtype
        self.tomo = TomoRealOracle(n, nz, theta, dtype=dtype)
        self.prop = PropagationOracle(n, nz, len(theta), 1, wavelength, voxelsize, [distance], dtype=dtype)
        self.s, self.ib = dtype(s), dtype(1.0 / float(beta_ratio))

    def psi(self, p):
        ph = (p * self.s).astype(self.dtype)
        ct = np.complex128 if self.dtype == np.float64 else np.complex64
        return (np.exp(-ph * self.ib) * (np.cos(ph) + 1j * np.sin(ph))).astype(ct)

    def forward(self, delta):
        return (np.abs(self.prop.D(self.psi(self.tomo.R(delta)), 0)) ** 2).astype(self.dtype)

    def loss(self, delta, d):
        return float(np.sum((self.forward(delta) - d) ** 2))

    def grad(self, delta, d):
        p = self.tomo.R(delta)
        psi = self.psi(p)
        u = self.prop.D(psi, 0)
        gu = (4 * (np.abs(u) ** 2 - d.astype(self.dtype)) * u).astype(u.dtype)
        gpsi = self.prop.DT(gu, 0)
        gp = (self.s * np.real(np.conj(gpsi) * (1j - self.ib) * psi)).astype(self.dtype)
        return self.tomo.RT(gp)
