"""The CPU oracle against the golden fixtures made from the reference's own
kernels (tests/golden/make_golden.py), plus the oracle's internal identities.
No GPU needed."""
import os

import numpy as np
import pytest

from oracle.usfft import TomoRealOracle, TomoLargeRealOracle, radon_direct, usfft_params
from oracle.fresnel import (PropagationOracle, PropagationLargeOracle, psi_from_proj,
                            abs2, mirror_index)

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rl2(a, b):
    return float(np.linalg.norm(np.asarray(a) - b) / np.linalg.norm(b))


def load(name):
    return np.load(os.path.join(GOLD, name))


def test_params_match_reference_constants():
    # eps = 1e-3 gives m = 4 for every n (processing/tomo.py:39-42)
    for n in (16, 64, 128, 512, 2048, 3072, 24576):
        assert usfft_params(n)[1] == 4


def test_oracle_R_vs_golden():
    g = load("tomo_R_n64_nz16_t24.npz")
    o = TomoRealOracle(64, 16, g["theta"])
    assert rl2(o.R(g["obj"]), g["sino"]) < 1e-5
    ol = TomoLargeRealOracle(64, 16, g["theta"])
    assert rl2(ol.R(g["obj"]), g["sino_large"]) < 1e-5


def test_oracle_RT_vs_golden():
    g = load("tomo_RT_n64_nz8_t24.npz")
    o = TomoRealOracle(64, 8, g["theta"])
    assert rl2(o.RT(g["sino_r"]), g["obj_r"]) < 1e-5
    rc = o.RT(g["sino_c"])
    assert np.iscomplexobj(rc) and rl2(rc, g["obj_c"]) < 1e-5


def test_oracle_n48_half_range_vs_golden():
    g = load("tomo_n48_nz3_t30.npz")
    o = TomoRealOracle(48, 3, g["theta"])
    assert rl2(o.R(g["obj"]), g["sino"]) < 1e-5
    assert rl2(o.RT(g["y"]), g["RTy"]) < 1e-5


def test_oracle_adjoint_identity_fp64():
    g = load("tomo_adjoint_n64_nz8_t24.npz")
    o = TomoRealOracle(64, 8, g["theta"])
    x, y = g["x"].astype(np.float64), g["y"].astype(np.float64)
    lhs, rhs = np.sum(o.R(x) * y), np.sum(x * o.RT(y))
    assert abs(lhs - rhs) / abs(lhs) < 1e-12
    # the reference's own FP32 kernels satisfy it to the reference's 1e-4 gate
    assert abs(np.sum(g["Rx"] * g["y"]) - np.sum(g["x"] * g["RTy"])) / abs(lhs) < 1e-4


def test_oracle_method_error_vs_direct_sum():
    # USFFT at eps=1e-3 approximates the exact non-uniform DFT to ~1e-3 (not a parity gate)
    theta = np.linspace(0, np.pi, 20, endpoint=False).astype(np.float32)
    x = np.random.default_rng(1).standard_normal((1, 32, 32))
    err = rl2(TomoRealOracle(32, 1, theta).R(x), radon_direct(x, theta))
    assert 1e-5 < err < 3e-3


def test_oracle_D_vs_golden_and_large():
    g = load("prop_D_n64_nz32_t3.npz")
    dist = list(g["distance"])
    P = PropagationOracle(64, 32, 3, 3, float(g["wavelength"]), float(g["voxelsize"]), dist)
    PL = PropagationLargeOracle(64, 32, float(g["wavelength"]), float(g["voxelsize"]), dist)
    for j in range(3):
        assert rl2(P.D(g["psi"], j), g["D"][j]) < 1e-5
        assert rl2(PL.D(g["psi"], j), g["D"][j]) < 1e-5
    assert np.abs(P.D(g["psi"], 0) - g["psi"]).max() < 1e-5     # L=0 is the identity


def test_oracle_D_DT_adjoint():
    rng = np.random.default_rng(3)
    P = PropagationOracle(32, 16, 2, 1, 4.13e-11, 1.4e-6, [0.05])
    a = rng.standard_normal((2, 16, 32)) + 1j * rng.standard_normal((2, 16, 32))
    b = rng.standard_normal((2, 16, 32)) + 1j * rng.standard_normal((2, 16, 32))
    lhs, rhs = np.vdot(b, P.D(a, 0)), np.vdot(P.DT(b, 0), a)
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_mirror_index_matches_pad_fwd():
    # kernels.py:541-542 for n = 8: [3,2,1,0, 0..7, 7,6,5,4]
    assert list(mirror_index(8)) == [3, 2, 1, 0, 0, 1, 2, 3, 4, 5, 6, 7, 7, 6, 5, 4]


def test_psi_abs2():
    p = np.array([0.0, 1.0, -2.0], np.float32)
    psi = psi_from_proj(p, 0.5, 0.01)
    ph = p * 0.5
    assert np.allclose(psi, np.exp(-ph * 0.01) * np.exp(1j * ph))
    assert np.allclose(abs2(psi), np.exp(-2 * ph * 0.01))


def test_model_oracle_gradient_vs_central_differences():
    # FP64 check of the chain rule used by the hand-written backward
    from oracle.model import ModelOracle
    n, nz, T = 32, 4, 24
    theta = np.linspace(0, np.pi, T, endpoint=False).astype(np.float32)
    rng = np.random.default_rng(0)
    m = ModelOracle(n, nz, theta, 4.133e-11, 0.69e-6, 0.12, s=40.0)
    delta = rng.uniform(0, 1, (nz, n, n)) * 1e-2
    d = m.forward(rng.uniform(0, 1, (nz, n, n)) * 1e-2)
    g = m.grad(delta, d)
    for _ in range(3):
        v = rng.standard_normal(delta.shape)
        h = 1e-6
        fd = (m.loss(delta + h * v, d) - m.loss(delta - h * v, d)) / (2 * h)
        assert abs(np.sum(g * v) - fd) / abs(fd) < 1e-7
