"""GPU parity of the Fresnel propagator D, its adjoint DT and the fused
psi -> D -> |.|^2 stage, against the reference-kernel fixtures and the FP64
oracle (relative L2 <= 1e-5)."""
import os

import numpy as np
import pytest
import torch

from oracle.fresnel import PropagationOracle, psi_from_proj, abs2

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL = 1e-5


def rl2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.complex128) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLD, "prop_D_n64_nz32_t3.npz"))


def test_D_matches_reference(gold):
    from model_mosaic_b200.processing.propagation import Propagation
    dist = list(gold["distance"])
    prop = Propagation(64, 32, 3, 3, float(gold["wavelength"]), float(gold["voxelsize"]), dist)
    psi = torch.from_numpy(gold["psi"]).cuda()
    for j in range(3):
        out = prop.D(psi, j).cpu().numpy()
        assert rl2(out, gold["D"][j]) < RTOL
    # 2-D input gives 2-D output (propagation.py:49-51,64), numpy in -> numpy out
    one = prop.D(gold["psi"][1], 2)
    assert one.shape == (32, 64) and rl2(one, gold["D"][2][1]) < RTOL
    # fewer angles than the constructor's
    assert rl2(prop.D(gold["psi"][:2], 1), gold["D"][1][:2]) < RTOL


def test_D_large_and_validation(gold):
    from model_mosaic_b200.processing.propagation_large import PropagationLarge
    dist = list(gold["distance"])
    pl = PropagationLarge(64, 32, float(gold["wavelength"]), float(gold["voxelsize"]), dist)
    for j in range(3):
        for chunks in [(32, 128), (16, 32), (8, 16), (4, 8)]:
            got = pl.D(gold["psi"], j, list(chunks))
            assert np.abs(got - gold["D"][j]).max() / np.abs(gold["D"][j]).max() < 1e-3
        assert rl2(got, gold["D"][j]) < RTOL
    bad = PropagationLarge(32, 16, 4.13e-11, 1.4e-6, [0.0])
    z = np.zeros((1, 16, 32), np.complex64)
    for chunks in [(5, 16), (8, 9)]:                 # tests/test_large_variants.py:205-223
        with pytest.raises(AssertionError):
            bad.D(z, 0, list(chunks))


@pytest.mark.parametrize("n,nz,nt", [(64, 32, 3), (256, 64, 5), (2048, 64, 2), (128, 8, 4), (8, 2, 2),
                                      (16, 4, 3), (2, 16, 2), (512, 128, 2), (32, 2048, 1),
                                      # general sizes (cuFFT 2-D path): odd, other lengths, mixed
                                      (12, 6, 3), (5, 7, 2), (64, 48, 2),
                                      # 3 * 2^k lengths on the native kernels
                                      (96, 64, 3), (768, 16, 2)])
def test_D_DT_vs_oracle_and_adjoint(n, nz, nt):
    from model_mosaic_b200.processing.propagation import Propagation
    wl, vs, dist = 4.133e-11, 0.69e-6, [0.12, 0.02]
    rng = np.random.default_rng(n + nz)
    a = (rng.standard_normal((nt, nz, n)) + 1j * rng.standard_normal((nt, nz, n))).astype(np.complex64)
    b = (rng.standard_normal((nt, nz, n)) + 1j * rng.standard_normal((nt, nz, n))).astype(np.complex64)
    prop = Propagation(n, nz, nt, 2, wl, vs, dist)
    ora = PropagationOracle(n, nz, nt, 2, wl, vs, dist)
    for j in range(2):
        Da = prop.D(a, j)
        assert rl2(Da, ora.D(a, j)) < RTOL
        DTb = prop.DT(b, j)
        assert rl2(DTb, ora.DT(b, j)) < RTOL
        lhs = np.vdot(b.astype(np.complex128), Da.astype(np.complex128))
        rhs = np.vdot(DTb.astype(np.complex128), a.astype(np.complex128))
        # normalised by |<b, Da>| or, where that sum happens to cancel on a
        # tiny case, by its typical size for random vectors ||b|| ||Da|| / sqrt(size)
        scale = max(abs(lhs), np.linalg.norm(b) * np.linalg.norm(Da) / np.sqrt(a.size))
        assert abs(lhs - rhs) / scale < 1e-6


@pytest.mark.parametrize("n,nz,nt", [(256, 32, 3), (96, 24, 3)])
def test_intensity_fused_stage(n, nz, nt):
    from model_mosaic_b200.processing.propagation import Propagation
    wl, vs = 4.133e-11, 0.69e-6
    rng = np.random.default_rng(5)
    p = (rng.uniform(0, 3, (nt, nz, n))).astype(np.float32)
    inv_norm, inv_beta = 0.7, 0.01
    prop = Propagation(n, nz, nt, 1, wl, vs, [0.12])
    got = prop.intensity(torch.from_numpy(p).cuda(), inv_norm, inv_beta, 0).cpu().numpy()
    ora = PropagationOracle(n, nz, nt, 1, wl, vs, [0.12])
    ref = abs2(ora.D(psi_from_proj(p, inv_norm, inv_beta), 0))
    assert rl2(got, ref) < RTOL
    # same as the unfused chain through D
    psi = torch.from_numpy(psi_from_proj(p, inv_norm, inv_beta, np.float32)).cuda()
    u = prop.D(psi, 0)
    assert rl2(got, (u.real ** 2 + u.imag ** 2).cpu().numpy()) < 1e-6
