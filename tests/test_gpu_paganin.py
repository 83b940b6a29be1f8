"""GPU Paganin retrieval (three fused passes for 2^k and 3 * 2^k sizes, cuFFT
otherwise) against the reference's own Paganin outputs
(tests/golden/make_golden_paganin.py) and the FP64 oracle: relative L2 <= 1e-5;
2-D input, batches smaller than ntheta, PaganinLarge's chunk validation
(tests/test_large_variants.py:227-290)."""
import os

import numpy as np
import pytest
import torch

from oracle.paganin import paganin_filter, retrieve

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "paganin.npz"))
WL, VOX, ALPHA = 4.13e-11, 1.4e-6, 1e-3
RTOL = 1e-5


def rl2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.mark.parametrize("L", [0.02, 0.1, 1.0])
def test_matches_reference(L):
    from model_mosaic_b200.processing.paganin import Paganin
    p = Paganin(64, 32, 3, WL, VOX, L, ALPHA)
    assert np.array_equal(p.filt, GOLD[f"filt_L{L}"])
    got = p.retrieve(torch.from_numpy(GOLD["intensity"]).cuda())
    assert got.shape == (3, 32, 64) and got.dtype == torch.float32
    assert rl2(got.cpu().numpy(), GOLD[f"phase_L{L}"]) < RTOL


def test_2d_and_partial_batch():
    from model_mosaic_b200.processing.paganin import Paganin
    p = Paganin(64, 32, 3, WL, VOX, 0.1, ALPHA)
    one = p.retrieve(GOLD["intensity"][1])                     # numpy in -> numpy out, (nz, n)
    assert isinstance(one, np.ndarray) and one.shape == (32, 64)
    assert rl2(one, GOLD["phase2d_L0.1"]) < RTOL
    two = p.retrieve(GOLD["intensity"][:2])
    assert rl2(two, GOLD["phase_b2_L0.1"]) < RTOL
    with pytest.raises(AssertionError):
        p.retrieve(np.zeros((4, 32, 64), np.float32))


@pytest.mark.parametrize("n,nz,nt", [(2, 2, 3), (256, 64, 3), (4096, 8, 2), (96, 40, 3), (48, 16, 2)])
def test_sizes_vs_fp64(n, nz, nt):
    from model_mosaic_b200.processing.paganin import Paganin
    rng = np.random.default_rng(n + nz)
    x = (0.5 + 0.5 * rng.random((nt, nz, n))).astype(np.float32)
    p = Paganin(n, nz, nt, WL, VOX, 0.1, ALPHA)
    ref = retrieve(x, paganin_filter(n, nz, WL, VOX, 0.1, ALPHA))
    assert rl2(p.retrieve(x), ref) < RTOL


def test_large_variant_and_validation():
    from model_mosaic_b200.processing.paganin_large import PaganinLarge
    pl = PaganinLarge(64, 32, WL, VOX, 0.1, ALPHA)
    for chunks in [(32, 64), (16, 32), (8, 16), (4, 8)]:
        got = pl.retrieve(GOLD["intensity"], list(chunks))
        assert rl2(got, GOLD["phase_L0.1"]) < RTOL
    with pytest.raises(AssertionError, match="CHUNK_NZ"):
        pl.retrieve(GOLD["intensity"], [5, 16])
    with pytest.raises(AssertionError, match="CHUNK_N"):
        pl.retrieve(GOLD["intensity"], [8, 9])
