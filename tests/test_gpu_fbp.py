"""GPU FBP filter (fused Stockham kernel for 4n a power of two up to 8192 or
3 * 2^k up to 12288, cuFFT otherwise) against the reference's FBPFilter outputs and the FP64
oracle: relative L2 <= 1e-5, in place, the reference's chunking and host
variants, and the filter followed by RT as step8_fbp.py does."""
import os

import numpy as np
import pytest
import torch

from oracle.fbp import calc_filter, filter_rows

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fbp_filter.npz"))
RTOL = 1e-5


def rl2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.mark.parametrize("n,name", [(64, "ramp"), (64, "shepp"), (100, "hann")])
def test_filter_matches_reference(n, name):
    from model_mosaic_b200.processing.fbp_filter import FBPFilter
    f = FBPFilter(n, batch_chunk=5)
    w = f.calc_filter(name)
    s = torch.from_numpy(GOLD[f"sino_{name}_n{n}"]).cuda()
    out = f.filter(s, w)
    assert out is s                                            # in place, returns its argument
    assert rl2(s.cpu().numpy(), GOLD[f"filt_{name}_n{n}"]) < RTOL


@pytest.mark.parametrize("n,rows,name", [(8, 3, "none"), (256, 9, "parzen"), (2048, 7, "shepp"),
                                         (96, 11, "cosine"), (3000, 4, "hamming")])
def test_filter_sizes_vs_fp64(n, rows, name):
    from model_mosaic_b200.processing.fbp_filter import FBPFilter
    rng = np.random.default_rng(n)
    s = rng.standard_normal((rows, n)).astype(np.float32)
    f = FBPFilter(n, batch_chunk=4)
    d = torch.from_numpy(s).cuda()
    f.filter(d, f.calc_filter(name))
    ref = filter_rows(s, calc_filter(n, name))
    assert rl2(d.cpu().numpy(), ref) < RTOL
    h = s.copy()
    f.filter_host(h, f.calc_filter(name), batch_chunk=3)
    assert rl2(h, ref) < RTOL


def test_filter_errors():
    from model_mosaic_b200.processing.fbp_filter import FBPFilter
    f = FBPFilter(64)
    w = f.calc_filter("ramp")
    with pytest.raises(ValueError):
        f.filter(torch.zeros((3, 32), device="cuda"), w)
    with pytest.raises(ValueError):
        f.filter(torch.zeros((64, 3), device="cuda").t(), w)    # not contiguous
    with pytest.raises(ValueError):
        f.filter(torch.zeros((3, 64)), w)                          # host tensor: filter_host


def test_filtered_backprojection_step8():
    # step8_fbp.py:203-205: filter the sinogram, then RT
    from model_mosaic_b200.processing.fbp_filter import FBPFilter
    from model_mosaic_b200.processing.tomo import TomoReal
    from oracle.usfft import TomoRealOracle
    n, nz, T = 64, 4, 48
    theta = np.linspace(0, np.pi, T, endpoint=False).astype(np.float32)
    rng = np.random.default_rng(3)
    sino = rng.standard_normal((T, nz, n)).astype(np.float32)
    f = FBPFilter(n)
    d = torch.from_numpy(sino).cuda()
    f.filter(d, f.calc_filter("shepp"))
    rec = TomoReal(n, nz, theta).RT(d)
    ref = TomoRealOracle(n, nz, theta).RT(filter_rows(sino, calc_filter(n, "shepp")))
    assert rl2(rec.cpu().numpy(), ref) < RTOL
