"""GPU parity of the 3 * 2^k line lengths (Stockham passes of radix 8 with a
last pass of radix 3, 6 or 12).  These are the reference pipeline's own sizes:
n = 3072 * ups in step2_radon.py / step3_propagation.py / step8_fbp.py, and the
768 / 1536 mosaic tiles.  Each case runs the native kernels (checked through
the stage timers or the workspace size) against the FP64 oracle at relative
L2 <= 1e-5, plus the adjoint identities."""
import numpy as np
import pytest
import torch

from oracle.fbp import calc_filter, filter_rows
from oracle.fresnel import PropagationOracle
from oracle.paganin import paganin_filter, retrieve
from oracle.usfft import TomoRealOracle

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def rl2(a, b):
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) else np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("n,nz", [(48, 3), (96, 3), (192, 2), (384, 3), (768, 2)])
def test_radon_pair_vs_fp64(n, nz):
    # step8_fbp.py geometry: 3n/4 angles on [0, pi)
    from model_mosaic_b200.phantom import ellipsoid_volume
    from model_mosaic_b200.processing.tomo import TomoReal
    T = 3 * n // 4
    theta = np.linspace(0, np.pi, T, endpoint=False).astype(np.float32)
    x = ellipsoid_volume(n, nz, seed=n, count=10)
    tomo = TomoReal(n, nz, theta)
    tomo.set_timing(True)
    sino = tomo.R(x)
    o = TomoRealOracle(n, nz, theta)
    assert rl2(sino, o.R(x)) < RTOL
    # RT of a second phantom's sinogram, gated at RTOL
    yp = o.R(ellipsoid_volume(n, nz, seed=n + 1, count=10)).astype(np.float32)
    assert rl2(tomo.RT(yp), o.RT(yp)) < RTOL
    # RT of white noise: float32 sums over many angles cancel, so the float32
    # algorithm has an error floor of its own (the float32 oracle's error,
    # e.g. 2.1e-5 at n = 768, 576 angles); gate at max(RTOL, 1.5 x floor)
    y = np.random.default_rng(n).standard_normal((T, nz, n)).astype(np.float32)
    rec = tomo.RT(y)
    r64 = o.RT(y)
    floor = rl2(TomoRealOracle(n, nz, theta, dtype=np.float32).RT(y), r64)
    err = rl2(rec, r64)
    print(f"n={n} {T} angles: RT of noise rel-L2 {err:.2e}, float32 oracle {floor:.2e}")
    assert err < max(RTOL, 1.5 * floor)
    stages, kernels = tomo.timing()
    # the fused x side ran (pad_phi), not the cuFFT rows (x_r2c)
    assert stages.get("pad_phi", (0, 0))[1] > 0 and stages.get("x_r2c", (0, 0))[1] == 0
    assert stages.get("crop_phi", (0, 0))[1] > 0 and stages.get("x_c2r", (0, 0))[1] == 0
    # adjoint identity <R x, y> = <x, RT y> on the phantom
    lhs = np.vdot(sino.astype(np.float64), y.astype(np.float64))
    rhs = np.vdot(x.astype(np.float64), rec.astype(np.float64))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


@pytest.mark.parametrize("n,nz,nt", [(192, 96, 3), (96, 384, 2), (768, 64, 2), (3072, 96, 1),
                                      (1536, 1536, 1), (96, 3072, 1)])
def test_fresnel_vs_fp64(n, nz, nt):
    from model_mosaic_b200.processing.propagation import Propagation
    wl, vs, dist = 4.133e-11, 0.69e-6, [0.12, 0.02]
    rng = np.random.default_rng(n + nz)
    a = (rng.standard_normal((nt, nz, n)) + 1j * rng.standard_normal((nt, nz, n))).astype(np.complex64)
    b = (rng.standard_normal((nt, nz, n)) + 1j * rng.standard_normal((nt, nz, n))).astype(np.complex64)
    prop = Propagation(n, nz, nt, 2, wl, vs, dist)
    ora = PropagationOracle(n, nz, nt, 2, wl, vs, dist)
    prop.set_timing(True)
    for j in range(2):
        Da = prop.D(a, j)
        assert rl2(Da, ora.D(a, j)) < RTOL
        DTb = prop.DT(b, j)
        assert rl2(DTb, ora.DT(b, j)) < RTOL
        lhs = np.vdot(b.astype(np.complex128), Da.astype(np.complex128))
        rhs = np.vdot(DTb.astype(np.complex128), a.astype(np.complex128))
        assert abs(lhs - rhs) / abs(lhs) < 1e-6
    stages, kernels = prop.timing()
    # native: one column-pass and one row-pass kernel per call (the cuFFT
    # path launches three of its own kernels per call)
    assert kernels == 4 * 2


@pytest.mark.parametrize("n,rows,name", [(24, 5, "ramp"), (48, 3, "shepp"), (192, 7, "parzen"),
                                         (768, 4, "hann"), (1536, 3, "cosine"), (3072, 5, "shepp")])
def test_fbp_filter_vs_fp64(n, rows, name):
    from model_mosaic_b200 import _ffi
    from model_mosaic_b200.processing.fbp_filter import FBPFilter
    rng = np.random.default_rng(n)
    s = rng.standard_normal((rows, n)).astype(np.float32)
    f = FBPFilter(n, batch_chunk=4)
    # native kernel: the handle holds only its two twiddle tables (2 x 2 * 4n float2)
    assert _ffi.lib().mm_fbp_workspace_bytes(f._h) == 4 * (4 * n) * 8
    d = torch.from_numpy(s).cuda()
    f.filter(d, f.calc_filter(name))
    assert rl2(d.cpu().numpy(), filter_rows(s, calc_filter(n, name))) < RTOL


@pytest.mark.parametrize("n,nz,nt", [(96, 192, 3), (384, 96, 2), (3072, 96, 1), (768, 1536, 1)])
def test_paganin_vs_fp64(n, nz, nt):
    from model_mosaic_b200.processing.paganin import Paganin
    wl, vox, alpha = 4.13e-11, 1.4e-6, 1e-3
    rng = np.random.default_rng(n + nz)
    x = (0.5 + 0.5 * rng.random((nt, nz, n))).astype(np.float32)
    p = Paganin(n, nz, nt, wl, vox, 0.1, alpha)
    ref = retrieve(x, paganin_filter(n, nz, wl, vox, 0.1, alpha))
    assert rl2(p.retrieve(x), ref) < RTOL


@pytest.mark.parametrize("n,nz", [(96, 3), (384, 1)])
def test_paired_360_and_complex_rt(n, nz):
    # 360-degree scans take the paired (theta, theta + pi) gather; complex RT input
    from model_mosaic_b200.phantom import ellipsoid_volume
    from model_mosaic_b200.processing.tomo import TomoReal
    T = 3 * n // 2
    theta = np.linspace(0, 2 * np.pi, T, endpoint=False).astype(np.float32)
    x = ellipsoid_volume(n, nz, seed=n + 7, count=10)
    tomo = TomoReal(n, nz, theta)
    o = TomoRealOracle(n, nz, theta)
    assert rl2(tomo.R(x), o.R(x)) < RTOL
    rng = np.random.default_rng(n)
    yp = o.R(ellipsoid_volume(n, nz, seed=n + 8, count=10))
    yc = (yp + 1j * o.R(ellipsoid_volume(n, nz, seed=n + 9, count=10))).astype(np.complex64)
    rec = tomo.RT(yc)
    assert rec.dtype == np.complex64
    assert rl2(rec, o.RT(yc)) < RTOL


def test_large_classes_at_3x2k():
    from model_mosaic_b200.phantom import ellipsoid_volume
    from model_mosaic_b200.processing.propagation import Propagation
    from model_mosaic_b200.processing.propagation_large import PropagationLarge
    from model_mosaic_b200.processing.tomo import TomoReal
    from model_mosaic_b200.processing.tomo_large import TomoLargeReal
    n, nz, T = 192, 5, 144
    theta = np.linspace(0, np.pi, T, endpoint=False).astype(np.float32)
    x = ellipsoid_volume(n, nz, seed=3, count=10)
    tl = TomoLargeReal(n, theta, 64)
    s = tl.R(x, [64, 48, 64]).copy()
    tr = TomoReal(n, nz, theta, clamp_xy=True)
    assert rl2(s, tr.R(x)) < 1e-6                      # the Large class runs the same kernels
    assert rl2(s, TomoRealOracle(n, nz, theta).R(x, clamp=True)) < RTOL
    assert rl2(tl.RT(s, [64, 48, 64]), tr.RT(s)) < 1e-6
    wl, vs = 4.133e-11, 0.69e-6
    psi = (np.random.default_rng(1).standard_normal((3, 96, 384))
           + 1j * np.random.default_rng(2).standard_normal((3, 96, 384))).astype(np.complex64)
    pl = PropagationLarge(384, 96, wl, vs, [0.12])
    pg = Propagation(384, 96, 3, 1, wl, vs, [0.12])
    ref = PropagationOracle(384, 96, 3, 1, wl, vs, [0.12]).D(psi, 0)
    assert rl2(pl.D(psi, 0, [48, 192]), ref) < RTOL
    assert rl2(pg.D(psi, 0), ref) < RTOL


@pytest.mark.parametrize("n,nz,nt", [(384, 96, 3), (192, 3072, 1)])
def test_intensity_fused_stage_3x2k(n, nz, nt):
    from oracle.fresnel import abs2, psi_from_proj
    from model_mosaic_b200.processing.propagation import Propagation
    wl, vs = 4.133e-11, 0.69e-6
    p = np.random.default_rng(5).uniform(0, 3, (nt, nz, n)).astype(np.float32)
    prop = Propagation(n, nz, nt, 1, wl, vs, [0.12])
    got = prop.intensity(torch.from_numpy(p).cuda(), 0.7, 0.01, 0).cpu().numpy()
    ref = abs2(PropagationOracle(n, nz, nt, 1, wl, vs, [0.12]).D(psi_from_proj(p, 0.7, 0.01), 0))
    assert rl2(got, ref) < RTOL
