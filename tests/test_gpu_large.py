"""The host-array classes and the reference scripts' largest sizes.

* The adjoint's scatter table in blocks of angles (the form it takes when
  the whole table does not fit, e.g. n = 24576 with 18432 angles): RT with
  small blocks against RT with one table, plain and Kahan-compensated.
* TomoLargeReal and PropagationLarge stream their host arrays through the
  device in slabs / chunks on three streams: several slabs and chunks
  against one device-resident call.
* The ups = 8 size of step2_radon_large / step3_propagation_large /
  step8_fbp_large (n = nz = 3072 * 8 = 24576), on one slice with a few
  angles and on one frame (the FP64 CPU oracle would need a 49152^2 FFT per
  slice).  R is compared with the reference's own gather kernel on this GPU
  (oracle/refgpu.py); the reference's scatter (RT) and pad (D) kernels
  index with 32-bit int and overflow at this size, so RT is checked by the
  adjoint identity and D against the reference's algorithm with the same
  mirror padding done by 64-bit torch gathers, plus D's adjoint identity.
Gates: relative L2 <= 1e-5 (float32), adjoint identity <= 1e-6."""
import numpy as np
import pytest
import torch

from oracle import refgpu

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def rl2(a, b):
    a, b = torch.as_tensor(a), torch.as_tensor(b)
    return float(torch.linalg.vector_norm((a - b).to(torch.complex128 if a.is_complex() else torch.float64))
                 / torch.linalg.vector_norm(b.to(torch.complex128 if b.is_complex() else torch.float64)))


@pytest.mark.parametrize("compensated", [False, True])
def test_table_blocks_match_one_table(compensated):
    from model_mosaic_b200.processing.tomo import TomoReal
    n, nz, T = 128, 16, 180
    theta = np.linspace(0, np.pi, T, endpoint=False).astype(np.float32)
    y = torch.randn((T, nz, n), generator=torch.Generator(device="cuda").manual_seed(21), device="cuda")
    one = TomoReal(n, nz, theta, compensated=compensated).RT(y)
    blocked = TomoReal(n, nz, theta, compensated=compensated, max_table_angles=7)
    got = blocked.RT(y)
    assert torch.equal(got, blocked.RT(y))          # still deterministic
    err = rl2(got, one)
    print(f"RT with 26 table blocks vs one table: rel-L2 {err:.2e}")
    assert err < 1e-6


def test_large_classes_stream_several_slabs():
    from model_mosaic_b200.processing.tomo import TomoReal
    from model_mosaic_b200.processing.tomo_large import TomoLargeReal
    from model_mosaic_b200.phantom import ellipsoid_volume
    n, nz, T = 64, 19, 24
    theta = np.linspace(0, 2 * np.pi, T, endpoint=False).astype(np.float32)
    x = ellipsoid_volume(n, nz, seed=4)
    tl = TomoLargeReal(n, theta, 64, max_nz=4)            # slabs of 4: five slabs, the last short
    s = tl.R(x, [64, 24, 64]).copy()
    ref = TomoReal(n, nz, theta, clamp_xy=True)
    assert rl2(s, ref.R(x)) < RTOL
    y = np.random.default_rng(5).standard_normal((T, nz, n)).astype(np.float32)
    assert rl2(tl.RT(y, [64, 24, 64]), ref.RT(y)) < RTOL
    yc = (y + 1j * np.random.default_rng(6).standard_normal((T, nz, n))).astype(np.complex64)
    assert rl2(tl.RT(yc, [32, 12, 32]), ref.RT(yc)) < RTOL


def test_propagation_large_streams_several_chunks(monkeypatch):
    from model_mosaic_b200.processing import propagation_large as pl
    from model_mosaic_b200.processing.propagation import Propagation
    monkeypatch.setattr(pl, "chunk_frames", lambda n, nz, nt, free: 3)
    n, nz, T = 96, 40, 10                                      # general path, four chunks
    rng = np.random.default_rng(7)
    psi = (rng.standard_normal((T, nz, n)) + 1j * rng.standard_normal((T, nz, n))).astype(np.complex64)
    big = pl.PropagationLarge(n, nz, 4.133e-11, 0.69e-6, [0.12, 0.05])
    got = big.D(psi, 1, [nz, 2 * n]).copy()
    ref = Propagation(n, nz, T, 2, 4.133e-11, 0.69e-6, [0.12, 0.05]).D(psi, 1)
    assert rl2(got, ref) < RTOL


def test_ups8_radon_n24576_vs_reference_kernels():
    # step2_radon_large / step8_fbp_large at ups = 8: n = 24576; one slice, 16 angles.
    # TomoLargeReal is the device operator with TomoLargeReal's clamped sample
    # coordinates (processing/kernels.py:478-481) behind host arrays: it must
    # equal TomoReal(clamp_xy=True) bit for bit; the unclamped operator is
    # compared with the reference's own TomoReal kernels.
    from model_mosaic_b200.processing.tomo import TomoReal
    from model_mosaic_b200.processing.tomo_large import TomoLargeReal
    from model_mosaic_b200.phantom import ellipsoid_volume_torch
    n, T = 24576, 16
    theta = np.linspace(0, np.pi, T, endpoint=False).astype(np.float32)
    x = ellipsoid_volume_torch(n, 1, seed=8)
    y = TomoReal(n, 1, theta).R(ellipsoid_volume_torch(n, 1, seed=9))
    tl = TomoLargeReal(n, theta, 256)
    s_large = torch.from_numpy(tl.R(x.cpu().numpy(), [256, 16, 256]).copy())
    r_large = torch.from_numpy(tl.RT(y.cpu().numpy(), [256, 16, 256]).copy())
    tl.free()
    tc = TomoReal(n, 1, theta, clamp_xy=True)
    assert torch.equal(s_large, tc.R(x).cpu())
    tc.free()
    tomo = TomoReal(n, 1, theta)
    s, rec = tomo.R(x), tomo.RT(y)
    assert torch.equal(r_large, rec.cpu())
    lhs, rhs = float((s.double() * y.double()).sum()), float((x.double() * rec.double()).sum())
    gap = abs(lhs - rhs) / max(abs(lhs), abs(rhs))
    tomo.free()
    torch.cuda.empty_cache()
    ref = refgpu.RefGpuTomoReal(n, 1, theta)
    er = rl2(s, ref.R(x))
    with pytest.raises(ValueError, match="32-bit"):
        ref.RT(y)                                   # its scatter would address past 2^31 entries
    print(f"n=24576 16 angles: R rel-L2 vs the reference's gather kernel {er:.2e}, adjoint {gap:.2e}")
    assert er < RTOL and gap < 1e-6


def test_ups8_propagation_n24576_vs_reference_kernels():
    # step3_propagation_large at ups = 8: one 24576 x 24576 frame
    from model_mosaic_b200.processing.propagation_large import PropagationLarge
    from model_mosaic_b200.phantom import ellipsoid_volume_torch
    n = nz = 24576
    wl, vox, dist = 4.133e-11, 0.69e-6, 0.12
    ph = ellipsoid_volume_torch(n, 1, seed=10)[0] * 1e6            # phase up to ~1 rad
    psi = torch.polar(torch.exp(-0.01 * ph), ph)
    del ph
    g = torch.polar(torch.ones_like(psi.real), 0.3 * psi.angle().flip(0))   # a second field
    big = PropagationLarge(n, nz, wl, vox, [dist])
    got = torch.from_numpy(big.D(psi.cpu().numpy(), 0, [nz, 2 * n]).copy()).cuda()
    dtg = torch.from_numpy(big.DT(g.cpu().numpy(), 0, [nz, 2 * n]).copy()).cuda()
    big.free()
    lhs = complex(torch.vdot(got.flatten().to(torch.complex128), g.flatten().to(torch.complex128)))
    rhs = complex(torch.vdot(psi.flatten().to(torch.complex128), dtg.flatten().to(torch.complex128)))
    gap = abs(lhs - rhs) / abs(lhs)
    del dtg, g
    torch.cuda.empty_cache()
    ref = refgpu.RefGpuPropagation(n, nz, 1, 1, wl, vox, [dist]).D(psi, 0)
    err = rl2(got, ref)
    print(f"D 24576^2 frame: rel-L2 vs the reference's algorithm {err:.2e}, D/DT adjoint {gap:.2e}")
    assert err < RTOL and gap < 1e-6
