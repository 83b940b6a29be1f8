"""GPU parity of the USFFT Radon pair (C-ABI through the drop-in classes)
against the golden fixtures from the reference's own kernels and against the
FP64 oracle.  Gates: relative L2 <= 1e-5 (FP32 arithmetic), adjoint
identity <= 1e-6, bitwise determinism."""
import os

import numpy as np
import pytest
import torch

from oracle.usfft import TomoRealOracle, TomoLargeRealOracle

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL = 1e-5      # relative L2, FP32 CUDA path vs reference / FP64 oracle


def rl2(a, b):
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) else np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def load(name):
    return np.load(os.path.join(GOLD, name))


@pytest.fixture(scope="module")
def TomoReal():
    from model_mosaic_b200.processing.tomo import TomoReal
    return TomoReal


def test_R_matches_reference_kernels(TomoReal):
    g = load("tomo_R_n64_nz16_t24.npz")
    tomo = TomoReal(64, 16, g["theta"])
    sino = tomo.R(torch.from_numpy(g["obj"]).cuda()).cpu().numpy()
    assert sino.shape == (24, 16, 64) and sino.dtype == np.float32
    assert rl2(sino, g["sino"]) < RTOL
    assert rl2(sino, TomoRealOracle(64, 16, g["theta"]).R(g["obj"])) < RTOL


def test_R_numpy_roundtrip_and_partial_chunk(TomoReal):
    g = load("tomo_R_n64_nz16_t24.npz")
    tomo = TomoReal(64, 16, g["theta"])
    full = tomo.R(g["obj"])                       # numpy in -> numpy out
    assert isinstance(full, np.ndarray)
    part = tomo.R(g["obj"][:5])                   # nz < ctor nz (tomo.py:124,150)
    assert part.shape == (24, 5, 64)
    assert rl2(part, g["sino"][:, :5]) < RTOL
    again = tomo.R(g["obj"])
    assert np.array_equal(again, full)            # deterministic and no stale state


def test_RT_real_and_complex_match_reference(TomoReal):
    g = load("tomo_RT_n64_nz8_t24.npz")
    tomo = TomoReal(64, 8, g["theta"])
    rr = tomo.RT(torch.from_numpy(g["sino_r"]).cuda())
    assert rr.dtype == torch.float32 and tuple(rr.shape) == (8, 64, 64)
    assert rl2(rr.cpu().numpy(), g["obj_r"]) < RTOL
    rc = tomo.RT(torch.from_numpy(g["sino_c"]).cuda())
    assert rc.dtype == torch.complex64
    assert rl2(rc.cpu().numpy(), g["obj_c"]) < RTOL
    o = TomoRealOracle(64, 8, g["theta"])
    assert rl2(rc.cpu().numpy(), o.RT(g["sino_c"])) < RTOL


def test_RT_partial_chunk_and_determinism(TomoReal):
    g = load("tomo_RT_n64_nz8_t24.npz")
    tomo = TomoReal(64, 8, g["theta"])
    a = tomo.RT(g["sino_r"][:, :3])
    assert a.shape == (3, 64, 64)
    assert rl2(a, g["obj_r"][:3]) < RTOL
    y = torch.from_numpy(g["sino_r"]).cuda()
    b1 = tomo.RT(y)
    b2 = tomo.RT(y)
    assert torch.equal(b1, b2)                    # no float atomics: bitwise repeatable


def test_n48_half_range(TomoReal):
    g = load("tomo_n48_nz3_t30.npz")
    tomo = TomoReal(48, 3, g["theta"])
    assert rl2(tomo.R(g["obj"]), g["sino"]) < RTOL
    assert rl2(tomo.RT(g["y"]), g["RTy"]) < RTOL


def test_adjoint_identity(TomoReal):
    g = load("tomo_adjoint_n64_nz8_t24.npz")
    tomo = TomoReal(64, 8, g["theta"])
    Rx = tomo.R(g["x"]).astype(np.float64)
    RTy = tomo.RT(g["y"]).astype(np.float64)
    lhs, rhs = np.sum(Rx * g["y"]), np.sum(g["x"] * RTy)
    assert abs(lhs - rhs) / max(abs(lhs), abs(rhs)) < 1e-6


def test_large_variant(TomoReal):
    from model_mosaic_b200.processing.tomo_large import TomoLargeReal
    g = load("tomo_R_n64_nz16_t24.npz")
    tl = TomoLargeReal(64, g["theta"], 64)
    s = tl.R(g["obj"], [64, 24, 64]).copy()
    assert rl2(s, g["sino_large"]) < RTOL
    assert rl2(s, TomoLargeRealOracle(64, 16, g["theta"]).R(g["obj"])) < RTOL
    for chunks in [(32, 12, 32), (16, 6, 16), (8, 6, 8)]:
        assert np.abs(tl.R(g["obj"], list(chunks)) - s).max() / np.abs(s).max() < 1e-4
    gr = load("tomo_RT_n64_nz8_t24.npz")
    tl = TomoLargeReal(64, gr["theta"], 128)
    assert rl2(tl.RT(gr["sino_r"], [64, 24, 128]), gr["obj_r"]) < RTOL
    assert rl2(tl.RT(gr["sino_c"], [32, 12, 32]), gr["obj_c"]) < RTOL
    with pytest.raises(AssertionError):
        tl.R(g["obj"], [5, 24, 64])


def ellipsoids(n, nz, seed=0, count=10):
    from model_mosaic_b200.phantom import ellipsoid_volume
    return ellipsoid_volume(n, nz, seed=seed, count=count)


@pytest.mark.parametrize("nz", [1, 2, 12, 64, 128])
def test_sizes_vs_fp64_oracle(TomoReal, nz):
    # config-1 geometry (n = 128, 180 angles on [0, pi)) at several slice counts,
    # covering every lane layout of the gather and scatter kernels
    n, T = 128, 180
    theta = np.linspace(0, np.pi, T, endpoint=False).astype(np.float32)
    x = ellipsoids(n, nz, seed=nz)
    tomo = TomoReal(n, nz, theta)
    nzo = min(nz, 4)
    o = TomoRealOracle(n, nzo, theta)
    sino = tomo.R(x)
    assert rl2(sino[:, :nzo], o.R(x[:nzo])) < RTOL
    y = np.random.default_rng(nz).standard_normal((T, nz, n)).astype(np.float32)
    rec = tomo.RT(y)
    assert rl2(rec[:nzo], o.RT(y[:, :nzo])) < RTOL


def test_errors_leave_handle_usable(TomoReal):
    theta = np.linspace(0, np.pi, 16, endpoint=False).astype(np.float32)
    tomo = TomoReal(32, 4, theta)
    with pytest.raises(ValueError):
        tomo.R(np.zeros((5, 32, 32), np.float32))        # nz above the ctor's
    with pytest.raises(ValueError):
        tomo.R(np.zeros((2, 32, 31), np.float32))
    with pytest.raises(ValueError):
        tomo.RT(np.zeros((15, 4, 32), np.float32))
    with pytest.raises(ValueError):
        TomoReal(33, 1, theta)
    x = np.random.default_rng(0).standard_normal((4, 32, 32)).astype(np.float32)
    assert rl2(tomo.R(x), TomoRealOracle(32, 4, theta).R(x)) < RTOL


def test_production_size_n2048(TomoReal):
    # n = 2048 with 64 slices exercises the 4096-point column transforms and the
    # two-slices-per-lane gather/scatter of the production workload.
    n, nz, T = 2048, 64, 8
    theta = np.linspace(0, 2 * np.pi, T, endpoint=False).astype(np.float32)
    tomo = TomoReal(n, nz, theta)
    pick = [0, 31, 63]
    o64 = TomoRealOracle(n, len(pick), theta)
    # (1) the benchmark's input class (seeded ellipsoids): 1e-5 against FP64
    from model_mosaic_b200.phantom import ellipsoid_volume_torch
    xd = ellipsoid_volume_torch(n, nz, seed=7)
    x = xd.cpu().numpy()
    sino = tomo.R(xd).cpu().numpy()
    assert rl2(sino[:, pick], o64.R(x[pick])) < RTOL
    # (2) white noise: at this size float32 arithmetic of the reference's own
    # algorithm is ~2.7e-5 away from FP64 (mostly the 4096^2 FFTs), so the
    # gate is "no worse than 1.5x the reference algorithm run in float32"
    o32 = TomoRealOracle(n, len(pick), theta, dtype=np.float32)
    rng = np.random.default_rng(2048)
    xn = rng.standard_normal((nz, n, n), dtype=np.float32)
    ref = o64.R(xn[pick])
    floor = rl2(o32.R(xn[pick]), ref)
    assert rl2(tomo.R(torch.from_numpy(xn).cuda()).cpu().numpy()[:, pick], ref) < 1.5 * floor
    y = rng.standard_normal((T, nz, n), dtype=np.float32)
    ref = o64.RT(y[:, pick])
    floor = rl2(o32.RT(y[:, pick]), ref)
    assert rl2(tomo.RT(torch.from_numpy(y).cuda()).cpu().numpy()[pick], ref) < 1.5 * floor


@pytest.mark.parametrize("n,nz", [(128, 64), (128, 16), (48, 8)])
def test_paired_gather_360(TomoReal, n, nz):
    # [0, 2 pi) with T even: angle t + T/2 = angle t + pi, so the gather takes
    # the two in one lane group, sharing taps where their windows coincide.
    # The same angles interleaved (no pairing) must give the same bits.
    T = 90
    theta = np.linspace(0, 2 * np.pi, T, endpoint=False).astype(np.float32)
    perm = np.stack([np.arange(T // 2), np.arange(T // 2) + T // 2], axis=1).ravel()
    rng = np.random.default_rng(n + nz)
    x = rng.standard_normal((nz, n, n)).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    paired = TomoReal(n, nz, theta).R(xd)
    single = TomoReal(n, nz, theta[perm]).R(xd)
    assert torch.equal(paired[perm], single)
    assert rl2(paired.cpu().numpy(), TomoRealOracle(n, nz, theta).R(x)) < RTOL
