"""GPU parity at the benchmark's full geometry and at the reference scripts'
own sizes, through the drop-in classes (C-ABI).

* The production workload: 64 slices of 2048^2, 2058 angles on [0, 2 pi)
  (the angles pair as theta, theta + pi, so R takes the paired gather), the
  seeded ellipsoid volume.  R and RT are compared slice by slice with the FP64
  oracle and R once with the reference's own gather kernel (host build, float32);
  the adjoint identity <R x, y> = <x, RT y> is checked on the whole slab.
* step2_radon / step8_fbp defaults (processing runs at n = 3072 * ups with
  3n/4 angles on [0, pi)): n = 3072 with 2304 angles, the size that runs the
  cuFFT transforms around the gather and the scatter.  n = 6144 (ups = 2,
  4608 angles) is checked by the adjoint identity only: its FP64 oracle takes
  minutes per slice.
* The differentiable model at config 3's in-plane geometry (512^2, 1024
  angles) on an 8-slice slab against the FP64 oracle (D couples the slices of
  a frame, so the oracle runs the whole slab).

The oracle slices run in a spawn pool while the GPU works.  Gates: relative L2
<= 1e-5 (RTOL); adjoint identity <= 1e-6 (ADJ_TOL) with y the sinogram of a
second phantom, and <= 1e-5 (ADJ_NOISE_TOL) with y white noise, where
<R x, y> is a sum of random-sign terms whose cancellation magnifies the
operators' float32 rounding (measured 3e-7 to 4e-6).  The gradient's residual
|D psi|^2 - d cancels to nothing over the background, so float32 arithmetic
has a floor of its own there: the gate is the larger of 1e-5 and 1.5x the
error of the same composition run in float32 by the oracle."""
import numpy as np
import pytest
import torch

from oracle import jobs

pytestmark = pytest.mark.gpu
RTOL = 1e-5       # relative L2, float32 CUDA path vs FP64 oracle / reference kernels
ADJ_TOL = 1e-6    # |<Rx, y> - <x, RT y>| / max(|.|, |.|), y a phantom's sinogram
ADJ_NOISE_TOL = 1e-5  # the same with y white noise

N, NZ, T = 2048, 64, 2058
PICK = (24, 40)   # slices checked against the FP64 oracle (both cut through ellipsoids)


def rl2(a, b):
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) else np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def adjoint_gap(tomo, x, y):
    lhs = float((tomo.R(x).double() * y.double()).sum())
    rhs = float((x.double() * tomo.RT(y).double()).sum())
    return abs(lhs - rhs) / max(abs(lhs), abs(rhs))


def adjoint_gaps(tomo, x, seed):
    """(gap with y = R of a second phantom, gap with y = white noise)."""
    from model_mosaic_b200.phantom import ellipsoid_volume_torch
    nz, n = x.shape[0], x.shape[1]
    y1 = tomo.R(ellipsoid_volume_torch(n, nz, seed=seed + 100))
    gen = torch.Generator(device="cuda").manual_seed(seed)
    y2 = torch.randn(tuple(y1.shape), generator=gen, device="cuda")
    return adjoint_gap(tomo, x, y1), adjoint_gap(tomo, x, y2)


@pytest.fixture(scope="module")
def pool():
    p = jobs.pool(4)
    yield p
    p.terminate()
    p.join()


@pytest.fixture(scope="module")
def production(pool):
    from model_mosaic_b200.processing.tomo import TomoReal
    from model_mosaic_b200.phantom import ellipsoid_volume_torch
    theta = np.linspace(0, 2 * np.pi, T, endpoint=False).astype(np.float32)
    xd = ellipsoid_volume_torch(N, NZ, seed=0)
    x = xd.cpu().numpy()
    pend = {"R": [pool.apply_async(jobs.tomo_R, (N, theta, x[z:z + 1])) for z in PICK],
            "refR": pool.apply_async(jobs.ref_tomo_R, (N, theta, x[PICK[0]:PICK[0] + 1]))}
    tomo = TomoReal(N, NZ, theta)
    sino = tomo.R(xd)
    s = sino.cpu().numpy()
    pend["RT"] = [pool.apply_async(jobs.tomo_RT, (N, theta, np.ascontiguousarray(s[:, z:z + 1]))) for z in PICK]
    rec = tomo.RT(sino).cpu().numpy()
    gap = adjoint_gaps(tomo, xd, 5)
    tomo.free()
    ck = TomoReal(N, NZ, theta, compensated=True)
    rec_k = ck.RT(sino).cpu().numpy()
    ck.free()
    return dict(sino=s, rec=rec, rec_k=rec_k, gap=gap, pend=pend)


def test_production_R_vs_fp64_oracle(production):
    for z, job in zip(PICK, production["pend"]["R"]):
        ref = job.get()[:, 0]
        err = rl2(production["sino"][:, z], ref)
        print(f"R n=2048 2058 angles slice {z}: rel-L2 vs FP64 {err:.2e}")
        assert err < RTOL


def test_production_R_vs_reference_kernels(production):
    ref = production["pend"]["refR"].get()[:, 0]
    err = rl2(production["sino"][:, PICK[0]], ref)
    print(f"R n=2048 2058 angles slice {PICK[0]}: rel-L2 vs the reference's gather kernel {err:.2e}")
    assert err < RTOL


def test_production_RT_vs_fp64_oracle(production):
    # RT sums grow with the angle count: the float32 scatter's error is stated
    # beside the gate, with the Kahan-compensated scatter's for comparison
    for z, job in zip(PICK, production["pend"]["RT"]):
        ref = job.get()[0]
        e32, ek = rl2(production["rec"][z], ref), rl2(production["rec_k"][z], ref)
        print(f"RT n=2048 2058 angles slice {z}: rel-L2 vs FP64 float32 {e32:.2e}, Kahan {ek:.2e}")
        assert e32 < RTOL
        assert ek < RTOL


def test_production_adjoint_identity(production):
    g1, g2 = production["gap"]
    print(f"adjoint identity n=2048 2058 angles 64 slices: phantom {g1:.2e}, white noise {g2:.2e}")
    assert g1 < ADJ_TOL and g2 < ADJ_NOISE_TOL


def test_step8_size_n3072_cufft_path(pool):
    # step8_fbp default (ups = 1): n = 3072, 3n/4 = 2304 angles on [0, pi)
    from model_mosaic_b200.processing.tomo import TomoReal
    from model_mosaic_b200.phantom import ellipsoid_volume_torch
    n, nz, Tn = 3072, 2, 2304
    theta = np.linspace(0, np.pi, Tn, endpoint=False).astype(np.float32)
    xd = ellipsoid_volume_torch(n, nz, seed=3)
    x = xd.cpu().numpy()
    jr = pool.apply_async(jobs.tomo_R, (n, theta, x[1:2]))
    tomo = TomoReal(n, nz, theta)
    sino = tomo.R(xd)
    s = sino.cpu().numpy()
    jt = pool.apply_async(jobs.tomo_RT, (n, theta, np.ascontiguousarray(s[:, 1:2])))
    rec = tomo.RT(sino).cpu().numpy()
    g1, g2 = adjoint_gaps(tomo, xd, 6)
    tomo.free()
    er, et = rl2(s[:, 1], jr.get()[:, 0]), rl2(rec[1], jt.get()[0])
    print(f"n=3072 2304 angles: R rel-L2 {er:.2e}, RT rel-L2 {et:.2e}, adjoint phantom {g1:.2e} "
          f"white noise {g2:.2e}")
    assert er < RTOL and et < RTOL and g1 < ADJ_TOL and g2 < ADJ_NOISE_TOL


def test_step2_size_n6144_adjoint():
    # step2_radon default (ups = 2): n = 6144, 4608 angles on [0, pi), one slice
    from model_mosaic_b200.processing.tomo import TomoReal
    n, Tn = 6144, 4608
    theta = np.linspace(0, np.pi, Tn, endpoint=False).astype(np.float32)
    from model_mosaic_b200.phantom import ellipsoid_volume_torch
    tomo = TomoReal(n, 1, theta)
    g1, g2 = adjoint_gaps(tomo, ellipsoid_volume_torch(n, 1, seed=7), 7)
    tomo.free()
    print(f"adjoint identity n=6144 4608 angles: phantom {g1:.2e}, white noise {g2:.2e}")
    assert g1 < ADJ_TOL and g2 < ADJ_NOISE_TOL


def test_model_gradient_c3_geometry(pool):
    # config 3's in-plane geometry: 512^2 slices, 1024 angles on [0, pi),
    # psi recomputed per 128-angle chunk; an 8-slice slab
    from model_mosaic_b200.model import ForwardModel
    from model_mosaic_b200.phantom import ellipsoid_volume
    from oracle.usfft import TomoRealOracle
    n, nz, Tn = 512, 8, 1024
    wl, vox, dist = 4.133e-11, 0.69e-6, 0.12
    theta = np.linspace(0, np.pi, Tn, endpoint=False).astype(np.float32)
    delta = ellipsoid_volume(n, nz, seed=0, vmin=0.2, vmax=1.0)
    delta2 = ellipsoid_volume(n, nz, seed=1, vmin=0.2, vmax=1.0)
    pmax = np.abs(TomoRealOracle(n, 1, theta).R(delta[nz // 2:nz // 2 + 1])).max()
    s = float(np.float32(1.5 / pmax))                     # phases up to ~1.5 rad
    d = pool.apply(jobs.model_forward, (n, theta, wl, vox, dist, s, delta2))
    job = pool.apply_async(jobs.model_grad, (n, theta, wl, vox, dist, s, delta, d))
    job32 = pool.apply_async(jobs.model_grad, (n, theta, wl, vox, dist, s, delta, d.astype(np.float32), np.float32))
    m = ForwardModel(n, nz, theta, wl, vox, dist, inv_norm=s, angle_chunk=128)
    loss, g = m.loss_and_grad(torch.from_numpy(delta).cuda(), torch.from_numpy(d.astype(np.float32)).cuda())
    lref, gref = job.get()
    floor = rl2(job32.get()[1], gref)
    el, eg = abs(float(loss) - lref) / lref, rl2(g.cpu().numpy(), gref)
    print(f"model 512^2 x 8 slices, 1024 angles: loss rel {el:.2e}, gradient rel-L2 {eg:.2e} "
          f"(float32 composition {floor:.2e})")
    assert el < RTOL and eg < max(RTOL, 1.5 * floor)
