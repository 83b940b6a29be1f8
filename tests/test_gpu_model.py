"""GPU differentiable forward model data = |D(exp(i(R delta + i R beta)))|^2:
loss and hand-written gradient against the FP64 oracle composed from the
restated reference operators, FP64 central differences, the unfused
composition of the same operators, angle chunking and the autograd wrapper.
Sizes follow the gradcheck case: 64^3 volume, 90 angles."""
import numpy as np
import pytest
import torch

from oracle.model import ModelOracle

pytestmark = pytest.mark.gpu
WL, VOX, DIST = 4.133e-11, 0.69e-6, 0.12


def rl2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def case():
    from model_mosaic_b200.phantom import ellipsoid_volume
    n = nz = 64
    T = 90
    theta = np.linspace(0, np.pi, T, endpoint=False).astype(np.float32)
    delta = ellipsoid_volume(n, nz, seed=0, vmin=0.2, vmax=1.0)
    delta2 = ellipsoid_volume(n, nz, seed=1, vmin=0.2, vmax=1.0)
    probe = ModelOracle(n, nz, theta, WL, VOX, DIST, s=1.0)
    s = 1.5 / np.abs(probe.tomo.R(delta)).max()          # phases up to ~1.5 rad
    ora = ModelOracle(n, nz, theta, WL, VOX, DIST, s=s)
    d = ora.forward(delta2)
    return dict(n=n, nz=nz, theta=theta, delta=delta, d=d, s=float(np.float32(s)), ora=ora)


def _model(case, chunk=None):
    from model_mosaic_b200.model import ForwardModel
    return ForwardModel(case["n"], case["nz"], case["theta"], WL, VOX, DIST, inv_norm=case["s"],
                        angle_chunk=chunk)


def test_forward_and_loss_match_oracle(case):
    m = _model(case)
    dl = torch.from_numpy(case["delta"]).cuda()
    data = m.forward(dl).cpu().numpy()
    assert rl2(data, case["ora"].forward(case["delta"])) < 1e-5
    loss, _ = m.loss_and_grad(dl, torch.from_numpy(case["d"].astype(np.float32)).cuda())
    ref = case["ora"].loss(case["delta"], case["d"])
    assert abs(float(loss) - ref) / ref < 1e-5


def test_gradient_vs_oracle_and_central_differences(case):
    m = _model(case)
    dl = torch.from_numpy(case["delta"]).cuda()
    d32 = torch.from_numpy(case["d"].astype(np.float32)).cuda()
    _, g = m.loss_and_grad(dl, d32)
    g = g.cpu().numpy()
    gref = case["ora"].grad(case["delta"], case["d"])
    assert rl2(g, gref) < 1e-5
    rng = np.random.default_rng(3)
    ora = case["ora"]
    for _ in range(2):                                    # FP64 central differences
        v = rng.standard_normal(case["delta"].shape)
        h = 1e-5
        fd = (ora.loss(case["delta"] + h * v, case["d"]) - ora.loss(case["delta"] - h * v, case["d"])) / (2 * h)
        assert abs(np.sum(g.astype(np.float64) * v) - fd) / abs(fd) < 1e-5


def test_fused_equals_plain_and_chunking(case):
    dl = torch.from_numpy(case["delta"]).cuda()
    d32 = torch.from_numpy(case["d"].astype(np.float32)).cuda()
    m = _model(case)
    l1, g1 = m.loss_and_grad(dl, d32)
    l2, g2 = m.plain_loss_and_grad(dl, d32)
    assert abs(float(l1) - float(l2)) / float(l2) < 1e-6
    assert rl2(g1.cpu().numpy(), g2.cpu().numpy()) < 1e-6
    mc = _model(case, chunk=32)                           # psi recomputed per 32-angle chunk
    l3, g3 = mc.loss_and_grad(dl, d32)
    assert abs(float(l3) - float(l1)) / float(l1) < 1e-6
    assert rl2(g3.cpu().numpy(), g1.cpu().numpy()) < 1e-6


def test_autograd_function(case):
    from model_mosaic_b200.model import FresnelRadonLoss
    m = _model(case)
    dl = torch.from_numpy(case["delta"]).cuda().requires_grad_(True)
    d32 = torch.from_numpy(case["d"].astype(np.float32)).cuda()
    loss = FresnelRadonLoss.apply(dl, d32, m)
    (2.0 * loss).backward()
    _, g = m.loss_and_grad(dl.detach(), d32)
    assert torch.allclose(dl.grad, 2.0 * g, rtol=1e-6, atol=0)


@pytest.mark.parametrize("n,nz,T", [(48, 24, 30), (96, 96, 36), (192, 48, 40)])
def test_general_sizes_gradient(n, nz, T):
    # n = 48, nz = 24: the Radon pair on the native 3 * 2^k kernels (2n = 96)
    # and D on the general (cuFFT) path; 96^3: every stage on the native
    # 3 * 2^k kernels (the row pass's per-block loss partials included);
    # 192 x 48: 3 * 2^k rows and columns of D.  Fused gradient against the
    # FP64 oracle
    from model_mosaic_b200.model import ForwardModel
    from model_mosaic_b200.phantom import ellipsoid_volume
    theta = np.linspace(0, np.pi, T, endpoint=False).astype(np.float32)
    delta = ellipsoid_volume(n, nz, seed=0, vmin=0.2, vmax=1.0)
    delta2 = ellipsoid_volume(n, nz, seed=1, vmin=0.2, vmax=1.0)
    s = float(np.float32(1.5 / np.abs(ModelOracle(n, nz, theta, WL, VOX, DIST, s=1.0).tomo.R(delta)).max()))
    ora = ModelOracle(n, nz, theta, WL, VOX, DIST, s=s)
    d = ora.forward(delta2)
    m = ForwardModel(n, nz, theta, WL, VOX, DIST, inv_norm=s, angle_chunk=16)
    dl = torch.from_numpy(delta).cuda()
    d32 = torch.from_numpy(d.astype(np.float32)).cuda()
    loss, g = m.loss_and_grad(dl, d32)
    assert abs(float(loss) - ora.loss(delta, d)) / ora.loss(delta, d) < 1e-5
    # the gradient ends in RT of a noise-like adjoint sinogram, whose float32
    # sums have an error floor of their own (the same composition in float32:
    # 2.3e-5 at 192 x 48, 40 angles): gate max(1e-5, 1.5 x that floor)
    g64 = ora.grad(delta, d)
    floor = rl2(ModelOracle(n, nz, theta, WL, VOX, DIST, s=s, dtype=np.float32).grad(delta, d), g64)
    assert rl2(g.cpu().numpy(), g64) < max(1e-5, 1.5 * floor)
    l2, g2 = m.plain_loss_and_grad(dl, d32)
    assert rl2(g.cpu().numpy(), g2.cpu().numpy()) < 1e-6
