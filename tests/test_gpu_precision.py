"""Precision variants of the USFFT Radon pair: bfloat16 storage of the volume
and the sinogram (float32 arithmetic) and the Kahan-compensated adjoint
scatter.  The reference stores and sums in float32 only
(processing/kernels.py:430-560), so these are checked two ways: bitwise
against the float32 path run on the same (bfloat16-representable) values and
rounded afterwards, and by their error against the FP64 oracle."""
import numpy as np
import pytest
import torch

from oracle.usfft import TomoRealOracle

pytestmark = pytest.mark.gpu
BF16_RTOL = 5e-3     # relative L2 of a bfloat16-stored result vs FP64 (8-bit mantissa)


def rl2(a, b):
    a = np.asarray(a, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def TomoReal():
    from model_mosaic_b200.processing.tomo import TomoReal
    return TomoReal


def _case(n, nz, nt, seed):
    rng = np.random.default_rng(seed)
    theta = np.linspace(0, np.pi, nt, endpoint=False).astype(np.float32)
    obj = rng.standard_normal((nz, n, n)).astype(np.float32)
    return theta, obj


@pytest.mark.parametrize("n,nz,nzc", [(64, 16, 16), (128, 64, 64), (128, 64, 37)])
def test_R_bf16_storage_bitwise(TomoReal, n, nz, nzc):
    theta, obj = _case(n, nz, 40, 11)
    tomo = TomoReal(n, nz, theta)
    xb = torch.from_numpy(obj[:nzc]).cuda().to(torch.bfloat16)
    ref32 = tomo.R(xb.float())                               # float32 path on the same values
    sb = tomo.R(xb)                                          # bf16 in, bf16 out
    assert sb.dtype == torch.bfloat16 and tuple(sb.shape) == (40, nzc, n)
    assert torch.equal(sb, ref32.to(torch.bfloat16))
    s32 = tomo.R(xb, out_dtype=torch.float32)                # bf16 in, float32 out
    assert torch.equal(s32, ref32)
    sb2 = tomo.R(xb.float(), out_dtype=torch.bfloat16)       # float32 in, bf16 out
    assert torch.equal(sb2, sb)
    o = TomoRealOracle(n, nz, theta).R(xb.float().cpu().numpy())
    assert rl2(sb.float().cpu().numpy(), o) < BF16_RTOL


@pytest.mark.parametrize("n,nz,nzc", [(64, 16, 16), (128, 64, 64), (128, 64, 21)])
def test_RT_bf16_storage_bitwise(TomoReal, n, nz, nzc):
    theta, _ = _case(n, nz, 40, 12)
    rng = np.random.default_rng(13)
    y = torch.from_numpy(rng.standard_normal((40, nzc, n)).astype(np.float32)).cuda().to(torch.bfloat16)
    tomo = TomoReal(n, nz, theta)
    ref32 = tomo.RT(y.float())
    ob = tomo.RT(y)
    assert ob.dtype == torch.bfloat16 and tuple(ob.shape) == (nzc, n, n)
    assert torch.equal(ob, ref32.to(torch.bfloat16))
    o = TomoRealOracle(n, nz, theta).RT(y.float().cpu().numpy())
    assert rl2(ob.float().cpu().numpy(), o) < BF16_RTOL


def test_bf16_needs_fused_sizes(TomoReal):
    theta, obj = _case(48, 3, 30, 14)
    tomo = TomoReal(48, 3, theta)
    with pytest.raises(ValueError, match="bfloat16"):
        tomo.R(torch.from_numpy(obj).cuda().to(torch.bfloat16))
    assert tomo.R(obj).shape == (30, 3, 48)                  # handle still usable


@pytest.mark.parametrize("n,nz,nt", [(128, 16, 180), (256, 8, 400)])
def test_RT_compensated(TomoReal, n, nz, nt):
    theta, _ = _case(n, nz, nt, 15)
    rng = np.random.default_rng(16)
    y = rng.standard_normal((nt, nz, n)).astype(np.float32)
    exact = TomoRealOracle(n, nz, theta).RT(y)
    plain = TomoReal(n, nz, theta).RT(torch.from_numpy(y).cuda())
    tk = TomoReal(n, nz, theta, compensated=True)
    comp = tk.RT(torch.from_numpy(y).cuda())
    e_plain = rl2(plain.cpu().numpy(), exact)
    e_comp = rl2(comp.cpu().numpy(), exact)
    print(f"RT n={n} nz={nz} ntheta={nt}: rel-L2 vs FP64 plain {e_plain:.3e} compensated {e_comp:.3e}")
    assert e_comp < 1e-5 and e_plain < 1e-5
    assert e_comp <= e_plain * 1.05                          # never worse than the plain sum
    assert torch.equal(comp, tk.RT(torch.from_numpy(y).cuda()))   # still deterministic
