"""The reference's GPU path on this box: its own CUDA kernels plus its host
glue restated with torch (cuFFT) in place of cupy.

TEST INFRASTRUCTURE AND BASELINE ONLY -- see ``oracle/__init__.py``.  cupy
is not installed, so the reference classes cannot run as they are; but all
of their device arithmetic is either one of the CUDA kernel strings of
``processing/kernels.py`` (compiled verbatim for sm_100a into
``oracle/_ref/libref_gpu.so`` by ``oracle/build_ref.py``, launched here with
the reference's own grid and block shapes) or a cuFFT transform, a fill or
an element-wise product, which torch issues on the same library.  Each
method follows the reference line by line:

* RefGpuTomoReal.R ........ processing/tomo.py:121-151
* RefGpuTomoReal.RT ....... processing/tomo.py:153-188 (atomic scatter)
* RefGpuPropagation.D ..... processing/propagation.py:36-64 (beyond the pad
  kernel's 32-bit index range, the same mirror padding with torch gathers)
* psi / |.|^2 ............. step3_propagation.py:94-110 (element-wise)

It serves three purposes: GPU parity of the product against the reference's
own kernels at sizes the CPU oracle cannot reach, the "cupy reference" time
of R, RT and D on the same GPU, and the plain composed forward+gradient step
(``ref_loss_and_grad``) that the fused model is compared with.  The adjoint
of D used there (``RefGpuPropagation.DT``) has no reference counterpart: it
is the exact adjoint of the reference's D written in the same style.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np
import torch

from .usfft import usfft_params, phi_table, c1dfftshift
from .fresnel import fresnel_kernel, mirror_index

_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libref_gpu.so")
_LIB = None
_INT_MAX = 2 ** 31 - 1


def _need_int32(what: str, count: int):
    """The reference's kernels compute element offsets in 32-bit int: past
    2^31 - 1 they address memory outside their buffers (at n = 24576 its
    scatter wrote out of bounds and its pad kernel made an illegal access).
    Such sizes are refused instead of run."""
    if count > _INT_MAX:
        raise ValueError(f"{what}: {count} elements exceed the reference kernel's 32-bit indexing")


def available() -> bool:
    return os.path.exists(_PATH)


def lib():
    global _LIB
    if _LIB is None:
        if not available():
            raise FileNotFoundError(f"{_PATH} missing: run python oracle/build_ref.py")
        L = C.CDLL(_PATH)
        u, p, i = C.c_uint, C.c_void_p, C.c_int
        grid = [u, u, u, u, u, u, p]
        L.refgpu_gather.argtypes = grid + [p, p, p, i, p, i, i, i, C.c_bool]
        L.refgpu_gather_rfft_full.argtypes = grid + [p, p, p, i, p, i, i, i]
        L.refgpu_pad_fwd.argtypes = grid + [p, p, i, i, i]
        for f in (L.refgpu_gather, L.refgpu_gather_rfft_full, L.refgpu_pad_fwd):
            f.restype = C.c_int
        _LIB = L
    return _LIB


def _launch(fn, grid, block, *args):
    st = torch.cuda.current_stream().cuda_stream
    rc = fn(*grid, *block, C.c_void_p(st), *args)
    if rc != 0:
        raise RuntimeError(f"reference kernel launch failed: cudaError {rc}")


def _p(t: torch.Tensor):
    return C.c_void_p(t.data_ptr())


class RefGpuTomoReal:
    """TomoReal (processing/tomo.py:17-188) with torch in place of cupy."""

    def __init__(self, n, nz, theta, device="cuda"):
        self.n, self._nz = int(n), int(nz)
        th = np.asarray(theta).astype(np.float32)
        self.ntheta = len(th)
        dev = torch.device(device)
        self.theta = torch.from_numpy(th).to(dev)
        mu, self.m = usfft_params(self.n)                                  # tomo.py:39-42
        self.mua = torch.tensor([mu], dtype=torch.float32, device=dev)
        self.phi = torch.from_numpy(phi_table(self.n, self.ntheta, mu, np.float32)).to(dev)
        self.c1d = torch.from_numpy(c1dfftshift(self.n).astype(np.float32)).to(dev)
        c2 = (1 - 2 * (np.arange(1, 2 * self.n + 1) % 2)).astype(np.float32)
        self.c2d = torch.from_numpy(np.outer(c2, c2)).to(dev)
        n = self.n
        _need_int32("gather_rfft_full spectrum", self._nz * 2 * n * (n + 1))
        _need_int32("gather_rfft_full sinogram", self.ntheta * self._nz * n)
        self._buf_padded = torch.zeros((self._nz, 2 * n, 2 * n), dtype=torch.float32, device=dev)
        self._buf_sino = torch.zeros((self.ntheta, self._nz, n), dtype=torch.complex64, device=dev)
        self._buf_fde_full = None

    def R(self, obj: torch.Tensor) -> torch.Tensor:
        """tomo.py:121-151."""
        nz, n = obj.shape[0], self.n
        self._buf_padded.zero_()
        torch.mul(obj, self.phi, out=self._buf_padded[:nz, n // 2:3 * n // 2, n // 2:3 * n // 2])
        fde = torch.fft.rfft2(self._buf_padded, dim=(-2, -1)).contiguous()
        self._buf_sino.zero_()
        _launch(lib().refgpu_gather_rfft_full, (math.ceil(n / 32), math.ceil(self.ntheta / 32), self._nz),
                (32, 32, 1), _p(self._buf_sino), _p(fde), _p(self.theta), self.m, _p(self.mua), n,
                self.ntheta, self._nz)
        self._buf_sino *= self.c1d
        self._buf_sino = torch.fft.ifft(self._buf_sino, dim=-1)
        self._buf_sino *= self.c1d
        return (self._buf_sino[:, :nz].real / 4).contiguous()

    def RT(self, data: torch.Tensor) -> torch.Tensor:
        """tomo.py:153-188: full complex path with the atomic scatter."""
        n, nz = self.n, data.shape[1]
        _need_int32("gather (dir=1) full spectrum", self._nz * 2 * n * 2 * n)
        if self._buf_fde_full is None:                                        # _lazy_init_rt, :90-107
            self._buf_fde_full = torch.zeros((self._nz, 2 * n, 2 * n), dtype=torch.complex64,
                                             device=self.theta.device)
        self._buf_sino[:, :nz] = (data * self.c1d).to(torch.complex64)
        self._buf_sino[:, nz:] = 0
        self._buf_sino = torch.fft.fft(self._buf_sino, dim=-1)
        self._buf_sino *= self.c1d
        self._buf_fde_full.zero_()
        _launch(lib().refgpu_gather, (math.ceil(n / 32), math.ceil(self.ntheta / 32), self._nz), (32, 32, 1),
                _p(self._buf_sino), _p(self._buf_fde_full), _p(self.theta), self.m, _p(self.mua), n,
                self.ntheta, self._nz, True)
        self._buf_fde_full *= self.c2d
        f = torch.fft.ifft2(self._buf_fde_full, dim=(-2, -1))
        f *= self.c2d
        res = f[:nz, n // 2:3 * n // 2, n // 2:3 * n // 2] * self.phi
        if data.dtype == torch.float32:
            res = res.real
        return res.contiguous()


class RefGpuPropagation:
    """Propagation (processing/propagation.py:15-64) with torch in place of cupy."""

    def __init__(self, n, nz, ntheta, ndist, wavelength, voxelsize, distance, device="cuda"):
        self.n, self.nz, self.ntheta = int(n), int(nz), int(ntheta)
        dev = torch.device(device)
        fk = fresnel_kernel(self.n, self.nz, wavelength, voxelsize, list(distance)[:ndist], np.float32)
        self.fker = torch.from_numpy(np.ascontiguousarray(fk)).to(dev)      # (ndist, 2nz, 2n), :22-31
        self._buf_big = torch.zeros((self.ntheta, 2 * self.nz, 2 * self.n), dtype=torch.complex64, device=dev)
        self.ix = torch.from_numpy(mirror_index(self.n)).to(dev)
        self.iy = torch.from_numpy(mirror_index(self.nz)).to(dev)

    def D(self, psi: torch.Tensor, j: int) -> torch.Tensor:
        """propagation.py:47-64."""
        added = psi.dim() == 2
        if added:
            psi = psi[None]
        nt, n, nz = psi.shape[0], self.n, self.nz
        psi = psi.contiguous()
        self._buf_big.zero_()
        if nt * 2 * nz * 2 * n <= _INT_MAX:
            _launch(lib().refgpu_pad_fwd, (math.ceil(2 * n / 32), math.ceil(2 * nz / 32), nt), (32, 32, 1),
                    _p(self._buf_big), _p(psi), n, nz, nt)
        else:
            # beyond the pad kernel's 32-bit indexing: the same mirror padding
            # (kernels.py:541-544) with torch's 64-bit gathers
            self._buf_big[:nt] = psi.index_select(1, self.iy).index_select(2, self.ix)
        f = torch.fft.fft2(self._buf_big, dim=(-2, -1))
        f *= self.fker[j]
        f = torch.fft.ifft2(f, dim=(-2, -1), norm="forward")
        res = f[:nt, nz // 2:nz // 2 + nz, n // 2:n // 2 + n].contiguous()
        return res[0] if added else res

    def DT(self, g: torch.Tensor, j: int) -> torch.Tensor:
        """Exact adjoint of D in the same style (no reference counterpart):
        zero embedding, FFT2, conj kernel, inverse, mirror fold."""
        nt, n, nz = g.shape[0], self.n, self.nz
        big = torch.zeros((nt, 2 * nz, 2 * n), dtype=torch.complex64, device=g.device)
        big[:, nz // 2:nz // 2 + nz, n // 2:n // 2 + n] = g
        f = torch.fft.fft2(big, dim=(-2, -1))
        f *= torch.conj(self.fker[j])
        f = torch.fft.ifft2(f, dim=(-2, -1), norm="forward")
        fx = torch.zeros((nt, 2 * nz, n), dtype=torch.complex64, device=g.device).index_add_(2, self.ix, f)
        return torch.zeros((nt, nz, n), dtype=torch.complex64, device=g.device).index_add_(1, self.iy, fx)


def psi_from_proj(p: torch.Tensor, inv_norm: float, inv_beta: float) -> torch.Tensor:
    """step3_propagation.py:94-103."""
    ph = p * inv_norm
    at = torch.exp(-ph * inv_beta)
    return torch.complex(at * torch.cos(ph), at * torch.sin(ph))


def abs2(z: torch.Tensor) -> torch.Tensor:
    """step3_propagation.py:105-110."""
    return z.real * z.real + z.imag * z.imag


def ref_loss_and_grad(tomo: RefGpuTomoReal, prop: RefGpuPropagation, delta, data, inv_norm, inv_beta,
                      chunk=128):
    """The plain composed step: p = R delta; per angle chunk psi, u = D psi,
    r = |u|^2 - d, loss += sum r^2, gu = 4 r u, gpsi = D^H gu,
    gp = s Re(conj(gpsi)(i - 1/beta_r) psi); then grad = R^T gp."""
    p = tomo.R(delta)
    T = p.shape[0]
    gp = torch.empty_like(p)
    loss = torch.zeros((), dtype=torch.float64, device=p.device)
    for t0 in range(0, T, chunk):
        t1 = min(T, t0 + chunk)
        psi = psi_from_proj(p[t0:t1], inv_norm, inv_beta)
        u = prop.D(psi, 0)
        r = abs2(u) - data[t0:t1]
        loss += (r.double() * r.double()).sum()
        gpsi = prop.DT(4 * r * u, 0)
        gp[t0:t1] = inv_norm * (torch.conj(gpsi) * torch.complex(-inv_beta * torch.ones_like(r),
                                                                  torch.ones_like(r)) * psi).real
    return loss, tomo.RT(gp)
