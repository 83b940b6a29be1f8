"""Differentiable forward model data = |D(exp(i(R delta + i R beta)))|^2.

The reference composes this model only across step2_radon (R) -> disk ->
step3_propagation (psi, D, |.|^2), with beta = delta / beta_r and the phase
scale s = PHASE_SCALE / sqrt(N / NTHETA) (step3_propagation.py:82,98-100,
182-183); it has no adjoint of D and no gradient.  Here the model and the
gradient of its L2 loss

    L(delta) = sum (|D psi(s R delta)|^2 - d)^2,   psi(p) = exp(-p/beta_r) e^{i p}

run on the GPU through the C-ABI:

    p   = R delta                                   mm_tomo_R
    gu  = 4 (|D psi|^2 - d) D psi, loss partials    mm_prop_grad_forward (fused)
    gp  = s Re(conj(D^H gu) (i - 1/beta_r) psi)     mm_prop_grad_backward (fused)
    dL/d delta = R^T gp                              mm_tomo_RT

D, D^H and the psi recompute work per chunk of angles (``angle_chunk``), so
nothing of size (ntheta, nz, n) complex is kept; only the float sinograms p
and gp are.  ``plain_loss_and_grad`` composes the same gradient from the
unfused operators (R, D, DT, RT plus torch element-wise ops) for comparison.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from model_mosaic_b200 import _ffi
from model_mosaic_b200._interop import require_cuda, stream_ptr
from model_mosaic_b200.processing.tomo import TomoReal
from model_mosaic_b200.processing.propagation import Propagation


class ForwardModel:
    def __init__(self, n, nz, theta, wavelength, voxelsize, distance, *, inv_norm=None, beta_ratio=100.0,
                 angle_chunk=None, compensated=False):
        require_cuda()
        self.n, self.nz = int(n), int(nz)
        self.theta = np.asarray(theta).astype(np.float32)
        self.ntheta = len(self.theta)
        self.s = float(np.float32(1.0 / np.sqrt(self.n / self.ntheta))) if inv_norm is None else float(inv_norm)
        self.ib = float(np.float32(1.0 / beta_ratio))
        self.chunk = int(angle_chunk or self.ntheta)
        self.tomo = TomoReal(self.n, self.nz, self.theta, compensated=compensated)
        self.prop = Propagation(self.n, self.nz, self.chunk, 1, wavelength, voxelsize, [float(distance)])
        self._gu = None
        self._partials = None

    def _bufs(self, dev):
        if self._gu is None:
            self._gu = torch.empty((self.chunk, self.nz, self.n), dtype=torch.complex64, device=dev)
            npart = _ffi.lib().mm_prop_grad_partials(self.prop._handle(), self.chunk)
            nchunks = (self.ntheta + self.chunk - 1) // self.chunk
            self._partials = torch.zeros((nchunks, npart), dtype=torch.float32, device=dev)
        return self._gu, self._partials

    def _chunks(self):
        for t0 in range(0, self.ntheta, self.chunk):
            yield t0, min(self.ntheta, t0 + self.chunk)

    def forward(self, delta: torch.Tensor) -> torch.Tensor:
        """(nz, n, n) float32 delta -> (ntheta, nz, n) float32 intensity."""
        p = torch.empty((self.ntheta, self.nz, self.n), dtype=torch.float32, device=delta.device)
        self.tomo.R_into(delta.contiguous(), p)
        out = torch.empty_like(p)
        for t0, t1 in self._chunks():
            self.prop.intensity_into(p[t0:t1], out[t0:t1], self.s, self.ib)
        return out

    def loss_and_grad(self, delta: torch.Tensor, data: torch.Tensor):
        """(L, dL/d delta) with the fused kernels."""
        L = _ffi.lib()
        dev = delta.device
        st = C.c_void_p(stream_ptr(dev))
        h = self.prop._handle()
        gu, partials = self._bufs(dev)
        p = torch.empty((self.ntheta, self.nz, self.n), dtype=torch.float32, device=dev)
        self.tomo.R_into(delta.contiguous(), p)
        gp = torch.empty_like(p)
        data = data.contiguous()
        partials.zero_()
        for c, (t0, t1) in enumerate(self._chunks()):
            nt = t1 - t0
            _ffi.check(L.mm_prop_grad_forward(h, C.c_void_p(p[t0:t1].data_ptr()), C.c_void_p(data[t0:t1].data_ptr()),
                                              self.s, self.ib, C.c_void_p(gu.data_ptr()),
                                              C.c_void_p(partials[c].data_ptr()), nt, 0, st))
            _ffi.check(L.mm_prop_grad_backward(h, C.c_void_p(gu.data_ptr()), C.c_void_p(p[t0:t1].data_ptr()),
                                               self.s, self.ib, C.c_void_p(gp[t0:t1].data_ptr()), nt, 0, st))
        grad = torch.empty_like(delta)
        self.tomo.RT_into(gp, grad)
        loss = partials.double().sum()
        return loss, grad

    def plain_loss_and_grad(self, delta: torch.Tensor, data: torch.Tensor):
        """The same gradient composed from the unfused operators: R, psi (torch),
        D (complex), |.|^2 and the loss (torch), then D^H, the chain through psi
        (torch) and R^T, with the complex intermediate kept for all angles."""
        p = torch.empty((self.ntheta, self.nz, self.n), dtype=torch.float32, device=delta.device)
        self.tomo.R_into(delta.contiguous(), p)
        phase = p * self.s
        psi = torch.exp(-phase * self.ib) * torch.complex(torch.cos(phase), torch.sin(phase))
        u = torch.empty_like(psi)
        gpsi = torch.empty_like(psi)
        for t0, t1 in self._chunks():
            self.prop.D_into(psi[t0:t1], u[t0:t1])
        r = u.real ** 2 + u.imag ** 2 - data
        loss = (r.double() ** 2).sum()
        gu = 4 * r * u
        for t0, t1 in self._chunks():
            self.prop.DT_into(gu[t0:t1].contiguous(), gpsi[t0:t1])
        w = torch.complex(torch.zeros_like(phase), torch.ones_like(phase)) - self.ib
        gp = self.s * (torch.conj(gpsi) * w * psi).real
        grad = torch.empty_like(delta)
        self.tomo.RT_into(gp.contiguous(), grad)
        return loss, grad


class FresnelRadonLoss(torch.autograd.Function):
    """loss = FresnelRadonLoss.apply(delta, data, model): L2 misfit of the
    forward model with its hand-written adjoint as the backward."""

    @staticmethod
    def forward(ctx, delta, data, model):
        loss, grad = model.loss_and_grad(delta.detach(), data.detach())
        ctx.save_for_backward(grad)
        return loss.to(delta.dtype)

    @staticmethod
    def backward(ctx, g):
        (grad,) = ctx.saved_tensors
        return g * grad, None, None
