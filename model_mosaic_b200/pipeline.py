"""Host-to-host forward hot path over a stream of volumes.

The reference moves its data between host and device with three private
streams so that copies overlap compute (processing/pipeline.py:298-300).
``StreamedForward`` does the same for the forward hot path of
step2_radon + step3_propagation -- R, then psi = exp(-p s/beta_r)(cos p s,
sin p s), Fresnel D and |.|^2 (step3_propagation.py:94-110,175-176) -- on
one GPU: every submitted volume is copied in on one stream, computed on a
second and its intensities copied out on a third, with two device buffers
per side, so the copy-in of volume i+1, the compute of volume i and the
copy-out of volume i-1 run at the same time (PCIe is full duplex).

    fwd = StreamedForward(n, nz, theta, wavelength, voxelsize, distance, inv_norm, inv_beta)
    for obj_h, out_h in zip(volumes, outputs):   # pinned host tensors
        fwd.submit(obj_h, out_h)                 # returns at once
    fwd.synchronize()                            # all outputs written

Host tensors must be pinned (page-locked) for the copies to be asynchronous;
``pinned_volume`` / ``pinned_intensity`` allocate them.  A host buffer
passed to ``submit`` must not be modified (input) or read (output) before
``synchronize`` (or the returned event) says the step is done.
"""
from __future__ import annotations

import numpy as np
import torch

from model_mosaic_b200._interop import require_cuda
from model_mosaic_b200.processing.propagation import Propagation
from model_mosaic_b200.processing.tomo import TomoReal


class StreamedForward:
    def __init__(self, n, nz, theta, wavelength, voxelsize, distance, inv_norm, inv_beta, *, device=None):
        require_cuda()
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.n, self.nz = int(n), int(nz)
        self.theta = np.asarray(theta).astype(np.float32)
        self.ntheta = len(self.theta)
        self.inv_norm, self.inv_beta = float(inv_norm), float(inv_beta)
        with torch.cuda.device(self.device):
            self.tomo = TomoReal(self.n, self.nz, self.theta)
            self.prop = Propagation(self.n, self.nz, self.ntheta, 1, wavelength, voxelsize, [float(distance)])
            shape_in, shape_out = (self.nz, self.n, self.n), (self.ntheta, self.nz, self.n)
            self._in = [torch.empty(shape_in, dtype=torch.float32, device=self.device) for _ in range(2)]
            self._out = [torch.empty(shape_out, dtype=torch.float32, device=self.device) for _ in range(2)]
            self._sino = torch.empty(shape_out, dtype=torch.float32, device=self.device)
            self.s_in = torch.cuda.Stream(self.device)
            self.s_compute = torch.cuda.Stream(self.device)
            self.s_out = torch.cuda.Stream(self.device)
        # per buffer slot: compute finished reading _in[k]; copy-out finished reading _out[k]
        self._in_free = [None, None]
        self._out_free = [None, None]
        self._i = 0

    def pinned_volume(self):
        return torch.empty((self.nz, self.n, self.n), dtype=torch.float32).pin_memory()

    def pinned_intensity(self):
        return torch.empty((self.ntheta, self.nz, self.n), dtype=torch.float32).pin_memory()

    def submit(self, obj_host: torch.Tensor, out_host: torch.Tensor) -> torch.cuda.Event:
        """Queue one volume; returns the event recorded after its copy-out."""
        if tuple(obj_host.shape) != (self.nz, self.n, self.n) or obj_host.dtype != torch.float32:
            raise ValueError(f"obj must be float32 ({self.nz}, {self.n}, {self.n}), got {obj_host.dtype} "
                             f"{tuple(obj_host.shape)}")
        if tuple(out_host.shape) != (self.ntheta, self.nz, self.n) or out_host.dtype != torch.float32:
            raise ValueError(f"out must be float32 ({self.ntheta}, {self.nz}, {self.n})")
        k = self._i & 1
        self._i += 1
        x, y = self._in[k], self._out[k]
        with torch.cuda.device(self.device):
            # copy in, once the compute two steps back has finished reading this slot
            if self._in_free[k] is not None:
                self.s_in.wait_event(self._in_free[k])
            with torch.cuda.stream(self.s_in):
                x.copy_(obj_host, non_blocking=True)
                loaded = torch.cuda.Event()
                loaded.record(self.s_in)
            # compute, once the copy-out two steps back has finished reading this slot
            self.s_compute.wait_event(loaded)
            if self._out_free[k] is not None:
                self.s_compute.wait_event(self._out_free[k])
            with torch.cuda.stream(self.s_compute):
                self.tomo.R_into(x, self._sino)
                self.prop.intensity_into(self._sino, y, self.inv_norm, self.inv_beta)
                done = torch.cuda.Event()
                done.record(self.s_compute)
            self._in_free[k] = done
            # copy out
            self.s_out.wait_event(done)
            with torch.cuda.stream(self.s_out):
                out_host.copy_(y, non_blocking=True)
                copied = torch.cuda.Event()
                copied.record(self.s_out)
            self._out_free[k] = copied
        return copied

    def synchronize(self):
        for s in (self.s_in, self.s_compute, self.s_out):
            s.synchronize()

    def free(self):
        self.synchronize()
        self.tomo.free()
        self.prop.free()
        self._in = self._out = self._sino = None
