"""Batches of uneven mosaic tiles through the hot path in one CUDA graph.

A mosaic scan is processed tile by tile: the reference runs step2_radon /
step3_propagation once per extracted tile (step4_extract.py,
step6_stitch.py:74-91), each tile with its own size n and angle count.
``TileBatch`` runs many such tiles on one GPU as a single CUDA graph: every
tile owns its TomoReal / Propagation handles and device buffers, its steps
(R, psi -> D -> |.|^2, and RT of its sinogram) are captured once, and the
tiles are spread over several streams inside the capture so that the kernels
of small tiles overlap.  One ``run()`` is one graph launch.

    batch = TileBatch([dict(n=512, nz=16, theta=th0), dict(n=768, nz=16, theta=th1), ...],
                      wavelength, voxelsize, distance)
    for i, vol in enumerate(volumes):
        batch.obj(i).copy_(vol)          # (nz, n, n) float32 device tensors
    batch.capture()                      # eager warm-up, then graph capture
    batch.run()                          # intensity(i), rec(i) hold the results

Per tile: inv_norm = 1/sqrt(n/ntheta) (step3_propagation.py:82) unless given,
beta = delta/beta_ratio.  Sizes without native kernels use the library's cuFFT
paths, which capture like the rest.
"""
from __future__ import annotations

import numpy as np
import torch

from model_mosaic_b200._interop import require_cuda
from model_mosaic_b200.processing.propagation import Propagation
from model_mosaic_b200.processing.tomo import TomoReal


class _Tile:
    def __init__(self, n, nz, theta, wavelength, voxelsize, distance, inv_norm, inv_beta, device,
                 eps=1e-3, m=None):
        self.n, self.nz = int(n), int(nz)
        self.theta = np.asarray(theta).astype(np.float32)
        self.ntheta = len(self.theta)
        self.inv_norm = float(np.float32(1.0 / np.sqrt(self.n / self.ntheta))) if inv_norm is None else float(inv_norm)
        self.inv_beta = float(inv_beta)
        self.eps, self.m = float(eps), m
        self.tomo = TomoReal(self.n, self.nz, self.theta, eps=self.eps, m=m)
        self.prop = Propagation(self.n, self.nz, self.ntheta, 1, wavelength, voxelsize, [float(distance)])
        f32 = dict(dtype=torch.float32, device=device)
        self.obj = torch.zeros((self.nz, self.n, self.n), **f32)
        self.sino = torch.empty((self.ntheta, self.nz, self.n), **f32)
        self.inten = torch.empty((self.ntheta, self.nz, self.n), **f32)
        self.rec = torch.empty((self.nz, self.n, self.n), **f32)

    def step(self):
        self.tomo.R_into(self.obj, self.sino)
        self.prop.intensity_into(self.sino, self.inten, self.inv_norm, self.inv_beta)
        self.tomo.RT_into(self.sino, self.rec)

    def voxel_angles(self):
        return self.nz * self.n * self.n * self.ntheta

    def free(self):
        self.tomo.free()
        self.prop.free()


class TileBatch:
    """``tiles``: dicts with n, theta and optionally nz (16), inv_norm, and the
    USFFT accuracy pair eps / m (default the reference's eps = 1e-3, m from
    eps).  ``params`` maps a tile size n to an (eps, m) pair for every tile of
    that size that does not give its own (``autotune.tune_tiles`` returns one)."""

    def __init__(self, tiles, wavelength, voxelsize, distance, *, beta_ratio=100.0, streams=4, device=None,
                 params=None):
        require_cuda()
        if isinstance(device, torch.device):
            self.device = device
        else:
            self.device = torch.device("cuda", torch.cuda.current_device() if device is None else int(device))
        params = params or {}
        with torch.cuda.device(self.device):
            self.tiles = []
            for t in tiles:
                eps, m = params.get(int(t["n"]), (1e-3, None))
                self.tiles.append(_Tile(t["n"], t.get("nz", 16), t["theta"], wavelength, voxelsize, distance,
                                        t.get("inv_norm"), 1.0 / beta_ratio, self.device,
                                        eps=t.get("eps", eps), m=t.get("m", m)))
            self.set_streams(streams)
        self.graph = None

    def set_streams(self, streams: int):
        """Worker streams the tiles are spread over (a captured graph is dropped)."""
        self.streams = [torch.cuda.Stream(self.device) for _ in range(max(1, int(streams)))]
        self.graph = None

    # -- buffers -------------------------------------------------------------
    def obj(self, i) -> torch.Tensor:
        return self.tiles[i].obj

    def intensity(self, i) -> torch.Tensor:
        return self.tiles[i].inten

    def sinogram(self, i) -> torch.Tensor:
        return self.tiles[i].sino

    def rec(self, i) -> torch.Tensor:
        return self.tiles[i].rec

    def voxel_angles(self) -> int:
        return sum(t.voxel_angles() for t in self.tiles)

    # -- execution -------------------------------------------------------------
    def _enqueue(self, origin: torch.cuda.Stream):
        """Fork from `origin` onto the worker streams (largest tiles first,
        round robin), run every tile, join back into `origin`."""
        fork = torch.cuda.Event()
        fork.record(origin)
        for s in self.streams:
            s.wait_event(fork)
        order = sorted(range(len(self.tiles)), key=lambda i: -self.tiles[i].voxel_angles())
        for k, i in enumerate(order):
            with torch.cuda.stream(self.streams[k % len(self.streams)]):
                self.tiles[i].step()
        for s in self.streams:
            done = torch.cuda.Event()
            done.record(s)
            origin.wait_event(done)

    def run_eager(self):
        with torch.cuda.device(self.device):
            self._enqueue(torch.cuda.current_stream(self.device))

    def capture(self):
        """One eager pass (scatter tables, cuFFT plans and kernel attributes
        are set up on first use), then capture the whole batch as one graph."""
        with torch.cuda.device(self.device):
            self.run_eager()
            torch.cuda.synchronize(self.device)
            self.graph = torch.cuda.CUDAGraph()
            cap = torch.cuda.Stream(self.device)
            with torch.cuda.graph(self.graph, stream=cap):
                self._enqueue(cap)
            torch.cuda.synchronize(self.device)

    def run(self):
        if self.graph is None:
            self.run_eager()
        else:
            self.graph.replay()

    def free(self):
        torch.cuda.synchronize(self.device)
        self.graph = None
        for t in self.tiles:
            t.free()
        self.tiles = []
