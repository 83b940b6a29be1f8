"""Seeded synthetic ellipsoid volumes (the inputs of the forward-model workloads).

The reference runs on measured volumes that are not distributed with it
(README.md:583-597); the workloads here use seeded random ellipsoids instead:
`count` ellipsoids with centres uniform in the cylinder inscribed in the
(nz, n, n) box, semi-axes uniform in [0.05, 0.3] * n, uniform random Euler
rotations, values uniform in [vmin, vmax] (summed where they overlap) and a
zero background.
"""
from __future__ import annotations

import numpy as np


def _rotation(a, b, c):
    ca, sa, cb, sb, cc, sc = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(c), np.sin(c)
    rz1 = np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1]])
    ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    rz2 = np.array([[cc, -sc, 0], [sc, cc, 0], [0, 0, 1]])
    return rz1 @ ry @ rz2


def ellipsoid_params(n, nz, seed=0, count=10, vmin=1e-7, vmax=1e-6):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        rad = 0.5 * n * np.sqrt(rng.uniform())
        ang = rng.uniform(0, 2 * np.pi)
        cx, cy = rad * np.cos(ang), rad * np.sin(ang)
        cz = rng.uniform(-0.5, 0.5) * nz
        axes = rng.uniform(0.05, 0.3, 3) * n
        rot = _rotation(*rng.uniform(0, 2 * np.pi, 3))
        val = rng.uniform(vmin, vmax)
        out.append((np.array([cz, cy, cx]), axes, rot, val))
    return out


def ellipsoid_volume(n, nz, seed=0, count=10, vmin=1e-7, vmax=1e-6, z0=0, z1=None):
    """float32 (z1 - z0, n, n) slab [z0, z1) of the seeded volume."""
    z1 = nz if z1 is None else z1
    vol = np.zeros((z1 - z0, n, n), np.float32)
    c = np.arange(n) - n / 2 + 0.5
    yy, xx = np.meshgrid(c, c, indexing="ij")
    for (ctr, axes, rot, val) in ellipsoid_params(n, nz, seed, count, vmin, vmax):
        inv = rot.T
        for iz in range(z0, z1):
            dz = iz - nz / 2 + 0.5 - ctr[0]
            d = np.stack([np.full_like(yy, dz), yy - ctr[1], xx - ctr[2]])      # (3, n, n) in (z, y, x)
            q = np.tensordot(inv, d, axes=1)
            inside = (q[0] / axes[0]) ** 2 + (q[1] / axes[1]) ** 2 + (q[2] / axes[2]) ** 2 <= 1.0
            vol[iz - z0][inside] += np.float32(val)
    return vol


def ellipsoid_volume_torch(n, nz, seed=0, count=10, vmin=1e-7, vmax=1e-6, device="cuda", zblock=16):
    """Same seeded volume as ``ellipsoid_volume``, evaluated on the GPU
    (float32 (nz, n, n) torch tensor); used for the large workloads."""
    import torch
    vol = torch.zeros((nz, n, n), dtype=torch.float32, device=device)
    c = torch.arange(n, device=device, dtype=torch.float64) - n / 2 + 0.5
    for (ctr, axes, rot, val) in ellipsoid_params(n, nz, seed, count, vmin, vmax):
        inv = rot.T
        for z0 in range(0, nz, zblock):
            z1 = min(nz, z0 + zblock)
            dz = (torch.arange(z0, z1, device=device, dtype=torch.float64) - nz / 2 + 0.5 - ctr[0])[:, None, None]
            dy = (c - ctr[1])[None, :, None]
            dx = (c - ctr[2])[None, None, :]
            acc = None
            for r in range(3):
                q = inv[r, 0] * dz + inv[r, 1] * dy + inv[r, 2] * dx
                t = (q / axes[r]) ** 2
                acc = t if acc is None else acc + t
            vol[z0:z1] += (acc <= 1.0).to(torch.float32) * float(np.float32(val))
    return vol
