"""NumPy restatement of the reference's mosaic tile crop and stitch -- test infrastructure.

Only tests/, smoke() and bench.py's CPU legs use this module, as the checker;
the product is model_mosaic_b200/csrc/mosaic.cu.

step4_extract.py:176-192: for every placement, the tile scan is the direct
crop data[:, rows, cols_dir] followed by the mirror crop data[:, rows,
cols_mir] flipped left-right.

step6_stitch.py:206-262: for one block of output angles [t0, t1), every
placement adds w * tile[t] at its direct footprint and w * flip(tile[t +
N_HALF]) at its mirror footprint into a zeroed float32 buffer, the weights w
into a float32 plane; covered pixels are divided by the plane (times the
float32 reciprocal), uncovered ones set to 1.0.  The additions run in the
reference's order (placement by placement, direct before mirror) in float32,
so a float32 implementation can match it bit for bit.
"""
from __future__ import annotations

import numpy as np


def tent_weight(h, w, cap) -> np.ndarray:
    """float32 min(i+½, h-i-½, cap) x min(j+½, w-j-½, cap) (step6_stitch.py:70-81)."""
    zi = np.arange(h, dtype=np.float32) + 0.5
    xi = np.arange(w, dtype=np.float32) + 0.5
    wz = np.minimum(np.minimum(zi, h - zi), float(cap))
    wx = np.minimum(np.minimum(xi, w - xi), float(cap))
    return (wz[:, None] * wx[None, :]).astype(np.float32)


def extract(data, placements):
    """Tile scans (2·nth, h, w) float32 of data (nth, NZ, N) (step4_extract.py:176-192)."""
    data = np.asarray(data, dtype=np.float32)
    nth = data.shape[0]
    tiles = []
    for p in placements:
        rows = slice(p["r_lo_dir"], p["r_hi_dir"])
        h = p["r_hi_dir"] - p["r_lo_dir"]
        w = p["c_hi_dir"] - p["c_lo_dir"]
        tile = np.empty((2 * nth, h, w), dtype=np.float32)
        tile[:nth] = data[:, rows, p["c_lo_dir"]:p["c_hi_dir"]]
        tile[nth:] = data[:, p["r_lo_mir"]:p["r_hi_mir"], p["c_lo_mir"]:p["c_hi_mir"]][:, :, ::-1]
        tiles.append(tile)
    return tiles


def stitch(tiles, placements, nz, n, n_half, overlap, t0, t1) -> np.ndarray:
    """Stitched projection (t1 - t0, NZ, N) float32 from tile scans (step6_stitch.py:206-262)."""
    nth = t1 - t0
    buf = np.zeros((nth, nz, n), dtype=np.float32)
    wsum = np.zeros((nz, n), dtype=np.float32)
    for p, tile in zip(placements, tiles):
        h = p["r_hi_dir"] - p["r_lo_dir"]
        w = p["c_hi_dir"] - p["c_lo_dir"]
        wt = tent_weight(h, w, overlap)
        rows = slice(p["r_lo_dir"], p["r_hi_dir"])
        cd = slice(p["c_lo_dir"], p["c_hi_dir"])
        cm = slice(p["c_lo_mir"], p["c_hi_mir"])
        buf[:, rows, cd] += tile[t0:t1] * wt
        wsum[rows, cd] += wt
        buf[:, rows, cm] += tile[n_half + t0:n_half + t1][:, :, ::-1] * wt
        wsum[rows, cm] += wt
    covered = wsum > 0
    inv = np.zeros_like(wsum)
    np.divide(1.0, wsum, out=inv, where=covered)
    buf *= inv[None]
    buf[:, ~covered] = 1.0
    return buf
