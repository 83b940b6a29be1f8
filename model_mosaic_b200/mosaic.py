"""Mosaic tiles -- the step4 extract / step6 stitch tile logic on one B200.

Host side, restating the reference scripts:

* ``mosaic_layout(ups)``: the tile placements step0_schematic.py computes for
  a pipeline upsampling factor (step0_schematic.py:57-100, 112-189, 300-320).
* ``write_positions_file`` / ``read_placements``: the mosaic_positions text
  format (step0_schematic.py:192-245) and its parser with the derived direct
  and mirror footprints (step4_extract.py:52-118).
* ``tent_weight``: the capped separable blending weight (step6_stitch.py:70-81).
* ``tile_theta`` / ``stitched_theta``: the angle arrays of the tile files and
  of the stitched projection (step4_extract.py:156-157, step6_stitch.py:137).

Device side (``libmosaic.so``):

* ``MosaicTiles.extract``: the crop loop of step4_extract.py:176-192, the
  direct crop and the h-flipped mirror crop of every placement.
* ``MosaicTiles.stitch``: the blend loop of step6_stitch.py:206-262, the
  tent-weighted mirror-folded sum over placements divided by the summed
  weights, 1.0 where nothing covers a pixel -- bit-identical to the
  reference's float32 arithmetic.
"""
from __future__ import annotations

import ctypes as C
import re

import numpy as np
import torch

from model_mosaic_b200 import _ffi
from model_mosaic_b200._interop import require_cuda, stream_ptr

HEADER_KEYS = ("NZ", "N", "DET_H", "DET_W", "n_z", "n_x", "NTHETA", "N_HALF", "OVERLAP")
RECT_KEYS = ("r_lo_dir", "r_hi_dir", "c_lo_dir", "c_hi_dir", "r_lo_mir", "r_hi_mir", "c_lo_mir", "c_hi_mir")


# --------------------------------------------------------------------------
# Layout (step0_schematic.py)

def _x_origins(det_w, overlap, axis_inset, sample_r_px):
    """Tile left edges relative to the rotation axis (step0_schematic.py:112-133):
    tile 0 puts the axis `axis_inset` inside its left border, every next tile
    moves right by det_w - overlap until the sample radius is covered."""
    step = det_w - overlap
    r0_max = det_w - axis_inset
    n_shifts = 0 if r0_max >= sample_r_px else int(np.ceil((sample_r_px - r0_max) / step))
    origins = np.empty(n_shifts + 1)
    origins[0] = 0.0 - axis_inset
    for i in range(1, n_shifts + 1):
        origins[i] = origins[i - 1] + step
    return origins


def _z_positions(det_h, z_overlap, sample_h_px):
    """Tile top edges (step0_schematic.py:136-148): uniform step det_h - z_overlap,
    the stack centred on the sample with equal overshoot at both ends."""
    step_z = det_h - z_overlap
    if sample_h_px <= det_h:
        return np.array([-(det_h - sample_h_px) / 2.0])
    n_z = int(np.ceil((sample_h_px - det_h) / step_z)) + 1
    span = n_z * det_h - (n_z - 1) * z_overlap
    return -((span - sample_h_px) / 2.0) + np.arange(n_z) * step_z


def compute_tile_placements(nz, n, det_h, det_w, z_pad, x_origins, z_positions):
    """Direct placement of every (z, x) tile in big-projection pixels with the
    crops that keep its footprint inside (nz, n) (step0_schematic.py:151-189)."""
    out = []
    for zi, zpos in enumerate(z_positions):
        z0 = int(round(float(zpos))) + z_pad
        ct, cb = max(0, -z0), max(0, z0 + det_h - nz)
        for xi, xorg in enumerate(x_origins):
            x0 = int(round(float(xorg))) + n // 2
            out.append(dict(zi=zi, xi=xi, z_center=z0 + det_h // 2, x_center=x0 + det_w // 2,
                            crop_top=ct, crop_bottom=cb,
                            crop_left=max(0, -x0), crop_right=max(0, x0 + det_w - n)))
    return out


def mosaic_layout(ups: int):
    """(meta, rows) of the mosaic the reference plans for upsampling factor
    `ups`: the physical detector (3232 x 2426 px at 1.38 um, 200 px overlaps
    and axis inset at ups = 8) scaled to the pipeline voxel, a cylinder of
    2918·ups x 2972·ups voxels in a (3072·ups)^3 volume, 3N/4 angles per 180°
    (step0_schematic.py:57-100, 300-320).  `rows` are the positions-file rows
    (zi, xi, z_center, x_center, crop_top, crop_bottom, crop_left, crop_right)."""
    ups = int(ups)
    det_w, det_h = 3232 * ups // 8, 2426 * ups // 8
    overlap = axis_inset = z_overlap = 200 * ups // 8
    pixel_um = 1.38 * 8 / ups
    sample_d_px, sample_h_px = 2918 * ups, 2972 * ups
    to_px = lambda mm: mm / (pixel_um * 1e-3)
    sample_r = to_px(sample_d_px * pixel_um * 1e-3) / 2.0
    sample_h = to_px(sample_h_px * pixel_um * 1e-3)
    xo = _x_origins(det_w, overlap, axis_inset, sample_r)
    zp = _z_positions(det_h, z_overlap, sample_h)
    n = nz = 3072 * ups
    n_half = 3 * n // 4
    pl = compute_tile_placements(nz, n, det_h, det_w, (nz - sample_h_px) // 2, xo, zp)
    meta = dict(NZ=nz, N=n, DET_H=det_h, DET_W=det_w, n_z=len(zp), n_x=len(xo), NTHETA=2 * n_half,
                N_HALF=n_half, OVERLAP=overlap)
    rows = [[p["zi"], p["xi"], p["z_center"], p["x_center"], p["crop_top"], p["crop_bottom"], p["crop_left"],
             p["crop_right"]] for p in pl]
    return meta, np.asarray(rows, dtype=np.int64)


def write_positions_file(path, meta, rows) -> None:
    """Write a mosaic_positions text file: '#' comment lines, one of them the
    KEY=value header read_placements needs, then one row of 8 integers per tile
    (the format of step0_schematic.py:192-245)."""
    head = " ".join(f"{k}={int(meta[k])}" for k in HEADER_KEYS)
    with open(path, "w") as f:
        f.write("# Mosaic tile positions (direct placements; mirrors derived by the reader).\n")
        f.write(f"# {head}\n")
        f.write("# columns: z_tile x_tile z_center x_center crop_top crop_bottom crop_left crop_right\n")
        for r in np.asarray(rows, dtype=np.int64):
            f.write(" ".join(str(int(v)) for v in r) + "\n")


def read_placements(txt_path):
    """Parse a positions file into (meta, placements) (step4_extract.py:52-118).

    meta holds the nine header integers; each placement dict has the file's
    columns plus the direct footprint rows [r_lo_dir, r_hi_dir) x cols
    [c_lo_dir, c_hi_dir) and the mirror footprint: same rows, centre
    reflected to N - x_center, left/right crops swapped by the h-flip.
    Missing header keys raise ValueError naming them."""
    kv, rows = {}, []
    with open(txt_path) as f:
        for line in f:
            s = line.strip()
            if not s:
                continue
            if s.startswith("#"):
                for m in re.finditer(r"(\w+)\s*=\s*(-?\d+)", s.lstrip("#")):
                    kv[m.group(1)] = int(m.group(2))
                continue
            rows.append([int(x) for x in s.split()])
    missing = [k for k in HEADER_KEYS if k not in kv]
    if missing:
        raise ValueError(f"positions file {txt_path} missing header keys: {missing}")
    meta = {k: kv[k] for k in HEADER_KEYS}
    dh, dw, n = meta["DET_H"], meta["DET_W"], meta["N"]
    placements = []
    for zi, xi, zc, xc, ct, cb, cl, cr in rows:
        z0, x0, x0m = zc - dh // 2, xc - dw // 2, (n - xc) - dw // 2
        placements.append(dict(
            zi=zi, xi=xi, z_center=zc, x_center=xc,
            crop_top=ct, crop_bottom=cb, crop_left=cl, crop_right=cr,
            r_lo_dir=z0 + ct, r_hi_dir=z0 + dh - cb, c_lo_dir=x0 + cl, c_hi_dir=x0 + dw - cr,
            r_lo_mir=z0 + ct, r_hi_mir=z0 + dh - cb, c_lo_mir=x0m + cr, c_hi_mir=x0m + dw - cl))
    return meta, placements


def tent_weight(h: int, w: int, cap: int) -> np.ndarray:
    """float32 (h, w) blending weight min(i+½, h-i-½, cap)·min(j+½, w-j-½, cap)
    (step6_stitch.py:70-81): positive on the whole tile, a linear ramp across
    an overlap band of width cap."""
    def ramp(k):
        a = np.arange(k, dtype=np.float32) + 0.5
        return np.minimum(np.minimum(a, k - a), float(cap))
    return (ramp(h)[:, None] * ramp(w)[None, :]).astype(np.float32)


def tile_theta(theta_data_deg) -> np.ndarray:
    """Angles of a tile file: the 180° scan then the same angles + 180°
    (step4_extract.py:156-157), float32 degrees."""
    t = np.asarray(theta_data_deg)
    return np.concatenate([t, t + 180.0]).astype(np.float32)


def stitched_theta(theta_tile_deg, n_half: int) -> np.ndarray:
    """Angles of the stitched 180° projection: the tiles' first N_HALF (step6_stitch.py:137)."""
    return np.asarray(theta_tile_deg)[:n_half]


def placement_rects(placements) -> np.ndarray:
    """int32 (n_place, 8) footprints in RECT_KEYS order."""
    return np.asarray([[p[k] for k in RECT_KEYS] for p in placements], dtype=np.int32)


# --------------------------------------------------------------------------
# Device extract / stitch

def _check_f32(t, shape, what):
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32):
        raise TypeError(f"{what}: expected a float32 CUDA tensor")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{what}: shape {tuple(t.shape)} is not {tuple(shape)}")
    if not t.is_contiguous():
        raise ValueError(f"{what}: must be contiguous")


class MosaicTiles:
    """Tile extraction and stitching for one mosaic (meta, placements of read_placements)."""

    def __init__(self, meta, placements):
        require_cuda()
        self.meta = dict(meta)
        self.nz, self.n = int(meta["NZ"]), int(meta["N"])
        self.n_half, self.overlap = int(meta["N_HALF"]), int(meta["OVERLAP"])
        self.placements = list(placements)
        rects = placement_rects(self.placements)
        self.shapes = [(int(r[1] - r[0]), int(r[3] - r[2])) for r in rects]
        h = C.c_void_p()
        _ffi.check(_ffi.lib().mm_mosaic_create(self.nz, self.n, len(rects), rects.ctypes.data_as(C.c_void_p),
                                               self.overlap, C.byref(h)), "mm_mosaic_create")
        self._h = h

    def free(self):
        if getattr(self, "_h", None):
            _ffi.lib().mm_mosaic_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def info(self):
        """(row cells, column cells, most footprints over one pixel)."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        _ffi.check(_ffi.lib().mm_mosaic_info(self._live(), C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def _live(self):
        if self._h is None:
            raise RuntimeError("MosaicTiles used after free()")
        return self._h

    def _ptrs(self, frames, nth, what):
        if len(frames) != len(self.shapes):
            raise ValueError(f"{what}: {len(frames)} tiles for {len(self.shapes)} placements")
        for k, (t, (h, w)) in enumerate(zip(frames, self.shapes)):
            _check_f32(t, (nth, h, w), f"{what}[{k}]")
        return (C.c_void_p * len(frames))(*[t.data_ptr() for t in frames])

    def extract_into(self, proj: torch.Tensor, direct, mirror):
        """proj (nth, NZ, N) -> direct[p], mirror[p] (nth, h_p, w_p): the direct
        crop and the h-flipped mirror crop of every placement."""
        nth = int(proj.shape[0])
        _check_f32(proj, (nth, self.nz, self.n), "proj")
        d, m = self._ptrs(direct, nth, "direct"), self._ptrs(mirror, nth, "mirror")
        _ffi.check(_ffi.lib().mm_mosaic_extract(self._live(), C.c_void_p(proj.data_ptr()), nth, d, m,
                                                C.c_void_p(stream_ptr(proj.device))), "mm_mosaic_extract")

    def extract(self, proj: torch.Tensor):
        """Tile scans of a 180° projection stack proj (nth, NZ, N): one
        (2·nth, h_p, w_p) tensor per placement, direct frames first, mirror
        frames second -- the tile-file layout of step4_extract.py:186-188
        when proj holds all N_HALF angles."""
        nth = int(proj.shape[0])
        tiles = [torch.empty((2 * nth, h, w), dtype=torch.float32, device=proj.device) for h, w in self.shapes]
        self.extract_into(proj, [t[:nth] for t in tiles], [t[nth:] for t in tiles])
        return tiles

    def stitch_into(self, direct, mirror, out: torch.Tensor):
        """direct[p] = tile p's frames at the output angles, mirror[p] = its
        frames N_HALF later, each (nth, h_p, w_p) -> out (nth, NZ, N)."""
        nth = int(out.shape[0])
        _check_f32(out, (nth, self.nz, self.n), "out")
        d, m = self._ptrs(direct, nth, "direct"), self._ptrs(mirror, nth, "mirror")
        _ffi.check(_ffi.lib().mm_mosaic_stitch(self._live(), d, m, nth, C.c_void_p(out.data_ptr()),
                                               C.c_void_p(stream_ptr(out.device))), "mm_mosaic_stitch")
        return out

    def stitch(self, tiles, t0: int = 0, nth: int | None = None, out: torch.Tensor | None = None):
        """Stitched projection at output angles [t0, t0 + nth) from tile scans
        (NTHETA, h_p, w_p) (step6_stitch.py:206-262).  The mirror angles
        t + N_HALF must stay inside the scans (the reference's no-wrap rule)."""
        nth = self.n_half - t0 if nth is None else int(nth)
        if t0 < 0 or nth < 0 or t0 + nth > self.n_half:
            raise ValueError(f"output angles [{t0}, {t0 + nth}) outside [0, N_HALF={self.n_half})")
        for k, t in enumerate(tiles):
            if t.shape[0] < self.n_half + t0 + nth:
                raise ValueError(f"tile {k} holds {t.shape[0]} angles; mirror range ends at "
                                 f"{self.n_half + t0 + nth}")
        dev = tiles[0].device
        if out is None:
            out = torch.empty((nth, self.nz, self.n), dtype=torch.float32, device=dev)
        return self.stitch_into([t[t0:t0 + nth] for t in tiles],
                                [t[self.n_half + t0:self.n_half + t0 + nth] for t in tiles], out)

    def workspace_bytes(self) -> int:
        return int(_ffi.lib().mm_mosaic_workspace_bytes(self._live()))
