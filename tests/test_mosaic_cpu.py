"""Mosaic tile logic on the CPU: the oracle and the host-side layout, parser
and weights against the reference's own outputs (tests/golden/mosaic.npz,
made by tests/golden/make_golden_mosaic.py from step4_extract.py,
step6_stitch.py and the shipped mosaic_positions files)."""
from __future__ import annotations

import os

import numpy as np
import pytest

from model_mosaic_b200 import mosaic as mo
from oracle import mosaic as om

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "mosaic.npz"))
META_KEYS = ("NZ", "N", "DET_H", "DET_W", "n_z", "n_x", "NTHETA", "N_HALF", "OVERLAP")
PL_KEYS = ("zi", "xi", "z_center", "x_center", "crop_top", "crop_bottom", "crop_left", "crop_right",
           "r_lo_dir", "r_hi_dir", "c_lo_dir", "c_hi_dir", "r_lo_mir", "r_hi_mir", "c_lo_mir", "c_hi_mir")


def case(name, tmp_path):
    meta = dict(zip(META_KEYS, (int(v) for v in GOLD[f"{name}_meta"])))
    path = tmp_path / f"positions_{name}.txt"
    mo.write_positions_file(path, meta, GOLD[f"{name}_rows"])
    meta2, pl = mo.read_placements(path)
    assert meta2 == meta
    return meta, pl


def split_tiles(flat, pl, nframes):
    out, k = [], 0
    for p in pl:
        h, w = p["r_hi_dir"] - p["r_lo_dir"], p["c_hi_dir"] - p["c_lo_dir"]
        out.append(flat[k:k + nframes * h * w].reshape(nframes, h, w))
        k += nframes * h * w
    assert k == flat.size
    return out


@pytest.mark.parametrize("name", ["A", "B"])
def test_oracle_extract_matches_reference(name, tmp_path):
    meta, pl = case(name, tmp_path)
    got = om.extract(GOLD[f"{name}_data"], pl)
    want = split_tiles(GOLD[f"{name}_tiles"], pl, meta["NTHETA"])
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)


@pytest.mark.parametrize("name", ["A", "B"])
def test_oracle_stitch_matches_reference_bitwise(name, tmp_path):
    meta, pl = case(name, tmp_path)
    tiles = split_tiles(GOLD[f"{name}_tiles_pre"], pl, meta["NTHETA"])
    chunk, n_half = int(GOLD[f"{name}_chunk"]), meta["N_HALF"]
    parts = [om.stitch(tiles, pl, meta["NZ"], meta["N"], n_half, meta["OVERLAP"], t0, min(t0 + chunk, n_half))
             for t0 in range(0, n_half, chunk)]
    got = np.concatenate(parts)
    np.testing.assert_array_equal(got.view(np.uint32), GOLD[f"{name}_stitched"].view(np.uint32))
    # uncovered pixels are air (1.0); case A leaves rows above and below the stack
    if name == "A":
        assert np.all(got[:, :2] == 1.0) and np.all(got[:, 54:] == 1.0)


def test_oracle_planted_order_change_is_detected(tmp_path):
    """Summing the mirror before the direct footprint changes float32 bits:
    the bitwise comparison can see the reference's accumulation order."""
    meta, pl = case("A", tmp_path)
    tiles = split_tiles(GOLD["A_tiles_pre"], pl, meta["NTHETA"])
    nz, n, nh, cap = meta["NZ"], meta["N"], meta["N_HALF"], meta["OVERLAP"]
    buf = np.zeros((nh, nz, n), np.float32)
    ws = np.zeros((nz, n), np.float32)
    for p, t in zip(pl, tiles):
        wt = om.tent_weight(p["r_hi_dir"] - p["r_lo_dir"], p["c_hi_dir"] - p["c_lo_dir"], cap)
        r = slice(p["r_lo_dir"], p["r_hi_dir"])
        buf[:, r, p["c_lo_mir"]:p["c_hi_mir"]] += t[nh:2 * nh][:, :, ::-1] * wt
        ws[r, p["c_lo_mir"]:p["c_hi_mir"]] += wt
        buf[:, r, p["c_lo_dir"]:p["c_hi_dir"]] += t[:nh] * wt
        ws[r, p["c_lo_dir"]:p["c_hi_dir"]] += wt
    cov = ws > 0
    buf *= np.divide(1.0, ws, out=np.zeros_like(ws), where=cov)[None]
    buf[:, ~cov] = 1.0
    gold = GOLD["A_stitched"]
    assert np.allclose(buf, gold, rtol=1e-6)
    assert not np.array_equal(buf.view(np.uint32), gold.view(np.uint32))


@pytest.mark.parametrize("ups", [int(u) for u in GOLD["pos_ups"]])
def test_layout_matches_shipped_positions(ups, tmp_path):
    """mosaic_layout restates step0's geometry: same header and rows as the
    reference's mosaic_positions{ups}.txt, and read_placements derives the
    same direct and mirror footprints as the reference's parser."""
    meta, rows = mo.mosaic_layout(ups)
    assert [meta[k] for k in META_KEYS] == list(GOLD[f"pos{ups}_meta"])
    want = GOLD[f"pos{ups}_placements"]
    np.testing.assert_array_equal(rows, want[:, :8])
    path = tmp_path / "pos.txt"
    mo.write_positions_file(path, meta, rows)
    meta2, pl = mo.read_placements(path)
    assert meta2 == meta
    np.testing.assert_array_equal(np.array([[p[k] for k in PL_KEYS] for p in pl]), want)


@pytest.mark.parametrize("shape", [(20, 24, 4), (15, 22, 5), (7, 9, 50), (606, 808, 50)])
def test_tent_weight_matches_reference(shape):
    h, w, cap = shape
    want = GOLD[f"tent_{h}_{w}_{cap}"]
    np.testing.assert_array_equal(mo.tent_weight(h, w, cap), want)
    np.testing.assert_array_equal(om.tent_weight(h, w, cap), want)
    assert want.dtype == np.float32 and want.min() > 0


@pytest.mark.parametrize("name", ["A", "B"])
def test_angle_arrays(name):
    t = mo.tile_theta(GOLD[f"{name}_theta"])
    np.testing.assert_array_equal(t, GOLD[f"{name}_tile_theta"])
    nh = int(GOLD[f"{name}_meta"][7])
    np.testing.assert_array_equal(mo.stitched_theta(t, nh), GOLD[f"{name}_stitched_theta"])


def test_read_placements_rejects_missing_header(tmp_path):
    p = tmp_path / "bad.txt"
    p.write_text("# NZ=10 N=10 DET_H=4 DET_W=4\n0 0 2 2 0 0 0 0\n")
    with pytest.raises(ValueError, match="missing header keys"):
        mo.read_placements(p)
