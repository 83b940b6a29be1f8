"""Mosaic tile extract / stitch on the GPU through the C-ABI, bit-exact against
the reference's outputs (tests/golden/mosaic.npz) and the oracle
(oracle/mosaic.py) on the reference's own mosaic geometry."""
from __future__ import annotations

import os

import numpy as np
import pytest
import torch

from model_mosaic_b200 import mosaic as mo
from oracle import mosaic as om

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "mosaic.npz"))
META_KEYS = ("NZ", "N", "DET_H", "DET_W", "n_z", "n_x", "NTHETA", "N_HALF", "OVERLAP")


def golden_case(name, tmp_path):
    meta = dict(zip(META_KEYS, (int(v) for v in GOLD[f"{name}_meta"])))
    path = tmp_path / f"positions_{name}.txt"
    mo.write_positions_file(path, meta, GOLD[f"{name}_rows"])
    return mo.read_placements(path)


def split_tiles(flat, pl, nframes):
    out, k = [], 0
    for p in pl:
        h, w = p["r_hi_dir"] - p["r_lo_dir"], p["c_hi_dir"] - p["c_lo_dir"]
        out.append(flat[k:k + nframes * h * w].reshape(nframes, h, w))
        k += nframes * h * w
    return out


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("name", ["A", "B"])
def test_extract_matches_reference(name, tmp_path):
    meta, pl = golden_case(name, tmp_path)
    mt = mo.MosaicTiles(meta, pl)
    proj = torch.from_numpy(GOLD[f"{name}_data"]).cuda()
    tiles = mt.extract(proj)
    want = split_tiles(GOLD[f"{name}_tiles"], pl, meta["NTHETA"])
    for g, w in zip(tiles, want):
        np.testing.assert_array_equal(g.cpu().numpy(), w)


@pytest.mark.parametrize("name", ["A", "B"])
def test_stitch_matches_reference_bitwise(name, tmp_path):
    meta, pl = golden_case(name, tmp_path)
    mt = mo.MosaicTiles(meta, pl)
    tiles = [torch.from_numpy(np.ascontiguousarray(t)).cuda()
             for t in split_tiles(GOLD[f"{name}_tiles_pre"], pl, meta["NTHETA"])]
    want = GOLD[f"{name}_stitched"]
    whole = mt.stitch(tiles).cpu().numpy()
    np.testing.assert_array_equal(bits(whole), bits(want))
    chunk, nh = int(GOLD[f"{name}_chunk"]), meta["N_HALF"]
    parts = [mt.stitch(tiles, t0, min(chunk, nh - t0)).cpu().numpy() for t0 in range(0, nh, chunk)]
    np.testing.assert_array_equal(bits(np.concatenate(parts)), bits(want))


@pytest.fixture(scope="module")
def layout1():
    """The reference's mosaic at ups = 1: 3072 x 3072 projection, 11 x 4 tiles
    of 303 x 404, overlap 25 (mosaic_positions1.txt)."""
    meta, rows = mo.mosaic_layout(1)
    import tempfile
    d = tempfile.mkdtemp()
    mo.write_positions_file(os.path.join(d, "p.txt"), meta, rows)
    return mo.read_placements(os.path.join(d, "p.txt"))


def test_full_geometry_extract_and_stitch_bitwise(layout1):
    meta, pl = layout1
    mt = mo.MosaicTiles(meta, pl)
    assert mt.info()[2] <= 4
    nth = 11  # one batch of 8 angles plus 3 more in both kernels
    rng = np.random.default_rng(7)
    data = rng.uniform(0.2, 1.8, (nth, meta["NZ"], meta["N"])).astype(np.float32)
    tiles = mt.extract(torch.from_numpy(data).cuda())
    want_tiles = om.extract(data, pl)
    for g, w in zip(tiles, want_tiles):
        np.testing.assert_array_equal(g.cpu().numpy(), w)
    # corrected tiles disagree in the overlaps: one gain per tile
    gains = (1.0 + 0.01 * np.arange(len(pl))).astype(np.float32)
    pre_np = [w * g for w, g in zip(want_tiles, gains)]
    pre = [torch.from_numpy(t).cuda() for t in pre_np]
    meta3 = dict(meta, N_HALF=nth, NTHETA=2 * nth)
    mt3 = mo.MosaicTiles(meta3, pl)
    got = mt3.stitch(pre).cpu().numpy()
    want = om.stitch(pre_np, pl, meta["NZ"], meta["N"], nth, meta["OVERLAP"], 0, nth)
    np.testing.assert_array_equal(bits(got), bits(want))


def test_round_trip_restores_covered_pixels(layout1):
    meta, pl = layout1
    nth = 2
    meta2 = dict(meta, N_HALF=nth, NTHETA=2 * nth)
    mt = mo.MosaicTiles(meta2, pl)
    x = torch.rand((nth, meta["NZ"], meta["N"]), device="cuda") + 0.5
    y = mt.stitch(mt.extract(x))
    cov = torch.zeros((meta["NZ"], meta["N"]), dtype=torch.bool, device="cuda")
    for p in pl:
        cov[p["r_lo_dir"]:p["r_hi_dir"], p["c_lo_dir"]:p["c_hi_dir"]] = True
        cov[p["r_lo_mir"]:p["r_hi_mir"], p["c_lo_mir"]:p["c_hi_mir"]] = True
    rel = ((y - x).abs() / x)[:, cov].max().item()
    assert rel < 1e-6, rel
    assert torch.all(y[:, ~cov] == 1.0)
    assert torch.equal(y, mt.stitch(mt.extract(x)))  # deterministic


def test_argument_errors(layout1, tmp_path):
    meta, pl = layout1
    bad = [dict(p) for p in pl]
    bad[3]["c_hi_dir"] = meta["N"] + 5
    with pytest.raises(ValueError, match="placement 3"):
        mo.MosaicTiles(meta, bad)
    mt = mo.MosaicTiles(meta, pl)
    tiles = [torch.zeros((2, h, w), device="cuda") for h, w in mt.shapes]
    with pytest.raises(ValueError, match="N_HALF"):
        mt.stitch(tiles, t0=meta["N_HALF"] - 1, nth=2)
    with pytest.raises(ValueError, match="mirror range"):
        mt.stitch(tiles, t0=0, nth=1)
    proj = torch.zeros((1, meta["NZ"], meta["N"] - 1), device="cuda")
    with pytest.raises(ValueError, match="shape"):
        mt.extract(proj)
    # zero angles is a no-op
    mt.extract_into(torch.zeros((0, meta["NZ"], meta["N"]), device="cuda"),
                    [torch.zeros((0, h, w), device="cuda") for h, w in mt.shapes],
                    [torch.zeros((0, h, w), device="cuda") for h, w in mt.shapes])
