"""Golden fixtures of the reference's mosaic tile logic (step4_extract.py, step6_stitch.py).

Both scripts do their work inside main() around h5py files, MPI helpers and
the iohdf5 writers; none of h5py, mpi4py or the bank writers run here.  This
script imports the two reference scripts unchanged with small in-memory
stand-ins registered for ``h5py`` (a dict of arrays per file path),
``mpi_utils`` (one rank) and ``iohdf5`` (the stitched vchunks are captured
instead of written), runs their main() on two small mosaics and records:

* the tile scans step4 writes (direct crop, then the h-flipped mirror crop),
* the projection step6 stitches from those tiles after a per-tile gain (so
  overlapping tiles disagree and the tent blend matters), in theta chunks
  whose last one is short,
* read_placements() of every mosaic_positions file the reference ships, and
  _tent_weight() on a few shapes.

Mosaic A: 64 x 64 projection, 3 x 2 tiles of 20 x 24, overlap 4, rows at
the top and bottom no tile covers (filled with 1.0).  Mosaic B: 37 x 50,
4 x 2 tiles of 15 x 22 cropped on all four sides, overlap 5.

Run from the repository root with the reference tree present:

    python tests/golden/make_golden_mosaic.py [path/to/reference]
"""
from __future__ import annotations

import glob
import os
import sys
import tempfile
import types

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(OUT))
REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"

STORE = {}        # absolute path -> root group of a stand-in HDF5 file
WRITTEN = {}      # stitched output path -> {theta offset: array}


class _Dataset:
    def __init__(self, data):
        self.data = np.array(data)
        self.attrs = {}

    @property
    def shape(self):
        return self.data.shape

    def __getitem__(self, key):
        return np.array(self.data[key])


class _Group(dict):
    def _walk(self, path):
        node = self
        for part in [p for p in path.split("/") if p]:
            node = dict.__getitem__(node, part)
        return node

    def __getitem__(self, path):
        return self._walk(path)

    def __contains__(self, path):
        try:
            self._walk(path)
            return True
        except KeyError:
            return False

    def __delitem__(self, path):
        head, _, last = path.rpartition("/")
        dict.__delitem__(self._walk(head) if head else self, last)

    def create_group(self, name):
        g = _Group()
        dict.__setitem__(self, name, g)
        return g

    def create_dataset(self, name, data=None, chunks=None):
        d = _Dataset(data)
        dict.__setitem__(self, name, d)
        return d


class _File:
    def __init__(self, path, mode="r"):
        key = os.path.abspath(path)
        if mode == "w":
            STORE[key] = _Group()
        self.root = STORE[key]

    def __enter__(self):
        return self.root

    def __exit__(self, *exc):
        return False


def install_stand_ins():
    h5py = types.ModuleType("h5py")
    h5py.File = _File
    mpi = types.ModuleType("mpi_utils")
    mpi.RANK, mpi.SIZE, mpi.COMM, mpi.MPI = 0, 1, None, None
    mpi.barrier = lambda *a, **k: None
    mpi.rprint = lambda *a, **k: None
    mpi.report_stage = lambda *a, **k: None
    mpi.banner = lambda *a, **k: None
    mpi.run_main = lambda f: f()
    io = types.ModuleType("iohdf5")
    vch = types.ModuleType("iohdf5.h5_vchunks")
    vch.describe_input = vch.describe_output = lambda *a, **k: None

    def initx_and_bcast(path, shape, dtype, vchunks, **k):
        g = _Group()
        g.create_group("exchange")
        STORE[os.path.abspath(path)] = g
        return dict(path=path, shape=shape, vchunks=vchunks)

    vch.initx_and_bcast = initx_and_bcast
    vch.alloc_shm = lambda vchunks, dtype: (None, np.zeros(vchunks, dtype=dtype))
    vch.free_shm = lambda shm: None
    vch.vchunk_bytes = lambda vchunks, dtype: int(np.prod(vchunks)) * np.dtype(dtype).itemsize
    vch.n_vchunks = lambda shape, vchunks: -(-shape[0] // vchunks[0])
    vch.iter_vchunks = lambda shape, vchunks: [(i, 0, 0) for i in range(-(-shape[0] // vchunks[0]))]
    dx = types.ModuleType("iohdf5.dxchange_hdf5_chunks")

    def tomo_writex(path, data, shm, ivchunk, ctx):
        c0, total = ctx["vchunks"][0], ctx["shape"][0]
        t0 = ivchunk[0] * c0
        WRITTEN.setdefault(path, {})[t0] = np.array(data[:min(c0, total - t0)])

    dx.tomo_writex = tomo_writex
    io.h5_vchunks, io.dxchange_hdf5_chunks = vch, dx
    sys.modules.update({"h5py": h5py, "mpi_utils": mpi, "iohdf5": io, "iohdf5.h5_vchunks": vch,
                        "iohdf5.dxchange_hdf5_chunks": dx})
    sys.path.insert(0, REF)
    import step4_extract
    import step6_stitch
    return step4_extract, step6_stitch


def small_mosaic(nz, n, det_h, det_w, overlap, z_tops, x_origins, n_half):
    from model_mosaic_b200.mosaic import compute_tile_placements
    pl = compute_tile_placements(nz, n, det_h, det_w, 0, x_origins, z_tops)
    rows = [[p["zi"], p["xi"], p["z_center"], p["x_center"], p["crop_top"], p["crop_bottom"], p["crop_left"],
             p["crop_right"]] for p in pl]
    meta = dict(NZ=nz, N=n, DET_H=det_h, DET_W=det_w, n_z=len(z_tops), n_x=len(x_origins),
                NTHETA=2 * n_half, N_HALF=n_half, OVERLAP=overlap)
    return meta, np.asarray(rows, dtype=np.int64)


def run_case(s4, s6, name, meta, rows, chunk, seed, out):
    from model_mosaic_b200.mosaic import write_positions_file
    tmp = tempfile.mkdtemp(prefix=f"mosaic_{name}_")
    ups = 1
    write_positions_file(os.path.join(tmp, f"mosaic_positions{ups}.txt"), meta, rows)
    s4._POSITIONS_DIR = s6._POSITIONS_DIR = tmp
    rng = np.random.default_rng(seed)
    n_half, nz, n = meta["N_HALF"], meta["NZ"], meta["N"]
    data = rng.uniform(0.2, 1.8, (n_half, nz, n)).astype(np.float32)
    theta = np.linspace(0, 180, n_half, endpoint=False).astype(np.float32)
    src = os.path.join(tmp, f"model_big{ups}x", "data.h5")
    os.makedirs(os.path.dirname(src))
    open(src, "w").close()
    with _File(src, "w") as f:
        g = f.create_group("exchange")
        g.create_dataset("data", data=data)
        g.create_dataset("theta", data=theta)
    sys.argv = ["step4_extract.py", "--ups", str(ups), "--path", tmp]
    s4.main()
    tiles, pre = [], []
    os.makedirs(os.path.join(tmp, "mosaic_h5_pre"))
    for k, (zi, xi) in enumerate(rows[:, :2]):
        t = STORE[os.path.abspath(os.path.join(tmp, "mosaic_h5", f"{zi}_{xi}.h5"))]["exchange"]
        tiles.append(np.array(t["data"].data))
        gain = np.float32(1.0 + 0.05 * (k + 1))
        with _File(os.path.join(tmp, "mosaic_h5_pre", f"{zi}_{xi}.h5"), "w") as f:
            g = f.create_group("exchange")
            g.create_dataset("data", data=tiles[-1] * gain)
            g.create_dataset("theta", data=np.array(t["theta"].data))
        pre.append(tiles[-1] * gain)
    tile_theta = np.array(t["theta"].data)
    sys.argv = ["step6_stitch.py", "--ups", str(ups), "--path", tmp, "--nthetachunk", str(chunk)]
    s6.main()
    dst = f"{tmp}/model_big{ups}x/stitched.h5"
    parts = WRITTEN[dst]
    stitched = np.concatenate([parts[k] for k in sorted(parts)])
    out[f"{name}_meta"] = np.array([meta[k] for k in ("NZ", "N", "DET_H", "DET_W", "n_z", "n_x", "NTHETA",
                                                      "N_HALF", "OVERLAP")], dtype=np.int64)
    out[f"{name}_rows"] = rows
    out[f"{name}_chunk"] = np.array(chunk)
    out[f"{name}_data"] = data
    out[f"{name}_theta"] = theta
    out[f"{name}_tile_theta"] = tile_theta
    out[f"{name}_tiles"] = np.concatenate([t.ravel() for t in tiles])
    out[f"{name}_tiles_pre"] = np.concatenate([t.ravel() for t in pre])
    out[f"{name}_stitched"] = stitched
    out[f"{name}_stitched_theta"] = np.array(STORE[os.path.abspath(dst)]["exchange/theta"].data)


def main():
    sys.path.insert(0, ROOT)
    s4, s6 = install_stand_ins()
    out = {}
    meta_a, rows_a = small_mosaic(64, 64, 20, 24, 4, [2, 18, 34], [-4.0, 16.0], 5)
    run_case(s4, s6, "A", meta_a, rows_a, 2, 0, out)
    meta_b, rows_b = small_mosaic(37, 50, 15, 22, 5, [-3, 7, 17, 27], [-5.0, 12.0], 3)
    run_case(s4, s6, "B", meta_b, rows_b, 3, 1, out)
    # read_placements of the shipped positions files (mosaic_positions/*.txt)
    keys = ("zi", "xi", "z_center", "x_center", "crop_top", "crop_bottom", "crop_left", "crop_right",
            "r_lo_dir", "r_hi_dir", "c_lo_dir", "c_hi_dir", "r_lo_mir", "r_hi_mir", "c_lo_mir", "c_hi_mir")
    ups_list = []
    for path in sorted(glob.glob(os.path.join(REF, "mosaic_positions", "mosaic_positions*.txt"))):
        ups = int(os.path.basename(path)[len("mosaic_positions"):-4])
        meta, pl = s4.read_placements(path)
        out[f"pos{ups}_meta"] = np.array([meta[k] for k in ("NZ", "N", "DET_H", "DET_W", "n_z", "n_x", "NTHETA",
                                                           "N_HALF", "OVERLAP")], dtype=np.int64)
        out[f"pos{ups}_placements"] = np.array([[p[k] for k in keys] for p in pl], dtype=np.int64)
        ups_list.append(ups)
    out["pos_ups"] = np.array(sorted(ups_list))
    for h, w, cap in ((20, 24, 4), (15, 22, 5), (7, 9, 50), (606, 808, 50)):
        out[f"tent_{h}_{w}_{cap}"] = s6._tent_weight(h, w, cap)
    np.savez_compressed(os.path.join(OUT, "mosaic.npz"), **out)
    print("wrote", os.path.join(OUT, "mosaic.npz"), sorted(out))


if __name__ == "__main__":
    main()
