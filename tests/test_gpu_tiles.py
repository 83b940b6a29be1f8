"""TileBatch: uneven tiles (native and cuFFT sizes) through R -> psi -> D ->
|.|^2 -> RT as one CUDA graph over several streams; every output equals the
same tile run on its own, and replays follow new inputs."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
WL, VOX, DIST = 4.133e-11, 0.69e-6, 0.12


def _tiles():
    rng = np.random.default_rng(5)
    out = []
    for n, T in [(64, 37), (48, 24), (32, 40), (40, 21), (64, 30)]:
        theta = np.sort(rng.uniform(0, np.pi, T)).astype(np.float32)
        out.append(dict(n=n, nz=4, theta=theta))
    return out


def _alone(t, obj, s):
    from model_mosaic_b200.processing.propagation import Propagation
    from model_mosaic_b200.processing.tomo import TomoReal
    tomo = TomoReal(t["n"], t["nz"], t["theta"])
    prop = Propagation(t["n"], t["nz"], len(t["theta"]), 1, WL, VOX, [DIST])
    sino = tomo.R(obj)
    return prop.intensity(sino, s, 0.01, 0), tomo.RT(sino)


def test_tile_batch_graph_matches_single_tiles():
    from model_mosaic_b200.tiles import TileBatch
    tiles = _tiles()
    batch = TileBatch(tiles, WL, VOX, DIST, streams=3)
    rng = np.random.default_rng(0)
    for rep in range(2):
        vols = [torch.from_numpy(rng.standard_normal((t["nz"], t["n"], t["n"])).astype(np.float32)).cuda()
                for t in tiles]
        for i, v in enumerate(vols):
            batch.obj(i).copy_(v)
        if rep == 0:
            batch.capture()
        batch.run()
        torch.cuda.synchronize()
        for i, (t, v) in enumerate(zip(tiles, vols)):
            inten, rec = _alone(t, v, batch.tiles[i].inv_norm)
            assert torch.equal(batch.intensity(i), inten), (rep, i)
            assert torch.equal(batch.rec(i), rec), (rep, i)
    assert batch.voxel_angles() == sum(t["nz"] * t["n"] ** 2 * len(t["theta"]) for t in tiles)
    batch.free()
