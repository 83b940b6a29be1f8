"""StreamedForward (host-to-host R -> psi -> D -> |.|^2 with overlapped copies):
every submitted volume's intensities equal those of the same operators called
one by one on the device, with buffers reused across steps."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
WL, VOX, DIST = 4.133e-11, 0.69e-6, 0.12


def test_streamed_forward_matches_direct_calls():
    from model_mosaic_b200.phantom import ellipsoid_volume
    from model_mosaic_b200.pipeline import StreamedForward
    from model_mosaic_b200.processing.propagation import Propagation
    from model_mosaic_b200.processing.tomo import TomoReal
    n, nz, T = 128, 16, 90
    theta = np.linspace(0, 2 * np.pi, T, endpoint=False).astype(np.float32)
    s, ib = 0.8, 0.01
    fwd = StreamedForward(n, nz, theta, WL, VOX, DIST, s, ib)
    vols = [torch.from_numpy(ellipsoid_volume(n, nz, seed=k)).pin_memory() for k in range(3)]
    outs = [fwd.pinned_intensity() for _ in range(3)]
    for v, o in zip(vols, outs):
        fwd.submit(v, o)
    fwd.synchronize()
    tomo = TomoReal(n, nz, theta)
    prop = Propagation(n, nz, T, 1, WL, VOX, [DIST])
    for v, o in zip(vols, outs):
        ref = prop.intensity(tomo.R(v.cuda()), s, ib, 0).cpu()
        assert torch.equal(o, ref)
    with pytest.raises(ValueError):
        fwd.submit(vols[0][:4], outs[0])
    fwd.free()
