"""Autotuner for batches of uneven mosaic tiles (R, psi -> D -> |.|^2, RT).

For every tile size n of a batch it picks the USFFT accuracy pair (eps, m)
and for the whole batch the number of worker streams of its CUDA graph:

* (eps, m) candidates are the reference's own formula (processing/tomo.py:
  39-42, m = ceil(2n/pi sqrt(-mu ln eps + (mu n)^2/4)), mu = -ln eps/(2n^2))
  at three accuracies: eps = 1e-2 -> m = 3, eps = 1e-3 -> m = 4 (the
  reference's default), eps = 1e-5 -> m = 6.  Each candidate's method error
  is estimated on the GPU: the relative L2 difference of R of a seeded
  ellipsoid slice against R at eps = 1e-5, m = 6, whose own error (~1e-5) is
  far below the candidates'.  Among the candidates whose error is at most
  ``tol`` (default: the error of the reference's setting measured the same
  way, so the default never loses accuracy against the reference), the one
  with the shortest tile step (R + intensity + RT at the class's median angle
  count, CUDA events) wins.
* streams: the batch is captured with each stream count in ``streams`` and
  the fastest graph replay wins.

The grid oversampling stays 2 (the reference's 2n padded spectrum); the
half-width m is the accuracy/speed knob.  Results are cached in a JSON file
keyed by the device name, the tile class (n, nz, angle count) and the
tolerance; a batch's stream count by its tile list.
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np
import torch

from model_mosaic_b200._interop import require_cuda

CANDIDATES = ((1e-2, 3), (1e-3, 4), (1e-5, 6))
REFERENCE = (1e-3, 4)
TRUTH = (1e-5, 6)
DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "model_mosaic_b200", "autotune.json")


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save(path, data):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _label(c) -> str:
    return f"eps={c[0]:g},m={c[1]}"


def _dev(device) -> torch.device:
    if isinstance(device, torch.device):
        return device
    return torch.device("cuda", torch.cuda.current_device() if device is None else int(device))


def _device_name(device) -> str:
    return torch.cuda.get_device_name(device)


def estimate_errors(n: int, device=None, ntheta: int = 64, seed: int = 0, candidates=CANDIDATES) -> dict:
    """{(eps, m): relative L2 of R against R at (1e-5, 6)} on one seeded
    ellipsoid slice of n^2 over ``ntheta`` angles on [0, pi)."""
    from model_mosaic_b200.phantom import ellipsoid_volume_torch
    from model_mosaic_b200.processing.tomo import TomoReal
    require_cuda()
    dev = _dev(device)
    theta = np.linspace(0, np.pi, ntheta, endpoint=False).astype(np.float32)
    with torch.cuda.device(dev):
        x = ellipsoid_volume_torch(n, 1, seed=seed, device=dev)
        ref_tomo = TomoReal(n, 1, theta, eps=TRUTH[0], m=TRUTH[1])
        ref = ref_tomo.R(x).double()
        ref_tomo.free()
        out = {}
        for eps, m in candidates:
            t = TomoReal(n, 1, theta, eps=eps, m=m)
            r = t.R(x).double()
            t.free()
            out[(eps, m)] = float(torch.linalg.vector_norm(r - ref) / torch.linalg.vector_norm(ref))
    return out


def _time_tile(n, nz, ntheta, eps, m, wavelength, voxelsize, distance, device, warmup=2, steps=3) -> float:
    from model_mosaic_b200.phantom import ellipsoid_volume_torch
    from model_mosaic_b200.tiles import _Tile
    theta = np.linspace(0, np.pi, ntheta, endpoint=False).astype(np.float32)
    tile = _Tile(n, nz, theta, wavelength, voxelsize, distance, None, 0.01, device, eps=eps, m=m)
    try:
        tile.obj.copy_(ellipsoid_volume_torch(n, nz, seed=1, device=device))
        st = torch.cuda.current_stream(device)
        for _ in range(warmup):
            tile.step()
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            tile.step()
        e1.record(st)
        torch.cuda.synchronize(device)
        return e0.elapsed_time(e1) / steps
    finally:
        tile.free()


def tune_classes(specs, wavelength, voxelsize, distance, *, tol=None, device=None, cache=DEFAULT_CACHE,
                 candidates=CANDIDATES) -> dict:
    """{n: (eps, m)} for the tile sizes of ``specs`` (dicts with n, theta, nz),
    plus a report {n: {"errors", "ms", "choice", "ntheta", "nz"}}."""
    require_cuda()
    dev = _dev(device)
    store = _load(cache) if cache else {}
    dname = _device_name(dev)
    classes = {}
    for t in specs:
        classes.setdefault(int(t["n"]), []).append((len(t["theta"]), int(t.get("nz", 16))))
    params, report = {}, {}
    with torch.cuda.device(dev):
        for n, members in sorted(classes.items()):
            T = int(np.median([a for a, _ in members]))
            nz = max(z for _, z in members)
            errs = estimate_errors(n, dev, candidates=candidates)
            lim, ok = admissible(errs, tol, candidates)
            key = f"{dname}|n={n}|nz={nz}|T={T}|tol={'ref' if tol is None else f'{tol:.3g}'}"
            hit = store.get(key)
            if hit and (float(hit["choice"][0]), int(hit["choice"][1])) in ok:
                choice, ms = (float(hit["choice"][0]), int(hit["choice"][1])), dict(hit["ms"])
            else:
                timed = {c: _time_tile(n, nz, T, c[0], c[1], wavelength, voxelsize, distance, dev) for c in ok}
                choice = min(timed, key=timed.get)
                ms = {_label(c): v for c, v in timed.items()}
                store[key] = {"choice": [choice[0], choice[1]], "ms": ms}
            params[n] = choice
            report[n] = {"errors": {_label(c): v for c, v in errs.items()}, "limit": lim, "ms": ms,
                         "choice": choice, "ntheta": T, "nz": nz}
    if cache:
        _save(cache, store)
    return {"params": params, "report": report}


def admissible(errs: dict, tol, candidates=CANDIDATES):
    """(limit, [(eps, m) ...]): the candidates whose estimated error is within
    ``tol`` -- by default the reference setting's own error, so that the
    default never picks a less accurate pair than the reference's."""
    if tol is None:
        lim = errs[REFERENCE] if REFERENCE in errs else np.inf
    else:
        lim = float(tol)
    return lim, [(float(e), int(m)) for e, m in candidates if errs[(e, m)] <= lim * (1 + 1e-6)]


def batch_signature(specs) -> str:
    h = hashlib.sha1()
    for t in specs:
        h.update(f"{int(t['n'])}:{len(t['theta'])}:{int(t.get('nz', 16))};".encode())
    return h.hexdigest()[:16]


def tune_streams(batch, specs, choices=(2, 4, 8), *, cache=DEFAULT_CACHE, warmup=2, steps=3) -> dict:
    """Capture ``batch`` (a TileBatch) with each stream count, keep the
    fastest; returns {"streams": k, "ms": {k: ms}} and leaves the batch
    captured with the winner."""
    store = _load(cache) if cache else {}
    key = f"{_device_name(batch.device)}|batch={batch_signature(specs)}|params=" + \
          ",".join(f"{t.n}:{t.eps:g}:{t.m}" for t in batch.tiles)
    hit = store.get(key)
    ms = {}
    if hit and int(hit["streams"]) in choices:
        best = int(hit["streams"])
        ms = {int(k): v for k, v in hit["ms"].items()}
    else:
        st = torch.cuda.current_stream(batch.device)
        for k in choices:
            batch.set_streams(k)
            batch.capture()
            for _ in range(warmup):
                batch.run()
            torch.cuda.synchronize(batch.device)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(steps):
                batch.run()
            e1.record(st)
            torch.cuda.synchronize(batch.device)
            ms[k] = e0.elapsed_time(e1) / steps
        best = min(ms, key=ms.get)
        store[key] = {"streams": best, "ms": {str(k): v for k, v in ms.items()}}
        if cache:
            _save(cache, store)
    batch.set_streams(best)
    batch.capture()
    return {"streams": best, "ms": ms}


def autotuned_batch(specs, wavelength, voxelsize, distance, *, tol=None, streams=(2, 4, 8), cache=DEFAULT_CACHE,
                    device=None, beta_ratio=100.0, fill=None):
    """Tune (eps, m) per tile size, build the TileBatch with them, fill the
    objects (``fill(batch)``, optional) and tune and capture the stream count.
    Returns (batch, report)."""
    from model_mosaic_b200.tiles import TileBatch
    cls = tune_classes(specs, wavelength, voxelsize, distance, tol=tol, device=device, cache=cache)
    batch = TileBatch(specs, wavelength, voxelsize, distance, beta_ratio=beta_ratio, device=device,
                      params=cls["params"])
    if fill is not None:
        fill(batch)
    st = tune_streams(batch, specs, streams, cache=cache)
    return batch, {"classes": cls["report"], "streams": st}
