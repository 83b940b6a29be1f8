"""Golden fixtures of the reference's FBP filter (processing/fbp_filter.py).

The reference class is written against cupy's array API only (arange, sinc,
linalg.inv, fft.rfft/irfft, ...).  cupy is not installed here, so this script
imports the reference module unchanged with NumPy registered under the name
``cupy`` and records, from the reference's own code:

* ``calc_filter(name)`` for all eight filters at n = 16, 64 and 100 (the
  12-point quadrature tapers its last 40 weights only when ne/2 + 1 > 40);
* ``filter(sino, w)`` of seeded sinograms (n = 64, ramp and shepp; n = 100,
  hann; batch chunks smaller than the batch), float32 as in step8_fbp.py.

Run from the repository root with the reference tree present:

    python tests/golden/make_golden_fbp.py [path/to/reference]
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"

FILTERS = ["none", "ramp", "shepp", "cosine", "cosine2", "hamming", "hann", "parzen"]


def load_reference_fbp():
    shim = types.ModuleType("cupy")
    shim.__dict__.update({k: getattr(np, k) for k in dir(np) if not k.startswith("__")})
    shim.ndarray = np.ndarray
    sys.modules["cupy"] = shim
    sys.path.insert(0, REF)
    from processing.fbp_filter import FBPFilter  # the reference's class, run on NumPy arrays
    return FBPFilter


def main():
    FBPFilter = load_reference_fbp()
    out = {}
    for n in (16, 64, 100):
        f = FBPFilter(n)
        for name in FILTERS:
            out[f"w_{name}_n{n}"] = np.asarray(f.calc_filter(name))
    rng = np.random.default_rng(8)
    cases = [(64, "ramp", (6, 5), 7), (64, "shepp", (3, 4), 256), (100, "hann", (2, 9), 5)]
    for n, name, lead, chunk in cases:
        f = FBPFilter(n, batch_chunk=chunk)
        sino = rng.standard_normal(lead + (n,)).astype(np.float32)
        out[f"sino_{name}_n{n}"] = sino.copy()
        out[f"filt_{name}_n{n}"] = np.asarray(f.filter(sino, f.calc_filter(name)))
    np.savez_compressed(os.path.join(OUT, "fbp_filter.npz"), **out)
    print("wrote", os.path.join(OUT, "fbp_filter.npz"), len(out), "arrays")


if __name__ == "__main__":
    main()
