"""Golden fixtures of the reference's Paganin retrieval (processing/paganin.py).

The reference class uses cupy's array API and cupyx.scipy.fft (rfft2, irfft2,
get_fft_plan).  Neither is installed here, so this script imports the
reference module unchanged with NumPy registered as ``cupy`` and NumPy's FFT
as ``cupyx.scipy.fft`` (plans become no-op context managers), and records the
reference's own outputs on the shapes of its test (tests/test_large_variants.py:
227-259: n = 64, nz = 32, three frames, intensities 0.5 + 0.5 U[0, 1), seed 0,
distances 0.02, 0.1, 1 m) plus a 2-D call and a batch smaller than ntheta.

Run from the repository root with the reference tree present:

    python tests/golden/make_golden_paganin.py [path/to/reference]
"""
from __future__ import annotations

import contextlib
import os
import sys
import types

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"


def load_reference_paganin():
    cp = types.ModuleType("cupy")
    cp.__dict__.update({k: getattr(np, k) for k in dir(np) if not k.startswith("__")})
    cp.ndarray = np.ndarray
    cpx = types.ModuleType("cupyx")
    cpx_scipy = types.ModuleType("cupyx.scipy")
    fft = types.ModuleType("cupyx.scipy.fft")
    fft.rfft2 = lambda a, s=None, axes=(-2, -1): np.fft.rfft2(a, s=s, axes=axes)
    fft.irfft2 = lambda a, s=None, axes=(-2, -1): np.fft.irfft2(a, s=s, axes=axes)
    fft.get_fft_plan = lambda *a, **k: contextlib.nullcontext()
    cpx.scipy = cpx_scipy
    cpx_scipy.fft = fft
    sys.modules.update({"cupy": cp, "cupyx": cpx, "cupyx.scipy": cpx_scipy, "cupyx.scipy.fft": fft})
    sys.path.insert(0, REF)
    from processing.paganin import Paganin  # the reference's class, run on NumPy arrays
    return Paganin


def main():
    Paganin = load_reference_paganin()
    n, nz, ntheta = 64, 32, 3
    wavelength, voxelsize, alpha = 4.13e-11, 1.4e-6, 1e-3
    np.random.seed(0)
    inten = (0.5 + 0.5 * np.random.rand(ntheta, nz, n)).astype(np.float32)
    out = {"intensity": inten}
    for L in (0.02, 0.1, 1.0):
        p = Paganin(n, nz, ntheta, wavelength, voxelsize, L, alpha)
        out[f"filt_L{L}"] = np.asarray(p.filt)
        out[f"phase_L{L}"] = np.asarray(p.retrieve(inten.copy()))
    p = Paganin(n, nz, ntheta, wavelength, voxelsize, 0.1, alpha)
    out["phase2d_L0.1"] = np.asarray(p.retrieve(inten[1].copy()))        # (nz, n) input
    out["phase_b2_L0.1"] = np.asarray(p.retrieve(inten[:2].copy()))      # batch < ntheta
    np.savez_compressed(os.path.join(OUT, "paganin.npz"), **out)
    print("wrote", os.path.join(OUT, "paganin.npz"), len(out), "arrays")


if __name__ == "__main__":
    main()
