"""Host-side fault injection: device allocations that fail on request.

The library's allocation hook (MM_FAIL_ALLOC_AFTER=k: the (k+1)-th device
allocation made by the library in this process reports MM_ENOMEM without
calling cudaMalloc) stands in for an out-of-memory GPU; no GPU fault is
involved.  Each case runs in a fresh child process, because the hook counts
allocations per process.  Checked: a create that fails frees what it took
and raises MemoryError; the next create succeeds; a failure inside a live
handle's lazy work (the adjoint's scatter table, the D handle's buffers)
leaves the handle usable, and its results still match the FP64 oracle."""
import os
import subprocess
import sys
import textwrap

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent("""
    import os, numpy as np, torch
    from model_mosaic_b200.processing.tomo import TomoReal
    from model_mosaic_b200.processing.propagation import Propagation
    from oracle.usfft import TomoRealOracle
    from oracle.fresnel import PropagationOracle

    def rl2(a, b):
        a = np.asarray(a, np.complex128 if np.iscomplexobj(a) else np.float64)
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    n, nz, T = 64, 4, 30
    theta = np.linspace(0, np.pi, T, endpoint=False).astype(np.float32)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((nz, n, n)).astype(np.float32)
    y = rng.standard_normal((T, nz, n)).astype(np.float32)
    o = TomoRealOracle(n, nz, theta)
    free0 = torch.cuda.mem_get_info()[0]

    os.environ["MM_FAIL_ALLOC_AFTER"] = "3"          # the 4th allocation of create fails
    try:
        TomoReal(n, nz, theta)
        raise SystemExit("create did not fail")
    except MemoryError as e:
        assert "injected allocation failure" in str(e), e
    del os.environ["MM_FAIL_ALLOC_AFTER"]
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] >= free0 - (8 << 20)   # the failed create released its buffers

    tomo = TomoReal(n, nz, theta)                      # the next create succeeds
    assert rl2(tomo.R(x), o.R(x)) < 1e-5
    os.environ["MM_FAIL_ALLOC_AFTER"] = "0"          # the lazy scatter-table build fails
    try:
        tomo.RT(y)
        raise SystemExit("RT did not fail")
    except MemoryError as e:
        assert "injected" in str(e), e
    del os.environ["MM_FAIL_ALLOC_AFTER"]
    assert rl2(tomo.R(x), o.R(x)) < 1e-5               # the handle still works
    assert rl2(tomo.RT(y), o.RT(y)) < 1e-5             # and builds its table on the next call
    tomo.free()

    os.environ["MM_FAIL_ALLOC_AFTER"] = "0"
    try:
        Propagation(n, 16, 2, 1, 4.133e-11, 0.69e-6, [0.12])
        raise SystemExit("Propagation create did not fail")
    except MemoryError:
        pass
    del os.environ["MM_FAIL_ALLOC_AFTER"]
    prop = Propagation(n, 16, 2, 1, 4.133e-11, 0.69e-6, [0.12])
    psi = (rng.standard_normal((2, 16, n)) + 1j * rng.standard_normal((2, 16, n))).astype(np.complex64)
    ref = PropagationOracle(n, 16, 2, 1, 4.133e-11, 0.69e-6, [0.12]).D(psi, 0)
    assert rl2(prop.D(psi, 0), ref) < 1e-5
    print("FAULTS_OK")
""")


def test_allocation_failures_leave_library_usable():
    env = dict(os.environ)
    env.pop("MM_FAIL_ALLOC_AFTER", None)
    env["PYTHONPATH"] = ROOT + os.pathsep + env.get("PYTHONPATH", "")
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0 and "FAULTS_OK" in r.stdout, r.stdout[-2000:] + r.stderr[-4000:]
