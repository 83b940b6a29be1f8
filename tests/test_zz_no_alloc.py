"""The allocation-free Fresnel D (mm_prop_D_noalloc) against the handle-based
mm_prop_D and the FP64 oracle, through the C-ABI.

mm_prop_D_noalloc exists for callers that cannot allocate device memory while
they run: a service whose GPU memory is reserved up front by its own pool
allocator sees cudaMalloc fail (or stall other work) once it is running.  Its
working memory is a static device array shared by all calls.  The tests run
calls in a row with different sizes and distances (nothing of one call may
leak into the next), check that a call leaves the device's free memory
unchanged, cover the 2048-wide frames of the production workload, and check
that sizes beyond the array are refused.  This file is collected last on
purpose."""
import ctypes as C

import numpy as np
import pytest
import torch

from model_mosaic_b200 import _ffi

pytestmark = pytest.mark.gpu
RTOL = 1e-5      # relative L2, the tolerance of the other propagator tests


def _lib():
    L = _ffi.lib()
    f = L.mm_prop_D_noalloc
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                  C.c_void_p]
    f.restype = C.c_int
    return L


def _handle_D(n, nz, nt, wl, vs, z, psi):
    L = _lib()
    h = C.c_void_p()
    d = np.array([z], np.float64)
    assert L.mm_prop_create(n, nz, nt, 1, wl, vs, d.ctypes.data_as(C.c_void_p), C.byref(h)) == 0
    out = torch.empty_like(psi)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.mm_prop_D(h, C.c_void_p(psi.data_ptr()), C.c_void_p(out.data_ptr()), nt, 0, stream) == 0
    torch.cuda.synchronize()
    L.mm_prop_destroy(h)
    return out


def _noalloc_into(n, nz, nt, wl, vs, z, psi, out):
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = _lib().mm_prop_D_noalloc(n, nz, nt, wl, vs, z, C.c_void_p(psi.data_ptr()), C.c_void_p(out.data_ptr()),
                                  stream)
    assert rc == 0, _ffi.last_error()
    torch.cuda.synchronize()
    return out


def _noalloc_D(n, nz, nt, wl, vs, z, psi):
    return _noalloc_into(n, nz, nt, wl, vs, z, psi, torch.empty_like(psi))


def _psi(nt, nz, n, seed):
    gen = torch.Generator(device="cpu").manual_seed(seed)
    return torch.complex(torch.randn(nt, nz, n, generator=gen), torch.randn(nt, nz, n, generator=gen)).cuda()


def rl2(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def test_noalloc_matches_handle_D_two_calls():
    cases = [(256, 64, 4, 4.133e-11, 0.69e-6, 0.12), (128, 32, 3, 4.13e-11, 1.4e-6, 0.02)]
    for k, (n, nz, nt, wl, vs, z) in enumerate(cases):
        psi = _psi(nt, nz, n, 11 + k)
        ref = _handle_D(n, nz, nt, wl, vs, z, psi)
        got = _noalloc_D(n, nz, nt, wl, vs, z, psi)
        assert rl2(got, ref) < RTOL


def test_noalloc_production_width_vs_oracle():
    # 2048-wide frames (the production detector rows: the compile-time row
    # kernel), two calls in a row at two distances, against mm_prop_D and the
    # FP64 oracle
    from oracle.fresnel import PropagationOracle
    n, nz, nt, wl, vs = 2048, 64, 4, 4.133e-11, 0.69e-6
    psi = _psi(nt, nz, n, 21)
    for z in (0.12, 0.05):
        got = _noalloc_D(n, nz, nt, wl, vs, z, psi)
        assert rl2(got, _handle_D(n, nz, nt, wl, vs, z, psi)) < RTOL
        ref = PropagationOracle(n, nz, nt, 1, wl, vs, [z]).D(psi.cpu().numpy().astype(np.complex128), 0)
        err = np.linalg.norm(got.cpu().numpy() - ref) / np.linalg.norm(ref)
        assert err < RTOL


def test_noalloc_leaves_free_memory_unchanged():
    # CUDA loads each kernel's code lazily on its first launch, which takes a
    # little device memory: both sizes run once before the measurement.
    a = (256, 64, 4, 4.133e-11, 0.69e-6, 0.12)
    b = (512, 16, 6, 4.133e-11, 1.2e-6, 0.03)
    bufs = {}
    for (n, nz, nt, wl, vs, z), seed in ((a, 31), (b, 32)):
        psi = _psi(nt, nz, n, seed)
        bufs[n] = (psi, torch.empty_like(psi))
        _noalloc_into(n, nz, nt, wl, vs, z, *bufs[n])
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for (n, nz, nt, wl, vs, z) in (a, b, a):
        _noalloc_into(n, nz, nt, wl, vs, z * 1.5, *bufs[n])
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_more_angles_than_one_launch_grid():
    # 70000 frames: the column pass goes in launches of at most 65535 frames
    n, nz, nt, wl, vs, z = 8, 4, 70000, 4.133e-11, 0.69e-6, 0.12
    psi = _psi(nt, nz, n, 41)
    got = _noalloc_D(n, nz, nt, wl, vs, z, psi)
    assert rl2(got, _handle_D(n, nz, nt, wl, vs, z, psi)) < RTOL
    from oracle.fresnel import PropagationOracle
    ref = PropagationOracle(n, nz, 3, 1, wl, vs, [z]).D(psi[-3:].cpu().numpy().astype(np.complex128), 0)
    assert np.linalg.norm(got[-3:].cpu().numpy() - ref) / np.linalg.norm(ref) < RTOL


def test_noalloc_rejects_oversize():
    L = _lib()
    dummy = C.c_void_p(16)
    rc = L.mm_prop_D_noalloc(2048, 2048, 4, 4.1e-11, 1e-6, 0.1, dummy, dummy, None)   # 128 MiB > 64 MiB
    assert rc == _ffi.MM_EINVAL and "static buffer" in _ffi.last_error()
    rc = L.mm_prop_D_noalloc(1536, 64, 1, 4.1e-11, 1e-6, 0.1, dummy, dummy, None)     # not a power of two
    assert rc == _ffi.MM_EINVAL and "power of two" in _ffi.last_error()
