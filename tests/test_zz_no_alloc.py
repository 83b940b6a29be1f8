"""The allocation-free Fresnel D (mm_prop_D_noalloc) against the handle-based
mm_prop_D, through the C-ABI.

mm_prop_D_noalloc exists for callers that cannot allocate device memory while
they run (their GPU memory is reserved up front by their own pool allocator);
its working memory is a static device array shared by all calls.  Two calls
in a row with different sizes and distances check that nothing of the first
call leaks into the second.  This file is collected last on purpose."""
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


def _noalloc_D(n, nz, nt, wl, vs, z, psi):
    L = _lib()
    out = torch.empty_like(psi)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.mm_prop_D_noalloc(n, nz, nt, wl, vs, z, C.c_void_p(psi.data_ptr()), C.c_void_p(out.data_ptr()), stream)
    assert rc == 0, _ffi.last_error()
    torch.cuda.synchronize()
    return out


def rl2(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def test_noalloc_matches_handle_D_two_calls():
    gen = torch.Generator(device="cpu").manual_seed(11)
    cases = [(256, 64, 4, 4.133e-11, 0.69e-6, 0.12), (128, 32, 3, 4.13e-11, 1.4e-6, 0.02)]
    for (n, nz, nt, wl, vs, z) in cases:
        psi = torch.complex(torch.randn(nt, nz, n, generator=gen), torch.randn(nt, nz, n, generator=gen)).cuda()
        ref = _handle_D(n, nz, nt, wl, vs, z, psi)
        got = _noalloc_D(n, nz, nt, wl, vs, z, psi)
        assert rl2(got, ref) < RTOL


def test_noalloc_rejects_oversize():
    L = _lib()
    dummy = C.c_void_p(16)
    rc = L.mm_prop_D_noalloc(2048, 2048, 4, 4.1e-11, 1e-6, 0.1, dummy, dummy, None)   # 128 MiB > 64 MiB
    assert rc == _ffi.MM_EINVAL and "static buffer" in _ffi.last_error()
