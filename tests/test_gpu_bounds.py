"""Caller-array checks (mm_set_bounds_check / MM_BOUNDS_CHECK=1): with the
switch on, an array too short for the call, pageable host memory or a
pointer outside any allocation is refused with ValueError before anything is
launched, and the handle stays usable.  Every refused case is first shown to
be caught by mm_check_array on the same pointer and size, so no call below
can reach a kernel with a short buffer."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture
def checks_on():
    from model_mosaic_b200 import _ffi
    _ffi.set_bounds_check(True)
    assert _ffi.bounds_check()
    yield _ffi
    _ffi.set_bounds_check(False)


def _refused(_ffi, ptr, nbytes):
    return _ffi.lib().mm_check_array(C.c_void_p(ptr), nbytes) == _ffi.MM_EINVAL


def test_short_output_refused_then_handle_usable(checks_on):
    _ffi = checks_on
    from model_mosaic_b200.processing.tomo import TomoReal
    n, nz, T = 128, 4, 64
    theta = np.linspace(0, np.pi, T, endpoint=False).astype(np.float32)
    tomo = TomoReal(n, nz, theta)
    obj = torch.rand((nz, n, n), device="cuda")
    # one 64 MiB block; the output pointer sits 8 KiB before its end, far
    # short of the T * nz * n * 4 = 131 KiB that R writes
    block = torch.empty(64 * 2 ** 20 // 4, device="cuda")
    ptr = block.data_ptr() + block.numel() * 4 - 8192
    need = T * nz * n * 4
    base_ok = _ffi.lib().mm_check_array(C.c_void_p(block.data_ptr()), block.numel() * 4) == _ffi.MM_OK
    if not base_ok or not _refused(_ffi, ptr, need):
        pytest.skip("the allocation range of this pointer cannot be queried here")
    rc = _ffi.lib().mm_tomo_R(tomo._handle(), C.c_void_p(obj.data_ptr()), C.c_void_p(ptr), nz, None)
    assert rc == _ffi.MM_EINVAL and "sino" in _ffi.last_error()
    # the handle still works, and with the checks on results are unchanged
    sino = tomo.R(obj)
    _ffi.set_bounds_check(False)
    assert torch.equal(sino, tomo.R(obj))


def test_host_memory_refused(checks_on):
    _ffi = checks_on
    from model_mosaic_b200.processing.propagation import Propagation
    n, nz, nt = 64, 32, 2
    host = np.zeros((nt, nz, n), np.complex64)
    if not _refused(_ffi, host.ctypes.data, host.nbytes):
        pytest.skip("pageable host memory is device-accessible here")
    prop = Propagation(n, nz, nt, 1, 4.133e-11, 0.69e-6, [0.12])
    out = torch.empty((nt, nz, n), dtype=torch.complex64, device="cuda")
    rc = _ffi.lib().mm_prop_D(prop._handle(), C.c_void_p(host.ctypes.data), C.c_void_p(out.data_ptr()), nt, 0, None)
    assert rc == _ffi.MM_EINVAL and "input" in _ffi.last_error()
    psi = torch.ones((nt, nz, n), dtype=torch.complex64, device="cuda")
    assert torch.isfinite(torch.view_as_real(prop.D(psi, 0))).all()


def test_unknown_pointer_refused(checks_on):
    _ffi = checks_on
    assert _refused(_ffi, 0x10, 4096)            # no allocation there
    x = torch.zeros(1024, device="cuda")
    assert _ffi.lib().mm_check_array(C.c_void_p(x.data_ptr()), 4096) == _ffi.MM_OK


def test_environment_switch():
    code = ("from model_mosaic_b200 import _ffi; import sys; "
            "sys.exit(0 if _ffi.bounds_check() else 1)")
    env = dict(os.environ, MM_BOUNDS_CHECK="1")
    assert subprocess.run([sys.executable, "-c", code], env=env, cwd=os.path.dirname(os.path.dirname(
        os.path.abspath(__file__)))).returncode == 0
    env["MM_BOUNDS_CHECK"] = "0"
    assert subprocess.run([sys.executable, "-c", code], env=env, cwd=os.path.dirname(os.path.dirname(
        os.path.abspath(__file__)))).returncode == 1
