"""The C-ABI library loads without a GPU and exports every entry point that
include/mosaic.h declares (no compute calls)."""
import ctypes
import os
import re

from model_mosaic_b200 import _ffi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    import glob
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(mm_[A-Za-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_all_declared_symbols():
    L = ctypes.CDLL(_ffi.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 13
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_error_text_without_gpu():
    L = _ffi.lib()
    assert L.mm_version() >= 1
    # argument validation happens before any CUDA call
    h = ctypes.c_void_p()
    theta = (ctypes.c_float * 4)(0, 1, 2, 3)
    rc = L.mm_tomo_create(7, 1, 4, ctypes.cast(theta, ctypes.c_void_p), None, ctypes.byref(h))
    assert rc == _ffi.MM_EINVAL and "even" in _ffi.last_error()
    rc = L.mm_prop_create(24, 8, 1, 1, 1e-10, 1e-6, None, ctypes.byref(h))
    assert rc == _ffi.MM_EINVAL
    assert L.mm_tomo_R(None, None, None, 1, None) == _ffi.MM_EINVAL
    assert "NULL handle" in _ffi.last_error()
