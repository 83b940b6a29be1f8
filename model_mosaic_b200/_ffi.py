"""ctypes binding of the C-ABI in include/mosaic.h (``libmosaic.so``).

The shared library is built in-tree by ``model_mosaic_b200/build.py``.  There
is no fallback: if the library is missing or fails to load, every operator
raises at construction time.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmosaic.so")

MM_OK, MM_EINVAL, MM_ENOMEM, MM_ECUDA, MM_ECUFFT, MM_ETIMEOUT = 0, -1, -2, -3, -4, -5
MM_F32, MM_C64, MM_BF16 = 0, 1, 2

_lib = None
_lock = threading.Lock()


class MosaicError(RuntimeError):
    """A C-ABI call returned a CUDA/cuFFT failure status."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"[status {status}] {msg}")
        self.status = status


class MosaicTimeout(MosaicError):
    pass


def _declare(L):
    p, i, f, d, sz = C.c_void_p, C.c_int, C.c_float, C.c_double, C.c_size_t
    L.mm_version.restype = i
    L.mm_last_error.argtypes = [C.c_char_p, sz]
    L.mm_last_error.restype = i
    L.mm_set_bounds_check.argtypes = [i]
    L.mm_set_bounds_check.restype = i
    L.mm_get_bounds_check.restype = i
    L.mm_check_array.argtypes = [p, sz]
    L.mm_check_array.restype = i
    L.mm_tomo_create.argtypes = [i, i, i, p, p, C.POINTER(p)]
    L.mm_tomo_destroy.argtypes = [p]
    L.mm_tomo_R.argtypes = [p, p, p, i, p]
    L.mm_tomo_R_ex.argtypes = [p, p, i, p, i, i, p]
    L.mm_tomo_RT.argtypes = [p, p, i, p, i, p]
    L.mm_tomo_prepare_rt.argtypes = [p, p]
    L.mm_tomo_workspace_bytes.argtypes = [p]
    L.mm_tomo_workspace_bytes.restype = sz
    L.mm_prop_create.argtypes = [i, i, i, i, d, d, p, C.POINTER(p)]
    L.mm_prop_destroy.argtypes = [p]
    L.mm_prop_D.argtypes = [p, p, p, i, i, p]
    L.mm_prop_DT.argtypes = [p, p, p, i, i, p]
    L.mm_prop_intensity.argtypes = [p, p, f, f, p, i, i, p]
    dp, llp = C.POINTER(C.c_double), C.POINTER(C.c_longlong)
    L.mm_tomo_set_timing.argtypes = [p, i]
    L.mm_tomo_get_timing.argtypes = [p, dp, llp, i, llp]
    L.mm_prop_set_timing.argtypes = [p, i]
    L.mm_prop_get_timing.argtypes = [p, dp, llp, i, llp]
    L.mm_prop_grad_partials.argtypes = [p, i]
    L.mm_prop_grad_partials.restype = C.c_long
    L.mm_prop_grad_forward.argtypes = [p, p, p, f, f, p, p, i, i, p]
    L.mm_prop_grad_backward.argtypes = [p, p, p, f, f, p, i, i, p]
    L.mm_prop_D_noalloc.argtypes = [i, i, i, d, d, d, p, p, p]
    L.mm_fbp_create.argtypes = [i, i, C.POINTER(p)]
    L.mm_fbp_destroy.argtypes = [p]
    L.mm_fbp_filter.argtypes = [p, p, C.c_long, p, p]
    L.mm_fbp_workspace_bytes.argtypes = [p]
    L.mm_fbp_workspace_bytes.restype = sz
    L.mm_pgn_create.argtypes = [i, i, i, p, C.POINTER(p)]
    L.mm_pgn_destroy.argtypes = [p]
    L.mm_pgn_retrieve.argtypes = [p, p, p, i, p]
    L.mm_pgn_workspace_bytes.argtypes = [p]
    L.mm_pgn_workspace_bytes.restype = sz
    L.mm_mosaic_create.argtypes = [i, i, i, p, i, C.POINTER(p)]
    L.mm_mosaic_destroy.argtypes = [p]
    L.mm_mosaic_extract.argtypes = [p, p, i, p, p, p]
    L.mm_mosaic_stitch.argtypes = [p, p, p, i, p, p]
    L.mm_mosaic_info.argtypes = [p, C.POINTER(i), C.POINTER(i), C.POINTER(i)]
    L.mm_mosaic_workspace_bytes.argtypes = [p]
    L.mm_mosaic_workspace_bytes.restype = sz
    for name in ("mm_prop_grad_forward", "mm_prop_grad_backward", "mm_prop_D_noalloc",
                 "mm_tomo_set_timing", "mm_tomo_get_timing", "mm_prop_set_timing", "mm_prop_get_timing",
                 "mm_tomo_create", "mm_tomo_destroy", "mm_tomo_R", "mm_tomo_R_ex", "mm_tomo_RT", "mm_tomo_prepare_rt",
                 "mm_prop_create", "mm_prop_destroy", "mm_prop_D", "mm_prop_DT", "mm_prop_intensity",
                 "mm_fbp_create", "mm_fbp_destroy", "mm_fbp_filter",
                 "mm_pgn_create", "mm_pgn_destroy", "mm_pgn_retrieve",
                 "mm_mosaic_create", "mm_mosaic_destroy", "mm_mosaic_extract", "mm_mosaic_stitch",
                 "mm_mosaic_info"):
        getattr(L, name).restype = i
    return L


def lib():
    """Load libmosaic.so once; raise if it is absent (no CPU fallback)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise RuntimeError(
                        f"{LIB_PATH} not found: build it with `python -m model_mosaic_b200.build` "
                        "(the CUDA library is required; there is no CPU path)")
                _lib = _declare(C.CDLL(LIB_PATH))
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().mm_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int, what: str = "") -> None:
    """Turn a C-ABI status into a Python exception (never aborts)."""
    if status == MM_OK:
        return
    msg = last_error() or what
    if status == MM_EINVAL:
        raise ValueError(msg)
    if status == MM_ENOMEM:
        raise MemoryError(msg)
    if status == MM_ETIMEOUT:
        raise MosaicTimeout(status, msg)
    raise MosaicError(status, msg)


TOMO_STAGES = ("pad_phi", "x_r2c", "transpose_in", "y_fft", "gather", "r_c2r", "r_r2c", "scatter",
               "y_ifft", "transpose_out", "x_c2r", "crop_phi", "table_build", "complex_prologue")
PROP_STAGES = ("y_pass", "x_pass")


def read_timing(get, handle, names):
    """{stage: (ms, calls)} and own-kernel launch count from mm_*_get_timing."""
    k = len(names)
    ms = (C.c_double * k)()
    calls = (C.c_longlong * k)()
    kern = C.c_longlong()
    check(get(handle, ms, calls, k, C.byref(kern)))
    return {names[i]: (ms[i], calls[i]) for i in range(k)}, kern.value


def set_bounds_check(on: bool = True) -> None:
    """Process-wide caller-array checks of every compute call (off by
    default): each array must be device memory of the current device holding
    the bytes the call touches; a failure raises ValueError before anything
    is launched.  Also on with the environment variable MM_BOUNDS_CHECK=1."""
    check(lib().mm_set_bounds_check(int(bool(on))), "mm_set_bounds_check")


def bounds_check() -> bool:
    return bool(lib().mm_get_bounds_check())
