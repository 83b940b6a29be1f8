"""Array carriers for the operators: torch CUDA tensors inside, and whatever
the caller passed outside.

The reference's GPU classes take and return cupy device arrays
(processing/tomo.py:121-188, processing/propagation.py:47-64).  Here a
call accepts a torch CUDA tensor, any object exposing
``__cuda_array_interface__`` (cupy, numba, ...) or a host numpy array, and
returns the same kind: torch -> torch, cupy -> cupy (zero-copy view of the
torch result), numpy -> numpy.
"""
from __future__ import annotations

import numpy as np
import torch

KIND_TORCH, KIND_CAI, KIND_NUMPY = "torch", "cai", "numpy"


def require_cuda() -> None:
    if not torch.cuda.is_available():
        raise RuntimeError("model_mosaic_b200 operators need a CUDA device (B200, sm_100a); none is visible")


def to_device(x, dtype: torch.dtype):
    """(contiguous CUDA tensor of `dtype`, kind of the original)."""
    if isinstance(x, torch.Tensor):
        kind = KIND_TORCH
        t = x
    elif hasattr(x, "__cuda_array_interface__"):
        kind = KIND_CAI
        t = torch.as_tensor(x, device="cuda")
    else:
        kind = KIND_NUMPY
        t = torch.from_numpy(np.ascontiguousarray(x))
    if not t.is_cuda:
        t = t.to("cuda", non_blocking=False)
    if t.dtype != dtype:
        if dtype == torch.complex64 and not t.is_complex():
            t = t.to(torch.float32).to(torch.complex64)
        else:
            t = t.to(dtype)
    return t.contiguous(), kind


def from_device(t: torch.Tensor, kind: str):
    if kind == KIND_TORCH:
        return t
    if kind == KIND_CAI:
        try:
            import cupy  # noqa: F401  (only when the caller itself uses cupy)
            return cupy.asarray(t)
        except ImportError:
            return t
    return t.cpu().numpy()


def stream_ptr(device=None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def dtype_of(x):
    """numpy-style dtype of a torch tensor / array-like."""
    if isinstance(x, torch.Tensor):
        return {torch.float32: np.dtype("float32"), torch.complex64: np.dtype("complex64"),
                torch.float64: np.dtype("float64"), torch.complex128: np.dtype("complex128")}.get(
                    x.dtype, np.dtype("float32"))
    if hasattr(x, "dtype"):
        return np.dtype(str(x.dtype))
    return np.asarray(x).dtype


def is_complex(x) -> bool:
    return np.issubdtype(dtype_of(x), np.complexfloating)


def pinned_empty(shape, dtype):
    """Pinned host numpy array (the reference allocates its large host
    buffers pinned, processing/pipeline.py:54-59)."""
    tdt = {np.dtype("float32"): torch.float32, np.dtype("complex64"): torch.complex64}[np.dtype(dtype)]
    try:
        return torch.empty(tuple(shape), dtype=tdt, pin_memory=True).numpy()
    except RuntimeError:
        return np.empty(shape, dtype=dtype)
