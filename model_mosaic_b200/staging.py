"""Chunked host <-> device streaming for the host-array operator classes.

The reference's ``*Large`` classes move their host arrays through pinned
buffers on three private streams so that copies overlap compute
(processing/pipeline.py:255-359).  ``ChunkStream`` does the same for any
operator applied chunk by chunk: chunk i is copied in on one stream, computed
on a second and copied out on a third, with two device buffers and two pinned
host staging buffers per side (one of each for a single chunk), so the
copy-in of chunk i+1, the compute of chunk i and the copy-out of chunk i-1
run at the same time.  The host thread
fills the pinned input staging buffer of chunk i+1 (a plain memcpy, also for
strided or pageable inputs) and empties the output staging buffer of chunk
i-1 while the GPU works.

    cs = ChunkStream(device)
    cs.run(keys, in_shape, in_dtype, out_shape, out_dtype, load, compute, store)

``load(key, dst)`` fills the pinned numpy array ``dst`` with the chunk's
input; ``compute(key, x, y)`` enqueues the device work on the current stream
(x and y are contiguous CUDA tensors of the chunk's shapes); ``store(key,
src)`` consumes the pinned numpy array ``src`` holding the chunk's output.
``in_shape(key)`` and ``out_shape(key)`` give each chunk's shapes.
"""
from __future__ import annotations

import numpy as np
import torch

_TDT = {np.dtype("float32"): torch.float32, np.dtype("complex64"): torch.complex64}


def _pinned(numel: int, dtype) -> torch.Tensor:
    t = torch.empty(max(1, numel), dtype=_TDT[np.dtype(dtype)])
    try:
        return t.pin_memory()
    except RuntimeError:
        return t


def _view(flat: torch.Tensor, shape) -> torch.Tensor:
    return flat[:int(np.prod(shape))].view(tuple(shape))


class ChunkStream:
    def __init__(self, device=None):
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        with torch.cuda.device(self.device):
            self.s_in = torch.cuda.Stream(self.device)
            self.s_compute = torch.cuda.Stream(self.device)
            self.s_out = torch.cuda.Stream(self.device)
        self._bufs = {}

    def _buffers(self, tag, numel, dtype, pinned, slots):
        """`slots` buffers (1 for a single chunk, else 2) of at least numel."""
        key = (tag, np.dtype(dtype).str, pinned)
        have = self._bufs.get(key)
        if have is None or have[0].numel() < numel or len(have) < slots:
            have = None
            self._bufs.pop(key, None)
            if pinned:
                have = [_pinned(numel, dtype) for _ in range(slots)]
            else:
                have = [torch.empty(max(1, numel), dtype=_TDT[np.dtype(dtype)], device=self.device)
                        for _ in range(slots)]
            self._bufs[key] = have
        return have

    def run(self, keys, in_shape, in_dtype, out_shape, out_dtype, load, compute, store):
        keys = list(keys)
        if not keys:
            return
        nin = max(int(np.prod(in_shape(k))) for k in keys)
        nout = max(int(np.prod(out_shape(k))) for k in keys)
        slots = 1 if len(keys) == 1 else 2
        hin = self._buffers("hin", nin, in_dtype, True, slots)
        din = self._buffers("din", nin, in_dtype, False, slots)
        dout = self._buffers("dout", nout, out_dtype, False, slots)
        hout = self._buffers("hout", nout, out_dtype, True, slots)
        loaded = [None, None]     # copy-in of the slot done: its pinned input may be refilled
        computed = [None, None]   # compute of the slot done: its device input may be overwritten
        copied = [None, None]     # copy-out of the slot done: its device output may be overwritten
        pending = None            # (key, slot) whose output is still to be stored
        with torch.cuda.device(self.device):
            for i, key in enumerate(keys):
                k = i & 1
                ishape, oshape = in_shape(key), out_shape(key)
                if loaded[k] is not None:
                    loaded[k].synchronize()
                hx = _view(hin[k], ishape)
                load(key, hx.numpy())
                x = _view(din[k], ishape)
                y = _view(dout[k], oshape)
                if computed[k] is not None:
                    self.s_in.wait_event(computed[k])
                with torch.cuda.stream(self.s_in):
                    x.copy_(hx, non_blocking=True)
                    loaded[k] = torch.cuda.Event()
                    loaded[k].record(self.s_in)
                self.s_compute.wait_event(loaded[k])
                if copied[k] is not None:
                    self.s_compute.wait_event(copied[k])
                with torch.cuda.stream(self.s_compute):
                    compute(key, x, y)
                    computed[k] = torch.cuda.Event()
                    computed[k].record(self.s_compute)
                self.s_out.wait_event(computed[k])
                with torch.cuda.stream(self.s_out):
                    _view(hout[k], oshape).copy_(y, non_blocking=True)
                    copied[k] = torch.cuda.Event()
                    copied[k].record(self.s_out)
                if pending is not None:
                    pk, ps = pending
                    copied[ps].synchronize()
                    store(pk, _view(hout[ps], out_shape(pk)).numpy())
                pending = (key, k)
            pk, ps = pending
            copied[ps].synchronize()
            store(pk, _view(hout[ps], out_shape(pk)).numpy())

    def free(self):
        self._bufs = {}
