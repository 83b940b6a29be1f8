"""Rank helpers for running the hot path on several GPUs of one node.

The path shards without any data exchange: R/RT are independent per slice
(the reference shards z-slabs per MPI rank, step2_radon.py:150-151,
step8_fbp.py:167-168) and D per angle (step3_propagation.py:188-189).  One
process per GPU owns a contiguous slab; ranks only meet to agree on timings
(max over ranks) or, when a caller wants the whole result on one rank, to
gather the slabs.  Works with the ``nccl`` (CUDA tensors) and ``gloo`` (CPU
tensors) backends of torch.distributed.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def slab(total: int, rank: int, world: int):
    """Contiguous [start, stop) share of `total` items for `rank` (sizes differ by <= 1)."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _device():
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(value: float) -> float:
    """Max of a scalar over all ranks (identity without a process group)."""
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_slabs(local: torch.Tensor, total: int, dim: int):
    """Concatenate every rank's slab along `dim` on all ranks (slab sizes as in
    `slab`).  Returns `local` itself without a process group."""
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return local
    world = dist.get_world_size()
    dev = _device()
    sizes = [slab(total, r, world)[1] - slab(total, r, world)[0] for r in range(world)]
    big = max(sizes)
    shape = list(local.shape)
    shape[dim] = big
    padded = torch.zeros(shape, dtype=local.dtype, device=dev)     # all_gather wants equal sizes
    padded.narrow(dim, 0, local.shape[dim]).copy_(local)
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded)
    return torch.cat([p.narrow(dim, 0, sz) for p, sz in zip(parts, sizes)], dim=dim)
