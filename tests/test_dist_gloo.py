"""Multi-rank path on CPU: two gloo ranks each run the operator (the oracle
stands in for the GPU kernels here) on their own slab of slices; the
gathered slabs must equal the single-process result, and the timing
reduction must return the maximum over ranks."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from model_mosaic_b200.dist import slab, max_over_ranks, gather_slabs


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        from oracle.usfft import TomoRealOracle
        n, nz, T = 32, 7, 12
        theta = np.linspace(0, np.pi, T, endpoint=False).astype(np.float32)
        x = np.random.default_rng(0).standard_normal((nz, n, n))
        a, b = slab(nz, rank, world)
        local = torch.from_numpy(TomoRealOracle(n, b - a, theta).R(x[a:b]))      # (T, nz_r, n)
        full = gather_slabs(local, nz, dim=1)
        t = max_over_ranks(10.0 + rank)
        if rank == 0:
            ref = TomoRealOracle(n, nz, theta).R(x)
            out.put((float(np.abs(full.numpy() - ref).max()), t))
    finally:
        dist.destroy_process_group()


def test_slab_split():
    assert [slab(10, r, 3) for r in range(3)] == [(0, 4), (4, 7), (7, 10)]
    assert [slab(2, r, 4) for r in range(4)] == [(0, 1), (1, 2), (2, 2), (2, 2)]


def test_two_gloo_ranks_match_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    err, t = q.get(timeout=5)
    assert err < 1e-12
    assert t == 11.0
