"""Multi-process sharding logic on CPU ranks (gloo, world size 2): every sample
is owned by exactly one rank, and an all-gather of per-rank partial outputs
reassembles the full grid."""
import os
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    sys.path.insert(0, os.path.join(ROOT, "partia.jl_b200"))
    from partia_b200.sharding import grid_slab
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    nx, ny, nz = 5, 4, 7
    (z0, z1), (lo, hi) = grid_slab(nx, ny, nz, rank, world)
    # each rank "interpolates" its samples: value = linear sample index
    part = torch.arange(lo, hi, dtype=torch.float64)
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([hi - lo]))
    maxn = int(max(s.item() for s in sizes))
    buf = torch.full((maxn,), -1.0, dtype=torch.float64)
    buf[: hi - lo] = part
    bufs = [torch.empty(maxn, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(bufs, buf)
    full = torch.cat([b[: int(s.item())] for b, s in zip(bufs, sizes)])
    if rank == 0:
        q.put((full.numpy().tolist(), [int(s.item()) for s in sizes]))
    dist.barrier()
    dist.destroy_process_group()


def test_grid_slabs_partition_the_samples():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    full, sizes = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sum(sizes) == 5 * 4 * 7
    assert full == list(range(5 * 4 * 7))


def test_slab_bounds():
    from partia_b200.sharding import slab
    for n in (0, 1, 7, 128):
        for w in (1, 2, 3, 8):
            spans = [slab(n, r, w) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
    with pytest.raises(ValueError):
        slab(4, 2, 2)
