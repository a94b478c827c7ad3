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


def _interp_worker(rank, world, port, q):
    sys.path.insert(0, os.path.join(ROOT, "partia.jl_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from partia_b200.sharding import allreduce_gradients, shard_samples
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    O.set_threads(2)
    P, cols, s, gout_all = _clustered_case()
    orc = O.Oracle(*P, cols)
    cat = O.Catalog(scalars=[0, 1], shepard=[0, 1], grads=[-1], divs=[1, 2, 3])
    # pair estimate per sample: the coarse pass counts the pairs of every
    # sample (the oracle's neighbour digest stands in for psb_neighbor_digest)
    est, _, _ = orc.digest(s, strategy=O.SYMMETRIC, hmode=O.H_NEAREST)
    mine = shard_samples(*s, est, rank, world)
    part = orc.interp_points(*(a[mine] for a in s), cat, strategy=O.SYMMETRIC, hmode=O.H_NEAREST)
    # gather (indices, outputs) of every rank
    n_mine = torch.tensor([len(mine)])
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, n_mine)
    maxn = int(max(int(x) for x in sizes))
    buf = torch.full((1 + cat.L, maxn), float("nan"), dtype=torch.float64)
    buf[0, :len(mine)] = torch.from_numpy(mine.astype(np.float64))
    for k in range(cat.L):
        buf[1 + k, :len(mine)] = torch.from_numpy(np.asarray(part[k]))
    bufs = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf)
    # adjoint: partial gradients of this rank's samples, summed over ranks
    g = orc.adjoint_points(*(a[mine] for a in s), cat, [go[mine] for go in gout_all], strategy=O.SYMMETRIC,
                           hmode=O.H_NEAREST)
    allreduce_gradients(g)
    if rank == 0:
        full = [np.full(len(s[0]), np.nan) for _ in range(cat.L)]
        for b, nb in zip(bufs, sizes):
            nb = int(nb)
            idx = b[0, :nb].numpy().astype(np.int64)
            for k in range(cat.L):
                full[k][idx] = b[1 + k, :nb].numpy()
        pairs = [float(est[shard_samples(*s, est, r, world)].sum()) for r in range(world)]
        q.put((full, {k: g[k] for k in ("m", "x", "y", "z")}, [c for c in g["cols"]], pairs))
    dist.barrier()
    dist.destroy_process_group()


def _clustered_case():
    rng = np.random.default_rng(77)
    n = 20_000
    r = 0.1 / np.sqrt(rng.uniform(0.02, 1.0, n) ** (-2 / 3) - 1)
    v = rng.standard_normal((3, n))
    v /= np.linalg.norm(v, axis=0)
    x, y, z = r * v
    m = np.full(n, 1.0 / n)
    h = 0.02 * (1 + 4 * r)
    rho = 1.0 / (1 + 10 * r * r)
    cols = [rho.copy(), np.sin(5 * x) + y, -y, x + 0.1 * z]
    s = tuple(rng.uniform(-0.5, 0.5, 6000) for _ in range(3))
    gout = [rng.standard_normal(6000) for _ in range(1 + 1 + 3 + 1)]
    return (x, y, z, m, h, rho), cols, s, gout


def test_weighted_morton_shards_reassemble_the_oracle_result():
    """Two gloo ranks, each the oracle on its Morton range of samples of equal
    estimated pair count: the gathered fields equal the single-rank result
    bit for bit, the ranges balance the work, and the summed per-particle
    adjoint partials equal the single-rank adjoint."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_interp_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    full, gsum, gcols, pairs = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    P, cols, s, gout = _clustered_case()
    orc = O.Oracle(*P, cols)
    cat = O.Catalog(scalars=[0, 1], shepard=[0, 1], grads=[-1], divs=[1, 2, 3])
    ref = orc.interp_points(*s, cat, strategy=O.SYMMETRIC, hmode=O.H_NEAREST)
    for a, b in zip(full, ref):
        assert np.array_equal(np.isnan(a), np.isnan(b))
        assert np.array_equal(a[~np.isnan(a)], np.asarray(b)[~np.isnan(b)])
    # balanced by pair count (an equal-count split of this clustered set is not)
    assert max(pairs) <= 1.05 * (sum(pairs) / 2)
    g = orc.adjoint_points(*s, cat, gout, strategy=O.SYMMETRIC, hmode=O.H_NEAREST)
    for k in ("m", "x", "y", "z"):
        scale = np.abs(g[k]).max()
        assert np.abs(gsum[k] - g[k]).max() <= 1e-12 * scale, k
    for c in range(len(cols)):
        scale = max(np.abs(g["cols"][c]).max(), 1e-300)
        assert np.abs(gcols[c] - g["cols"][c]).max() <= 1e-12 * scale, c


def test_weighted_ranges_and_morton_order():
    from partia_b200.sharding import morton_order, weighted_ranges
    rng = np.random.default_rng(3)
    for world in (1, 2, 3, 8):
        w = rng.exponential(size=1000) ** 3
        rs = weighted_ranges(w, world)
        assert rs[0][0] == 0 and rs[-1][1] == 1000
        assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
        share = w.sum() / world
        for lo, hi in rs:
            assert w[lo:hi].sum() <= share + w.max() + 1e-9
    assert weighted_ranges(np.zeros(5), 2) == [(0, 2), (2, 5)]
    with pytest.raises(ValueError):
        weighted_ranges([-1.0], 1)
    # Morton order: a permutation; points in one octant come before the next
    x = rng.random(4000)
    y, z = rng.random(4000), rng.random(4000)
    o = morton_order(x, y, z)
    assert sorted(o.tolist()) == list(range(4000))
    # x's top quantisation bit is the code's most significant bit
    q = np.floor((x - x.min()) / (x.max() - x.min()) * 2097151.0)
    hi_x = (q >= 2 ** 20)[o]
    k = int(np.count_nonzero(~hi_x))
    assert not np.any(hi_x[:k]) and np.all(hi_x[k:])


def test_plane_pair_estimates_with_the_oracle_digest():
    """plane_pair_estimates' layout logic (subsampled x-y points of every
    z-plane, column-major) on a stand-in context whose digest is the oracle's;
    equal to the per-plane sums of the subsample's pair counts, scaled."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from partia_b200 import _lib as L
    from partia_b200.sharding import plane_pair_estimates, weighted_slabs
    P, cols, _, _ = _clustered_case()
    orc = O.Oracle(*P, cols)

    class OracleDigest:
        def digest(self, a, strategy=None, hmode=None):
            return orc.digest(a, strategy=O.SYMMETRIC, hmode=O.H_NEAREST)

    ax = np.linspace(-0.4, 0.4, 24)
    w = plane_pair_estimates(OracleDigest(), ax, ax, ax, stride=4, strategy=L.PSB_SYMMETRIC,
                             hmode=L.PSB_H_NEAREST)
    assert w.shape == (24,)
    sub = ax[::4]
    for k in (0, 11, 23):
        X, Y = np.meshgrid(sub, sub, indexing="ij")
        cnt, _, _ = orc.digest((X.ravel(), Y.ravel(), np.full(X.size, ax[k])), strategy=O.SYMMETRIC,
                               hmode=O.H_NEAREST)
        assert w[k] == pytest.approx(cnt.sum() * (24 * 24) / sub.size ** 2)
    # the clustered core holds most pairs: the middle slab is the thinnest
    slabs = weighted_slabs(w, 3)
    sizes = [hi - lo for lo, hi in slabs]
    assert sizes[1] < sizes[0] and sizes[1] < sizes[2]
