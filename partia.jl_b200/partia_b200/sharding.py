"""Sample sharding across GPUs (one process per GPU).

Samples are independent (PointSamples_driver.jl:38 loops over them), so a
multi-GPU run replicates the particle set and its LBVH on every rank (the
build is deterministic, so every rank builds the same tree) and gives each
rank a disjoint block of samples; the forward outputs need no collective
beyond gathering them where they are wanted.

Work per sample is its accepted-pair count, which varies by orders of
magnitude over a clustered particle set (a Plummer core against its
outskirts).  Blocks are therefore balanced by an estimate of that count:

 * explicit samples are put in Morton order (spatially coherent blocks, the
   order the library tiles them in) and cut into contiguous ranges of equal
   estimated work (``weighted_ranges``);
 * a StructuredGrid is cut into slabs of z-planes of equal estimated work
   (``weighted_slabs``), which keeps each rank's samples contiguous in the
   column-major output layout.

The estimate comes from a coarse pass: ``psb_neighbor_digest`` counts the
pairs of a sparse subset of the samples (``plane_pair_estimates`` for
grids).  The adjoint's per-particle gradients are partial sums over each
rank's samples; ``allreduce_gradients`` adds them (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import numpy as np


def slab(n: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) of n items owned by rank (balanced to within one item)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("rank must be in 0..world-1")
    return (n * rank) // world, (n * (rank + 1)) // world


def grid_slab(nx: int, ny: int, nz: int, rank: int, world: int):
    """z-plane range and the linear sample range of this rank's equal slab."""
    z0, z1 = slab(nz, rank, world)
    return (z0, z1), (nx * ny * z0, nx * ny * z1)


def weighted_ranges(weights, world: int) -> list[tuple[int, int]]:
    """Contiguous [lo, hi) ranges of equal total weight, one per rank.

    Cut k is the first index whose prefix sum reaches k/world of the total,
    so every range is contiguous, ranges tile 0..n, and no rank's weight
    exceeds its share by more than one item's weight.  Zero total weight
    falls back to equal counts."""
    w = np.asarray(weights, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be positive")
    if np.any(w < 0) or not np.all(np.isfinite(w)):
        raise ValueError("weights must be finite and non-negative")
    n = len(w)
    tot = float(w.sum())
    if tot <= 0.0:
        return [slab(n, r, world) for r in range(world)]
    c = np.cumsum(w)
    cuts = [0] + [int(np.searchsorted(c, tot * k / world, side="left")) + 1 for k in range(1, world)] + [n]
    cuts = [min(max(x, 0), n) for x in cuts]
    for k in range(1, len(cuts)):  # monotone
        cuts[k] = max(cuts[k], cuts[k - 1])
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def weighted_slabs(plane_weights, world: int) -> list[tuple[int, int]]:
    """z-plane ranges of equal estimated work (plane_weights[k] for plane k)."""
    return weighted_ranges(plane_weights, world)


def _spread21(v: np.ndarray) -> np.ndarray:
    v = v.astype(np.uint64) & np.uint64(0x1FFFFF)
    v = (v | (v << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
    v = (v | (v << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
    v = (v | (v << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
    v = (v | (v << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
    v = (v | (v << np.uint64(2))) & np.uint64(0x1249249249249249)
    return v


def morton_order(sx, sy, sz) -> np.ndarray:
    """Stable order of samples along a 63-bit Morton curve over their own
    bounding box (x most significant), the coherent order of sample tiles."""
    pts = [np.asarray(a, dtype=np.float64) for a in (sx, sy, sz)]
    codes = np.zeros(len(pts[0]), dtype=np.uint64)
    for d, a in enumerate(pts):
        if len(a) == 0:
            return np.zeros(0, dtype=np.int64)
        lo, hi = float(a.min()), float(a.max())
        f = np.zeros_like(a) if hi <= lo else (a - lo) / (hi - lo)
        q = np.floor(f * 2097151.0).astype(np.uint64)
        codes |= _spread21(q) << np.uint64(2 - d)
    return np.argsort(codes, kind="stable")


def shard_samples(sx, sy, sz, pair_estimate, rank: int, world: int):
    """This rank's samples: indices into the caller's arrays (in Morton order)
    of the contiguous Morton range of equal estimated pair count."""
    order = morton_order(sx, sy, sz)
    w = np.asarray(pair_estimate, dtype=np.float64)[order]
    lo, hi = weighted_ranges(w, world)[rank]
    return order[lo:hi]


def plane_pair_estimates(ctx, ax, ay, az, stride: int = 8, strategy=None, hmode=None):
    """Estimated accepted pairs per z-plane of a Cartesian grid: neighbour
    digests (pair counts) of every stride-th point in x and y of each plane,
    scaled to the plane.  One psb_neighbor_digest call (a coarse pass)."""
    from . import _lib as L
    strategy = L.PSB_SYMMETRIC if strategy is None else strategy
    hmode = L.PSB_H_NEAREST if hmode is None else hmode
    ax, ay, az = (np.asarray(a, dtype=np.float64) for a in (ax, ay, az))
    sx, sy = ax[::stride], ay[::stride]
    X, Y, Z = np.meshgrid(sx, sy, az, indexing="ij")
    cnt, _, _ = ctx.digest((X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")), strategy=strategy,
                           hmode=hmode)
    per_plane = cnt.reshape(len(sx) * len(sy), len(az), order="F").sum(axis=0).astype(np.float64)
    return per_plane * (len(ax) * len(ay)) / float(len(sx) * len(sy))


def allreduce_gradients(g: dict, group=None):
    """Sum the adjoint's per-particle partial gradients over ranks in place
    (dict with 'm', 'x', 'y', 'z' and the 'cols' list, as the adjoint calls
    return them); torch tensors on the process group's device, or numpy
    arrays (summed through CPU tensors, for gloo)."""
    import torch
    import torch.distributed as dist
    keys = ["m", "x", "y", "z"]
    arrs = [g[k] for k in keys] + list(g.get("cols", []))
    for k, a in enumerate(arrs):
        t = a if isinstance(a, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(a))
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        if not isinstance(a, torch.Tensor):
            a[...] = t.numpy()
    return g
