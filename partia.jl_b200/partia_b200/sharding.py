"""Sample sharding across GPUs (one process per GPU).

Samples are independent (PointSamples_driver.jl:38 loops over them), so a
multi-GPU run replicates the particle set and its LBVH on every rank and gives
each rank a disjoint block of samples; outputs need no collective.  For a
StructuredGrid the block is a slab of z-planes, which keeps every rank's
samples contiguous in the column-major output layout.
"""
from __future__ import annotations


def slab(n: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) of n items owned by rank (balanced to within one item)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("rank must be in 0..world-1")
    return (n * rank) // world, (n * (rank + 1)) // world


def grid_slab(nx: int, ny: int, nz: int, rank: int, world: int):
    """z-plane range and the linear sample range of this rank's slab."""
    z0, z1 = slab(nz, rank, world)
    return (z0, z1), (nx * ny * z0, nx * ny * z1)
