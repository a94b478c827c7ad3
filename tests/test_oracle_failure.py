"""Failure detection in the oracle's walks (checker side of the GPU test).

Every escape link that ends a traversal is pointed at the root, so every walk
cycles; the stackless traversal's step bound (4n + 4) must end each of them
with an error instead of looping, and a rebuild restores the results.
"""
import numpy as np
import pytest

import oracle as O


def test_walk_bound_reports_a_cycle_and_rebuild_recovers():
    rng = np.random.default_rng(9)
    n = 2000
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    m, h, rho = np.full(n, 1.0 / n), 0.05 * rng.uniform(0.7, 1.3, n), np.ones(n)
    orc = O.Oracle(x, y, z, m, h, rho, [x.copy()])
    s = tuple(rng.uniform(0.1, 0.9, 200) for _ in range(3))
    cat = O.Catalog(scalars=[0], shepard=[1])
    ref = orc.interp_points(*s, cat, strategy=O.SYMMETRIC, hmode=O.H_NEAREST)
    orc.test_loop_escapes()
    with pytest.raises(RuntimeError):
        orc.interp_points(*s, cat, strategy=O.SYMMETRIC, hmode=O.H_NEAREST)
    with pytest.raises(RuntimeError):
        orc.density(*s, strategy=O.SCATTER)
    orc.rebuild()
    again = orc.interp_points(*s, cat, strategy=O.SYMMETRIC, hmode=O.H_NEAREST)
    assert np.array_equal(ref[0], again[0])
