"""The Partia-API layer (partia_b200.api) on the GPU: the reference's
driver-level tests, run through the drop-in surface against brute force and
the oracle.

 * PointSamples_interpolation, symmetric, nearest-particle h, on the
   4-particle fixture: scalar and divergence vs brute force at rtol 1e-10,
   names, shared coordinate containers
   (test/point_samples_interpolation_tests.jl:53-79,
    test/grid_interpolation_test_common.jl:40-71)
 * auto vs externally supplied LBVH give identical grids; an input in another
   leaf order is rejected with ArgumentError (:83-117; the driver at
   src/julia/KernelInterpolation/grid_interpolation/drivers/PointSamples_driver.jl:98-118)
 * LineSamples_interpolation, scatter, on the line fixture vs brute force, and
   the ArgumentError of gather and symmetric (:121-207)
 * StructuredGrid_interpolation equals its flattened PointSamples
   (test/structured_grid_interpolation_tests.jl:256-322)
 * LinearBVH! permutes the input in place exactly as the reference does
   (src/julia/KernelInterpolation/interpolation_setup/InterpolationInput.jl:201-221),
   with the oracle's permutation
 * the input keeps one device context: a second driver call on the same input
   builds nothing and allocates nothing, a changed value column is picked up,
   and changed coordinates rebuild the tree.
"""
import copy
import math

import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

if not has_gpu():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

import torch  # noqa: E402

import bruteforce as B  # noqa: E402
import oracle as O  # noqa: E402
import partia_b200 as P  # noqa: E402
from partia_b200 import _lib as L  # noqa: E402


def grid_fixture():
    """make_grid_interpolation_fixture: 4 particles, (temp, vx, vy, vz), M4."""
    x = np.array([0.15, 0.35, 0.55, 0.75])
    y = np.array([0.20, 0.60, 0.25, 0.70])
    z = np.array([0.25, 0.45, 0.80, 0.30])
    h = np.array([0.28, 0.24, 0.26, 0.22])
    rho = np.array([1.0, 0.95, 1.05, 1.1])
    m = np.array([0.4, 0.45, 0.42, 0.38])
    temp = np.array([10.0, 11.0, 13.0, 12.0])
    vx = np.array([0.1, -0.2, 0.3, -0.1])
    vy = np.array([0.0, 0.25, -0.15, 0.2])
    vz = np.array([-0.05, 0.1, 0.2, -0.1])
    inp = P.InterpolationInput(x, y, z, m, h, rho, (temp, vx, vy, vz), smoothed_kernel=P.M4_spline)
    cat = P.InterpolationCatalog.from_columns(("temp", "vx", "vy", "vz"), scalars=("temp",), divergences=("v",))
    lbvh = P.LinearBVH_(inp, P.B200ComputeBackend())
    return inp, cat, lbvh


def point_template():
    x = np.array([0.20, 0.40, 0.65])
    y = np.array([0.25, 0.55, 0.50])
    z = np.array([0.30, 0.50, 0.35])
    return P.PointSamples(np.zeros(3), (x, y, z))


def brute_input(inp):
    Pd = dict(x=inp.coord[0], y=inp.coord[1], z=inp.coord[2], m=inp.m, h=inp.h, rho=inp.rho)
    return Pd, list(inp.quant)


def test_point_samples_symmetric_nearest_h_vs_brute_force():
    inp, cat, _ = grid_fixture()
    tpl = point_template()
    res = P.PointSamples_interpolation(P.B200ComputeBackend(), tpl, inp, cat, P.itpSymmetric)
    assert res.names == cat.ordered_names == ("temp", "∇⋅v")
    assert len(res.grids) == 2
    assert res.grids[0].coor is res.grids[1].coor
    assert all(np.array_equal(a, b) for a, b in zip(res.grids[0].coor, tpl.coor))
    Pd, cols = brute_input(inp)
    for i in range(3):
        p = np.array([tpl.coor[0][i], tpl.coor[1][i], tpl.coor[2][i]])
        ha = B.nearest_h(Pd, p)
        ref = B.general(Pd, cols, p, ha, "symmetric", scalars=[0], shepard=[1], divs=[(1, 2, 3)])
        assert res.grids[0].grid[i] == pytest.approx(ref[0], rel=1e-10, abs=1e-12)
        assert res.grids[1].grid[i] == pytest.approx(ref[1], rel=1e-10, abs=1e-12)


def test_external_lbvh_matches_auto_and_rejects_other_order():
    inp, cat, lbvh = grid_fixture()
    tpl = point_template()
    be = P.B200ComputeBackend()
    auto = P.PointSamples_interpolation(be, tpl, inp, cat, P.itpSymmetric)
    manual = P.PointSamples_interpolation(be, tpl, inp, lbvh, cat, P.itpSymmetric)
    assert manual.names == auto.names
    for a, b in zip(auto.grids, manual.grids):
        assert all(np.array_equal(u, v) for u, v in zip(a.coor, b.coor))
        assert np.array_equal(a.grid, b.grid)
    assert P.matches_lbvh_leaf_order(inp, lbvh)
    bad = copy.deepcopy(inp)
    p = [1, 0, 2, 3]
    for a in (*bad.coord, bad.m, bad.h, bad.rho, *bad.quant):
        a[:] = a[p]
    assert not P.matches_lbvh_leaf_order(bad, lbvh)
    with pytest.raises(P.ArgumentError):
        P.PointSamples_interpolation(be, tpl, bad, lbvh, cat, P.itpSymmetric)


def line_fixture():
    x = np.array([0.15, 0.35, 0.55, 0.75])
    y = np.array([0.20, 0.60, 0.25, 0.70])
    z = np.array([0.25, 0.45, 0.80, 0.30])
    h = np.array([0.28, 0.24, 0.26, 0.22])
    rho = np.array([1.0, 0.95, 1.05, 1.1])
    m = np.array([0.4, 0.45, 0.42, 0.38])
    temp = np.array([10.0, 11.0, 13.0, 12.0])
    vx = np.array([0.1, -0.2, 0.3, -0.1])
    inp = P.InterpolationInput(x, y, z, m, h, rho, (temp, vx), smoothed_kernel=P.M4_spline)
    cat = P.InterpolationCatalog.from_columns(("temp", "vx"), scalars=("temp", "vx"))
    lbvh = P.LinearBVH_(inp, P.B200ComputeBackend())
    return inp, cat, lbvh


def line_template():
    r2 = 1 / math.sqrt(2.0)
    o = (np.array([0.20, 0.40, 0.55]), np.array([0.25, 0.35, 0.45]), np.array([0.00, 0.10, 0.20]))
    d = (np.array([0.0, r2, 1.0]), np.array([0.0, 0.0, 0.0]), np.array([1.0, r2, 0.0]))
    return P.LineSamples(np.zeros(3), o, d)


def test_line_samples_scatter_vs_brute_force_and_modes():
    inp, cat, lbvh = line_fixture()
    tpl = line_template()
    be = P.B200ComputeBackend()
    res = P.LineSamples_interpolation(be, tpl, inp, cat, P.itpScatter)
    assert res.names == ("temp", "vx")
    assert res.grids[0].origin is res.grids[1].origin and res.grids[0].direction is res.grids[1].direction
    Pd, cols = brute_input(inp)
    table = O.line_table()
    for i in range(3):
        o = [tpl.origin[k][i] for k in range(3)]
        d = [tpl.direction[k][i] for k in range(3)]
        # the catalog's scalars: temp and vx are Shepard-normalised (not named rho)
        ref = B.line_quantities(Pd, cols, o, d, 0.0, "scatter", [0, 1], [1, 1], table)
        assert res.grids[0].grid[i] == pytest.approx(ref[0], rel=1e-10, abs=1e-12)
        assert res.grids[1].grid[i] == pytest.approx(ref[1], rel=1e-10, abs=1e-12)
    manual = P.LineSamples_interpolation(be, tpl, inp, lbvh, cat, P.itpScatter)
    for a, b in zip(res.grids, manual.grids):
        assert np.array_equal(a.grid, b.grid)
    for st in (P.itpGather, P.itpSymmetric):
        with pytest.raises(P.ArgumentError):
            P.LineSamples_interpolation(be, tpl, inp, cat, st)
    pinp, pcat, _ = grid_fixture()
    with pytest.raises(P.ArgumentError):  # a divergence has no line-integrated form
        P.LineSamples_interpolation(be, tpl, pinp, pcat, P.itpScatter)


@pytest.mark.parametrize("strategy", [P.itpGather, P.itpScatter, P.itpSymmetric])
def test_structured_grid_equals_flattened_point_samples(strategy):
    inp, _, _ = grid_fixture()
    cat = P.InterpolationCatalog.from_columns(("temp", "vx", "vy", "vz"), scalars=("temp",), gradients=("temp",),
                                              divergences=("v",), curls=("v",))
    g = P.StructuredGrid.cartesian((0.20, 0.70, 3), (0.25, 0.55, 2), (0.30, 0.60, 2))
    be = P.B200ComputeBackend()
    res = P.StructuredGrid_interpolation(be, P.Cartesian, g, inp, cat, strategy)
    flat = P.flatten(P.Cartesian, g)
    ref = P.PointSamples_interpolation(be, flat, inp, cat, strategy)
    assert res.names == ref.names
    for a, b in zip(res.grids, ref.grids):
        assert a.size == g.size
        assert all(np.array_equal(u, v) for u, v in zip(a.axes, g.axes))
        ga, gb = a.grid.ravel(order="F"), b.grid
        assert np.array_equal(np.isnan(ga), np.isnan(gb))
        assert np.array_equal(ga[~np.isnan(ga)], gb[~np.isnan(gb)])


def test_linear_bvh_permutes_input_in_place_like_the_reference():
    rng = np.random.default_rng(21)
    n = 5000
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    m, h, rho = rng.uniform(0.5, 1.5, n) / n, 0.03 * rng.uniform(0.5, 2, n), rng.uniform(0.5, 2, n)
    A = rng.standard_normal(n)
    inp = P.InterpolationInput(x.copy(), y.copy(), z.copy(), m.copy(), h.copy(), rho.copy(), (A.copy(),),
                               smoothed_kernel=P.M4_spline)
    arrays_before = [inp.coord[0], inp.m, inp.quant[0]]
    lbvh = P.LinearBVH_(inp, P.B200ComputeBackend())
    orc = O.Oracle(x, y, z, m, h, rho, [A])
    assert np.array_equal(lbvh.perm, orc.perm)
    for got, orig in ((inp.coord[0], x), (inp.coord[1], y), (inp.coord[2], z), (inp.m, m), (inp.h, h),
                      (inp.rho, rho), (inp.quant[0], A)):
        assert np.array_equal(got, orig[orc.perm])
    # in place: the same array objects
    assert inp.coord[0] is arrays_before[0] and inp.m is arrays_before[1] and inp.quant[0] is arrays_before[2]
    assert P.matches_lbvh_leaf_order(inp, lbvh)
    # a second LinearBVH! finds the input in Morton order: identity permutation
    lbvh2 = P.LinearBVH_(inp, P.B200ComputeBackend())
    assert np.array_equal(lbvh2.perm, np.arange(n))


def test_input_keeps_one_context_and_reuses_its_lbvh():
    rng = np.random.default_rng(5)
    n = 20000
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    m, h, rho = np.full(n, 1.0 / n), 1.2 * (1.0 / n) ** (1 / 3) * rng.uniform(0.7, 1.4, n), rng.uniform(0.8, 1.2, n)
    T = np.sin(3 * x) + y
    inp = P.InterpolationInput(x, y, z, m, h, rho, (rho.copy(), T), smoothed_kernel=P.M4_spline)
    cat = P.InterpolationCatalog.from_columns(("rho", "T"), scalars=("rho", "T"), gradients=("T",))
    s = tuple(rng.uniform(0.1, 0.9, 3000) for _ in range(3))
    tpl = P.PointSamples(np.zeros(3000), s)
    be = P.B200ComputeBackend()
    r1 = P.PointSamples_interpolation(be, tpl, inp, cat)
    ctx = inp._b200_ctx
    assert ctx is not None and ctx.builds == 1
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    r2 = P.PointSamples_interpolation(be, tpl, inp, cat)
    torch.cuda.synchronize()
    assert inp._b200_ctx is ctx and ctx.builds == 1, "the second call rebuilt the LBVH"
    assert torch.cuda.mem_get_info()[0] == free0, "the second call allocated device memory"
    for a, b in zip(r1.grids, r2.grids):
        assert np.array_equal(a.grid, b.grid)
    # a changed value column is picked up without a rebuild
    inp.quant[1][:] = 2.0 * inp.quant[1]
    r3 = P.PointSamples_interpolation(be, tpl, inp, cat)
    assert ctx.builds == 1
    np.testing.assert_allclose(r3.grids[1].grid, 2.0 * r1.grids[1].grid, rtol=1e-12, atol=0)
    orc = O.Oracle(*inp.coord, inp.m, inp.h, inp.rho, list(inp.quant))
    ref = orc.interp_points(*s, O.Catalog(scalars=[0, 1], shepard=[0, 1], grads=[1]), strategy=O.SYMMETRIC,
                            hmode=O.H_NEAREST)
    for k, g in enumerate(r3.grids):
        err = np.max(np.abs(g.grid - ref[k])) / np.max(np.abs(ref[k]))
        assert err <= 1e-12, k
    # moved particles: the leaf order no longer matches, the tree is rebuilt on the same context
    inp.coord[0][:] = inp.coord[0][::-1].copy()
    P.PointSamples_interpolation(be, tpl, inp, cat)
    assert inp._b200_ctx is ctx and ctx.builds == 2
    assert P.matches_lbvh_leaf_order(inp, inp._b200_lbvh)


def test_external_lbvh_after_its_context_was_rebuilt():
    """An LBVH handle whose context now holds another build is rebound from
    the (matching) input instead of using the other tree."""
    inp, cat, lbvh = grid_fixture()
    tpl = point_template()
    be = P.B200ComputeBackend()
    ref = P.PointSamples_interpolation(be, tpl, inp, lbvh, cat, P.itpSymmetric)
    other = copy.deepcopy(inp)
    other._b200_ctx = lbvh.ctx  # share the context, then build other particles on it
    for a in other.coord:
        a[:] = a + 0.01
    P.LinearBVH_(other, be)
    assert lbvh.ctx.generation != lbvh.generation
    again = P.PointSamples_interpolation(be, tpl, inp, lbvh, cat, P.itpSymmetric)
    for a, b in zip(ref.grids, again.grids):
        assert np.array_equal(a.grid, b.grid)
