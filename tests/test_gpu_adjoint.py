"""GPU adjoint against the oracle's (finite-difference-pinned) adjoint.

dL/dm, dL/dA_c and dL/dx for L = sum_k sum_s gout[k][s] out_k(s): point
samples for every strategy and h mode, every output kind; structured grids;
parallel-beam line-integrated samples; each of the kernel families M5, M6 and
Wendland C2/C4/C6 besides M4.  The GPU sums the pair terms per
particle over an LBVH of the samples (or the pixel lattice); the oracle sums
them per sample.  Tolerance: 1e-10 of each gradient array's max |value| (the
two sum in different orders).
"""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

if not has_gpu():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

import oracle as O  # noqa: E402
from partia_b200 import _lib as L  # noqa: E402
from partia_b200.engine import CatalogC, Context  # noqa: E402

TOL = 1e-10
CAT = dict(scalars=[0, 1, 3], shepard=[0, 1, 1], grads=[-1, 1], divs=[1, 2, 3], curls=[3, 2, 1])


def particles(n, seed):
    rng = np.random.default_rng(seed)
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    m = rng.uniform(0.5, 1.5, n) / n
    h = 1.3 * (1.0 / n) ** (1 / 3) * rng.uniform(0.6, 1.6, n)
    rho = rng.uniform(0.5, 2.0, n)
    cols = [rho.copy(), np.sin(3 * x) + y, -y + 0.3 * z, x * x + 0.2 * rng.standard_normal(n)]
    return [x, y, z, m, h, rho], cols


def setup(n, seed, kernel=L.PSB_KERNEL_M4):
    arrs, cols = particles(n, seed)
    orc = O.Oracle(*arrs, cols=cols, kernel=kernel)
    ctx = Context(0)
    ctx.set_particles(*arrs, cols=cols, kernel=kernel)
    ctx.build(want_perm=False)
    return orc, ctx


def close(a, b, tol=TOL):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def compare(g, r, ncol):
    for key in ("m", "x", "y", "z"):
        assert close(g[key], r[key]) <= TOL, (key, close(g[key], r[key]))
    for c in range(ncol):
        if np.abs(r["cols"][c]).max() == 0:
            assert np.abs(g["cols"][c]).max() == 0, c
        else:
            assert close(g["cols"][c], r["cols"][c]) <= TOL, (c, close(g["cols"][c], r["cols"][c]))


@pytest.mark.parametrize("strategy", [L.PSB_GATHER, L.PSB_SCATTER, L.PSB_SYMMETRIC])
@pytest.mark.parametrize("hmode", [L.PSB_H_NEAREST, L.PSB_H_PER_SAMPLE])
def test_point_adjoint_matches_oracle(strategy, hmode):
    orc, ctx = setup(6000, 101)
    rng = np.random.default_rng(102)
    ns = 3000
    s = tuple(rng.uniform(-0.05, 1.05, ns) for _ in range(3))
    hs = rng.uniform(0.02, 0.05, ns) if hmode == L.PSB_H_PER_SAMPLE else None
    nl = O.Catalog(**CAT).L
    gout = [rng.standard_normal(ns) for _ in range(nl)]
    r = orc.adjoint_points(*s, O.Catalog(**CAT), gout, strategy=strategy, hmode=hmode, hs=hs)
    g = ctx.adjoint_points(*s, CatalogC(**CAT), gout, strategy=strategy, hmode=hmode, hs=hs)
    compare(g, r, 4)
    assert ctx.last_stats.pairs > 0


KERNELS = [L.PSB_KERNEL_M5, L.PSB_KERNEL_M6, L.PSB_KERNEL_C2, L.PSB_KERNEL_C4, L.PSB_KERNEL_C6]


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("strategy,hmode,spec", [
    (L.PSB_SYMMETRIC, L.PSB_H_NEAREST, CAT),
    (L.PSB_GATHER, L.PSB_H_PER_SAMPLE, CAT),
    (L.PSB_SCATTER, L.PSB_H_NEAREST, dict(scalars=[0, 2], shepard=[1, 0]))])  # scalar catalog: no Hessian
def test_point_adjoint_kernel_families(kernel, strategy, hmode, spec):
    orc, ctx = setup(5000, 121, kernel)
    rng = np.random.default_rng(122)
    ns = 2000
    s = tuple(rng.uniform(-0.05, 1.05, ns) for _ in range(3))
    hs = rng.uniform(0.02, 0.05, ns) if hmode == L.PSB_H_PER_SAMPLE else None
    nl = O.Catalog(**spec).L
    gout = [rng.standard_normal(ns) for _ in range(nl)]
    r = orc.adjoint_points(*s, O.Catalog(**spec), gout, strategy=strategy, hmode=hmode, hs=hs)
    g = ctx.adjoint_points(*s, CatalogC(**spec), gout, strategy=strategy, hmode=hmode, hs=hs)
    compare(g, r, 4)
    assert ctx.last_stats.pairs > 0


@pytest.mark.parametrize("kernel", KERNELS)
def test_beam_adjoint_kernel_families(kernel):
    from partia_b200 import workloads as W
    orc, ctx = setup(6000, 123, kernel)
    fr = W.Frame((0.5, 0.5, 0.5), (0.3, -0.2, 1.0), (1.0, 0.0, -0.3))
    farr = fr.as_array()
    prm = np.array([-0.35, 0.3, -0.25, 0.3])
    nx, ny = 30, 27
    nl = nx * ny
    rng = np.random.default_rng(124)
    scal, shep = [0, 1], [0, 1]
    gout = [rng.standard_normal(nl) for _ in scal]
    hs = np.array([0.03])
    ox = W.plane_coordinates(farr, (prm[0], prm[1], nx), (prm[2], prm[3], ny))
    fw = tuple(np.full(nl, farr[9 + c]) for c in range(3))
    r = orc.adjoint_lines(ox, fw, scal, gout, shepard=shep, strategy=O.SYMMETRIC, hmode=O.H_CONSTANT, hs=hs)
    g = ctx.adjoint_beam(farr, prm, nx, ny, CatalogC(scalars=scal, shepard=shep), gout, strategy=L.PSB_SYMMETRIC,
                         hmode=L.PSB_H_CONSTANT, hs=hs)
    compare(g, r, 4)
    assert ctx.last_stats.pairs > 0


def test_point_adjoint_device_pointers_and_unused_column():
    import torch
    orc, ctx = setup(4000, 103)
    rng = np.random.default_rng(104)
    ns = 1500
    s = tuple(rng.uniform(0.0, 1.0, ns) for _ in range(3))
    spec = dict(scalars=[1], shepard=[1], grads=[1])  # columns 0, 2, 3 unused
    gout = [rng.standard_normal(ns) for _ in range(4)]
    r = orc.adjoint_points(*s, O.Catalog(**spec), gout, strategy=O.SYMMETRIC)
    ts = tuple(torch.from_numpy(a).cuda() for a in s)
    tg = [torch.from_numpy(a).cuda() for a in gout]
    g = ctx.adjoint_points(*ts, CatalogC(**spec), tg, strategy=L.PSB_SYMMETRIC)
    g = {k: ([c.cpu().numpy() for c in v] if k == "cols" else v.cpu().numpy()) for k, v in g.items()}
    compare(g, r, 4)
    for c in (0, 2, 3):
        assert np.abs(g["cols"][c]).max() == 0


@pytest.mark.parametrize("kernel", [L.PSB_KERNEL_M4, L.PSB_KERNEL_C4])
@pytest.mark.parametrize("strategy,spec", [(L.PSB_SYMMETRIC, CAT), (L.PSB_GATHER, CAT),
                                           (L.PSB_SCATTER, dict(scalars=[0, 2], shepard=[1, 0]))])
def test_point_adjoint_two_kernels_bit_identical(kernel, strategy, spec):
    """The two-kernel point adjoint (pair lists in pooled blocks, partial sums
    per list block, added per particle in the walk's order): the same bits
    whatever the pool's size (a pool of 3 blocks grows and walks again),
    within 1e-12 of the single kernel (which adds the same terms in one
    running sum) and equal to the oracle."""
    orc, ctx = setup(6000, 131, kernel)
    rng = np.random.default_rng(132)
    ns = 3000
    s = tuple(rng.uniform(-0.05, 1.05, ns) for _ in range(3))
    nl = O.Catalog(**spec).L
    gout = [rng.standard_normal(ns) for _ in range(nl)]
    res = []
    npairs = []
    for blocks, split in ((0, 1), (3, 1), (0, 0)):  # default pool, 3 blocks, single kernel
        assert ctx.lib.psb_test_adjoint_pool(ctx.h, blocks, split) == L.PSB_OK
        res.append(ctx.adjoint_points(*s, CatalogC(**spec), gout, strategy=strategy))
        npairs.append(ctx.last_stats.pairs)
    assert npairs[0] > 0 and npairs[1] == npairs[0] and npairs[2] == npairs[0]
    for key in ("m", "x", "y", "z"):
        assert np.array_equal(res[1][key], res[0][key]), key
        assert close(res[2][key], res[0][key]) <= 1e-12, key
    for c in range(4):
        assert np.array_equal(res[1]["cols"][c], res[0]["cols"][c]), c
        if np.abs(res[0]["cols"][c]).max() > 0:
            assert close(res[2]["cols"][c], res[0]["cols"][c]) <= 1e-12, c
    r = orc.adjoint_points(*s, O.Catalog(**spec), gout, strategy=strategy)
    compare(res[0], r, 4)
    # a pool of 3 blocks that keeps its size: most tiles run in the single kernel
    assert ctx.lib.psb_test_adjoint_pool(ctx.h, 3, 2) == L.PSB_OK
    g = ctx.adjoint_points(*s, CatalogC(**spec), gout, strategy=strategy)
    assert ctx.last_stats.pairs == npairs[0]
    for key in ("m", "x", "y", "z"):
        assert close(g[key], res[0][key]) <= 1e-12, key
    compare(g, r, 4)
    assert ctx.lib.psb_test_adjoint_pool(ctx.h, -1, 1) == L.PSB_EINVAL
    assert ctx.lib.psb_test_adjoint_pool(ctx.h, 0, 3) == L.PSB_EINVAL
    assert ctx.lib.psb_test_adjoint_pool(ctx.h, 0, 1) == L.PSB_OK


@pytest.mark.parametrize("spec", [
    dict(scalars=[0, 4, 5], shepard=[1, 0, 1], grads=[4, 5], divs=[1, 2, 3], curls=[5, 4, 1]),
    dict(scalars=[0, 1, 2, 3, 4, 5], shepard=[1, 0, 1, 0, 1, 0])])  # scalar catalog
def test_point_adjoint_six_columns(spec):
    """Six columns take the 8-column instantiations: records with the columns
    past the fourth, and the general form's cotangents read from global
    memory in the single kernel.  The two forms agree within 1e-12, and both
    equal the oracle."""
    arrs, cols = particles(5000, 141)
    rng = np.random.default_rng(142)
    cols = cols + [np.cos(2 * arrs[1]) + 0.1 * rng.standard_normal(5000), arrs[2] ** 2 - arrs[0]]
    orc = O.Oracle(*arrs, cols=cols)
    ctx = Context(0)
    ctx.set_particles(*arrs, cols=cols)
    ctx.build(want_perm=False)
    ns = 2500
    s = tuple(rng.uniform(-0.05, 1.05, ns) for _ in range(3))
    nl = O.Catalog(**spec).L
    gout = [rng.standard_normal(ns) for _ in range(nl)]
    res = []
    for split in (1, 0):
        assert ctx.lib.psb_test_adjoint_pool(ctx.h, 0, split) == L.PSB_OK
        res.append(ctx.adjoint_points(*s, CatalogC(**spec), gout, strategy=L.PSB_SYMMETRIC))
    for key in ("m", "x", "y", "z"):
        assert close(res[1][key], res[0][key]) <= 1e-12, key
    for c in range(6):
        if np.abs(res[0]["cols"][c]).max() > 0:
            assert close(res[1]["cols"][c], res[0]["cols"][c]) <= 1e-12, c
    r = orc.adjoint_points(*s, O.Catalog(**spec), gout, strategy=O.SYMMETRIC)
    compare(res[0], r, 6)
    compare(res[1], r, 6)


def test_grid_adjoint_matches_points():
    orc, ctx = setup(5000, 105)
    ax = np.linspace(0.05, 0.95, 14)
    ay = np.linspace(0.1, 0.9, 11)
    az = np.linspace(0.0, 1.0, 9)
    ns = len(ax) * len(ay) * len(az)
    rng = np.random.default_rng(106)
    spec = dict(scalars=[0], shepard=[0], grads=[0], divs=[1, 2, 3], curls=[1, 2, 3])
    gout = [rng.standard_normal(ns) for _ in range(8)]
    X, Y, Z = np.meshgrid(ax, ay, az, indexing="ij")
    s = (X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F"))
    r = orc.adjoint_points(*s, O.Catalog(**spec), gout, strategy=O.SYMMETRIC)
    g = ctx.adjoint_grid(ax, ay, az, CatalogC(**spec), gout, strategy=L.PSB_SYMMETRIC)
    compare(g, r, 4)


@pytest.mark.parametrize("strategy", [L.PSB_SCATTER, L.PSB_GATHER, L.PSB_SYMMETRIC])
def test_beam_adjoint_matches_oracle(strategy):
    from partia_b200 import workloads as W
    orc, ctx = setup(8000, 107)
    fr = W.Frame((0.5, 0.5, 0.5), (0.3, -0.2, 1.0), (1.0, 0.0, -0.3))
    fr.rotate(0.3, -0.2, 0.5)
    farr = fr.as_array()
    prm = np.array([-0.35, 0.3, -0.25, 0.3])
    nx, ny = 40, 33
    nl = nx * ny
    rng = np.random.default_rng(108)
    scal, shep = [0, 1], [0, 1]
    gout = [rng.standard_normal(nl) for _ in scal]
    hs = None if strategy == L.PSB_SCATTER else np.array([0.03])
    hm = L.PSB_H_CONSTANT
    ox = W.plane_coordinates(farr, (prm[0], prm[1], nx), (prm[2], prm[3], ny))
    fw = tuple(np.full(nl, farr[9 + c]) for c in range(3))
    r = orc.adjoint_lines(ox, fw, scal, gout, shepard=shep, strategy=strategy, hmode=O.H_CONSTANT, hs=hs)
    g = ctx.adjoint_beam(farr, prm, nx, ny, CatalogC(scalars=scal, shepard=shep), gout, strategy=strategy,
                         hmode=hm, hs=hs)
    compare(g, r, 4)
    assert ctx.last_stats.pairs > 0


@pytest.mark.parametrize("strategy,hmode", [(L.PSB_SCATTER, L.PSB_H_NEAREST), (L.PSB_GATHER, L.PSB_H_PER_SAMPLE),
                                            (L.PSB_SYMMETRIC, L.PSB_H_CONSTANT)])
def test_plain_scalar_adjoint_without_forward_pass(strategy, hmode):
    """Plain (non-Shepard) scalars: the sum cotangents are the output
    cotangents themselves, so no forward pass runs; points and beams."""
    from partia_b200 import workloads as W
    orc, ctx = setup(5000, 111)
    rng = np.random.default_rng(112)
    ns = 2000
    s = tuple(rng.uniform(0.0, 1.0, ns) for _ in range(3))
    hs = {L.PSB_H_NEAREST: None, L.PSB_H_PER_SAMPLE: rng.uniform(0.02, 0.05, ns),
          L.PSB_H_CONSTANT: np.array([0.035])}[hmode]
    spec = dict(scalars=[0, 2, 0], shepard=[0, 0, 0])
    gout = [rng.standard_normal(ns) for _ in range(3)]
    r = orc.adjoint_points(*s, O.Catalog(**spec), gout, strategy=strategy, hmode=hmode, hs=hs)
    g = ctx.adjoint_points(*s, CatalogC(**spec), gout, strategy=strategy, hmode=hmode, hs=hs)
    compare(g, r, 4)
    if strategy != L.PSB_SCATTER and hmode == L.PSB_H_NEAREST:
        return
    fr = W.c3_frame().as_array()
    prm = np.array([0.0, 1.0, 0.0, 1.0])
    nx = ny = 37
    gl = [rng.standard_normal(nx * ny)]
    hl = None if strategy == L.PSB_SCATTER else np.array([0.03])
    ox = W.plane_coordinates(fr, (0.0, 1.0, nx), (0.0, 1.0, ny))
    fw = tuple(np.full(nx * ny, fr[9 + c]) for c in range(3))
    r = orc.adjoint_lines(ox, fw, [0], gl, shepard=[0], strategy=strategy, hmode=O.H_CONSTANT, hs=hl)
    g = ctx.adjoint_beam(fr, prm, nx, ny, CatalogC(scalars=[0], shepard=[0]), gl, strategy=strategy,
                         hmode=L.PSB_H_CONSTANT, hs=hl)
    compare(g, r, 4)


def test_adjoint_error_paths():
    orc, ctx = setup(500, 109)
    s = (np.array([0.5]), np.array([0.5]), np.array([0.5]))
    with pytest.raises(L.PsbError):  # gather needs hs unless nearest
        ctx.adjoint_points(*s, CatalogC(scalars=[0]), [np.ones(1)], strategy=L.PSB_GATHER,
                           hmode=L.PSB_H_PER_SAMPLE, hs=None)
    # a frame whose right and up axes coincide
    bad = np.array([0, 0, 0, 1, 0, 0, 1, 0, 0, 0, 0, 1], dtype=float)
    with pytest.raises(L.PsbError):
        ctx.adjoint_beam(bad, np.array([0.0, 1.0, 0.0, 1.0]), 4, 4, CatalogC(scalars=[0]), [np.ones(16)])
