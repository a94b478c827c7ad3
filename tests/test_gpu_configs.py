"""The benchmark configurations at their own sizes.

Where the oracle would take minutes, parity is checked on a random subset of
samples and, at full size, through properties that do not depend on the size:
the FP32C path against the FP64 path field by field, and FP32C accept/reject
decisions against FP64 ones (identical neighbour sets).

 * C1: 100k uniform particles, rho from the density sum, gather with the mean
   h and with the nearest particle's h, 64^3 cell-centre grid: all samples
   against the oracle.
 * C2: 2M-particle Plummer sphere, symmetric, 8 fields on the 128^3 grid:
   FP32C within 1e-6 of FP64 on every field, identical neighbour sets on 200k
   grid points, oracle on 20k of them.
 * C3: 8M clump particles (h from the density sum), column density on the
   1024^2 beam: FP32C against FP64, oracle on 2000 lines.
 * C4: 1M clump particles, adjoint of the column density on a 128^2 beam
   against the oracle's adjoint; and at the configuration itself (512^2
   beam, loss 0.5 ||Sigma - Sigma_target||^2) against central finite
   differences of the GPU FP64 forward on 64 random particles.
 * C5-shaped: 4M float32 disc + halo particles, rho, grad rho, curl v,
   Shepard z^2 on a grid and an oriented box: FP32C against FP64, oracle
   subset at float accuracy.  The adjoint of the grid scalar's L2 norm for
   2M of them: identities at full grid size, oracle on a sample subset.
"""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

if not has_gpu():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

import oracle as O  # noqa: E402
from partia_b200 import _lib as L  # noqa: E402
from partia_b200 import linrange  # noqa: E402
from partia_b200 import workloads as W  # noqa: E402
from partia_b200.engine import CatalogC, Context  # noqa: E402


def rel_err(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb), "NaN masks differ"
    fin = ~na
    if not fin.any():
        return 0.0
    scale = np.max(np.abs(b[fin]))
    return float(np.max(np.abs(a[fin] - b[fin])) / scale) if scale > 0 else float(np.max(np.abs(a[fin])))


def grid_points(ax, ay, az):
    X, Y, Z = np.meshgrid(ax, ay, az, indexing="ij")
    return X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")


def make_ctx(d, h, rho, cols, dtype=np.float64):
    ctx = Context(0)
    ctx.set_particles(d["x"], d["y"], d["z"], d["m"], h, rho, cols, dtype=dtype)
    ctx.build(want_perm=False)
    return ctx


def test_c1_uniform_gather_full_size():
    d = W.uniform_c1()
    x, y, z, m, h = d["x"], d["y"], d["z"], d["m"], d["h"]
    # rho_b from the method's own density sum at the particles (gather, ha = h_b)
    rho = O.Oracle(x, y, z, m, h, np.ones_like(m)).density(x, y, z, strategy=O.GATHER, hmode=O.H_PER_SAMPLE, hs=h)
    cols = [rho, d["A"]]
    orc = O.Oracle(x, y, z, m, h, rho, cols)
    ctx = make_ctx(d, h, rho, cols)
    ax = linrange(*W.cell_centre_axis(64))
    s = grid_points(ax, ax, ax)
    spec = dict(scalars=[0, 1], shepard=[0, 1])
    for hmode, hs in ((O.H_CONSTANT, np.array([np.mean(h)])), (O.H_NEAREST, None)):
        ref = orc.interp_points(*s, O.Catalog(**spec), strategy=O.GATHER, hmode=hmode, hs=hs)
        for prec, tol in ((L.PSB_PREC_FP64, 1e-12), (L.PSB_PREC_FP32C, 1e-6)):
            g = ctx.interp_grid(ax, ax, ax, CatalogC(**spec), strategy=L.PSB_GATHER, hmode=hmode, hs=hs, prec=prec)
            for k in range(2):
                assert rel_err(g[k], ref[k]) <= tol, (hmode, prec, k, rel_err(g[k], ref[k]))
        co, ho, _ = orc.digest(s, strategy=O.GATHER, hmode=hmode, hs=hs)
        for fp32c in (False, True):
            cg, hg, _ = ctx.digest(s, strategy=L.PSB_GATHER, hmode=hmode, hs=hs, fp32c=fp32c)
            assert np.array_equal(cg, co) and np.array_equal(hg, ho)


def test_c2_plummer_full_size():
    d = W.plummer_c2()
    cols = [d["rho"], d["Ax"], d["Ay"], d["Az"]]
    ctx = make_ctx(d, d["h"], d["rho"], cols)
    spec = dict(scalars=[0], shepard=[0], grads=[0], divs=[1, 2, 3], curls=[1, 2, 3])
    ax = linrange(-0.5, 0.5, 128)
    g64 = ctx.interp_grid(ax, ax, ax, CatalogC(**spec), strategy=L.PSB_SYMMETRIC, prec=L.PSB_PREC_FP64)
    g32 = ctx.interp_grid(ax, ax, ax, CatalogC(**spec), strategy=L.PSB_SYMMETRIC, prec=L.PSB_PREC_FP32C)
    for k in range(8):  # the precision target: every field within 1e-6 of FP64
        assert rel_err(g32[k], g64[k]) <= 1e-6, (k, rel_err(g32[k], g64[k]))
    rng = np.random.default_rng(21)
    s_all = grid_points(ax, ax, ax)
    idx = rng.choice(len(s_all[0]), 200_000, replace=False)
    s = tuple(a[idx] for a in s_all)
    c64, h64, a64 = ctx.digest(s, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST)
    c32, h32, a32 = ctx.digest(s, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST, fp32c=True)
    assert np.array_equal(c64, c32) and np.array_equal(h64, h32) and np.array_equal(a64, a32)
    orc = O.Oracle(d["x"], d["y"], d["z"], d["m"], d["h"], d["rho"], cols)
    sub = idx[:20_000]
    ss = tuple(a[sub] for a in s_all)
    ref = orc.interp_points(*ss, O.Catalog(**spec), strategy=O.SYMMETRIC, hmode=O.H_NEAREST)
    for k in range(8):
        assert rel_err(g64[k][sub], ref[k]) <= 1e-12, k
    co, ho, _ = orc.digest(ss, strategy=O.SYMMETRIC, hmode=O.H_NEAREST)
    assert np.array_equal(co, c64[:20_000]) and np.array_equal(ho, h64[:20_000])


def test_c3_lines_full_size():
    d = W.clumps(8_000_000, 2)
    h, rho = W.density_h(d)
    ctx = make_ctx(d, h, rho, [rho])
    fr = W.c3_frame().as_array()
    prm = np.array([0.0, 1.0, 0.0, 1.0])
    npix = 1024
    cat = CatalogC(scalars=[0], shepard=[0])
    g32 = ctx.interp_beam(fr, prm, npix, npix, cat, strategy=L.PSB_SCATTER, prec=L.PSB_PREC_FP32C)
    g64 = ctx.interp_beam(fr, prm, npix, npix, cat, strategy=L.PSB_SCATTER, prec=L.PSB_PREC_FP64)
    assert rel_err(g32[0], g64[0]) <= 1e-6
    rng = np.random.default_rng(31)
    k = rng.choice(npix * npix, 2000, replace=False)
    ox = tuple(a[k] for a in W.plane_coordinates(fr, (0.0, 1.0, npix), (0.0, 1.0, npix)))
    fw = tuple(np.full(len(k), fr[9 + c]) for c in range(3))
    orc = O.Oracle(d["x"], d["y"], d["z"], d["m"], h, rho, [rho])
    ref = orc.interp_lines(ox, fw, [0], shepard=[0], strategy=O.SCATTER)
    assert rel_err(g64[0][k], ref[0]) <= 1e-12
    co, ho, _ = orc.digest(ox, fw, strategy=O.SCATTER, hmode=O.H_PER_SAMPLE, hs=np.zeros(len(k)))
    cg, hg, _ = ctx.digest(ox, fw, strategy=L.PSB_SCATTER, hmode=L.PSB_H_PER_SAMPLE, hs=np.zeros(len(k)))
    assert np.array_equal(cg, co) and np.array_equal(hg, ho)


def test_c4_adjoint_1m_particles():
    """Column density plus a Shepard-normalised quantity A (the A-gradient
    check of the configuration) on a 128^2 beam: dL/dm, dL/dA, dL/dx."""
    d = W.clumps(1_000_000, 3)
    h, rho = W.density_h(d)
    rng = np.random.default_rng(41)
    A = np.sin(5 * d["x"]) + d["y"] + 0.1 * rng.standard_normal(len(d["x"]))
    ctx = make_ctx(d, h, rho, [rho, A])
    orc = O.Oracle(d["x"], d["y"], d["z"], d["m"], h, rho, [rho, A])
    fr = W.c3_frame().as_array()
    prm = np.array([0.0, 1.0, 0.0, 1.0])
    npix = 128
    gout = [rng.standard_normal(npix * npix), rng.standard_normal(npix * npix)]
    g = ctx.adjoint_beam(fr, prm, npix, npix, CatalogC(scalars=[0, 1], shepard=[0, 1]), gout,
                         strategy=L.PSB_SCATTER)
    ox = W.plane_coordinates(fr, (0.0, 1.0, npix), (0.0, 1.0, npix))
    fw = tuple(np.full(npix * npix, fr[9 + c]) for c in range(3))
    threads = O.set_threads(0)
    O.set_threads(min(threads, 4))  # per-thread gradient buffers of 1M particles
    try:
        r = orc.adjoint_lines(ox, fw, [0, 1], gout, shepard=[0, 1], strategy=O.SCATTER)
    finally:
        O.set_threads(threads)
    for key in ("m", "x", "y", "z"):
        assert rel_err(g[key], r[key]) <= 1e-10, key
    for c in range(2):
        assert rel_err(g["cols"][c], r["cols"][c]) <= 1e-10, c


def test_c5_shaped_float_inputs():
    d = W.disc_halo_c5(4_000_000, 4)
    h, rho = W.density_h(d)
    cols = [rho, d["vx"], d["vy"], d["vz"], d["z2"]]
    ctx = make_ctx(d, h, rho, cols, dtype=np.float32)
    spec = dict(scalars=[0, 4], shepard=[0, 1], grads=[0], curls=[1, 2, 3])
    cat = CatalogC(**spec)
    ax = linrange(-1.0, 1.0, 64).astype(np.float32)
    g64 = ctx.interp_grid(ax, ax, ax, cat, strategy=L.PSB_SYMMETRIC, prec=L.PSB_PREC_FP64)
    g32 = ctx.interp_grid(ax, ax, ax, cat, strategy=L.PSB_SYMMETRIC, prec=L.PSB_PREC_FP32C)
    for k in range(len(g64)):
        assert rel_err(g32[k], g64[k]) <= 1e-5, (k, rel_err(g32[k], g64[k]))
    fr = W.Frame((0.1, -0.2, 0.0), (0.3, 0.2, 1.0), (1.0, 0.0, -0.3))
    fr.rotate(0.4, -0.3, 0.2)
    farr = fr.as_array().astype(np.float32)
    bprm = np.array([-0.5, 0.5, -0.5, 0.5, -0.5, 0.5], dtype=np.float32)
    gb = ctx.interp_box(farr, bprm, 32, 32, 32, cat, strategy=L.PSB_SYMMETRIC, prec=L.PSB_PREC_FP32C)
    assert np.isfinite(gb[0]).mean() > 0.5
    # oracle (float arithmetic, as the reference with Float32 inputs) on grid samples
    orc = O.Oracle(d["x"], d["y"], d["z"], d["m"], h, rho, cols, dtype=np.float32)
    rng = np.random.default_rng(51)
    s_all = grid_points(ax, ax, ax)
    idx = rng.choice(len(s_all[0]), 5000, replace=False)
    ss = tuple(a[idx] for a in s_all)
    ref = orc.interp_points(*ss, O.Catalog(**spec), strategy=O.SYMMETRIC, hmode=O.H_NEAREST)
    for k in range(len(ref)):
        assert rel_err(g64[k][idx], ref[k]) <= 2e-4, (k, rel_err(g64[k][idx], ref[k]))


def test_c5_shaped_adjoint_of_grid_scalar():
    """Gradient of the grid scalar's L2 norm (Shepard z^2) for 2M disc + halo
    particles (the float32 values in double).  At full grid size: S is linear
    in A and invariant under a common mass scaling, so <dL/dA, A> = <gout, S>
    and <dL/dm, m> = 0.  Against the oracle's adjoint with the cotangent on
    1500 random grid samples."""
    d = W.disc_halo_c5(2_000_000, 4)
    h, rho = W.density_h(d)
    dd = {k: np.asarray(d[k], dtype=np.float64) for k in ("x", "y", "z", "m", "z2")}
    h, rho = np.asarray(h, dtype=np.float64), np.asarray(rho, dtype=np.float64)
    cols = [rho, dd["z2"]]
    ctx = make_ctx(dd, h, rho, cols)
    spec = dict(scalars=[1], shepard=[1])
    ax = linrange(-1.0, 1.0, 48)
    S = ctx.interp_grid(ax, ax, ax, CatalogC(**spec), strategy=L.PSB_SYMMETRIC, prec=L.PSB_PREC_FP64)[0]
    S0 = np.nan_to_num(S, nan=0.0)
    gout = S0 / np.linalg.norm(S0)
    g = ctx.adjoint_grid(ax, ax, ax, CatalogC(**spec), [gout], strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST)
    lhs, rhs = float(np.dot(g["cols"][1], dd["z2"])), float(np.dot(gout, S0))
    assert abs(lhs - rhs) <= 1e-10 * abs(rhs), (lhs, rhs)
    gm = g["m"] * dd["m"]
    assert abs(gm.sum()) <= 1e-10 * np.abs(gm).sum()
    assert np.abs(g["cols"][0]).max() == 0  # column 0 enters only as rho_b
    # oracle on a subset of samples
    rng = np.random.default_rng(52)
    s_all = grid_points(ax, ax, ax)
    idx = rng.choice(len(S0), 1500, replace=False)
    gsub = np.zeros_like(gout)
    gsub[idx] = rng.standard_normal(len(idx))
    g2 = ctx.adjoint_grid(ax, ax, ax, CatalogC(**spec), [gsub], strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST)
    orc = O.Oracle(dd["x"], dd["y"], dd["z"], dd["m"], h, rho, cols)
    threads = O.set_threads(0)
    O.set_threads(min(threads, 4))  # per-thread gradient buffers of 2M particles
    try:
        r = orc.adjoint_points(*(a[idx] for a in s_all), O.Catalog(**spec), [gsub[idx]], strategy=O.SYMMETRIC,
                               hmode=O.H_NEAREST)
    finally:
        O.set_threads(threads)
    for key in ("m", "x", "y", "z"):
        assert rel_err(g2[key], r[key]) <= 1e-10, key
    assert rel_err(g2["cols"][1], r["cols"][1]) <= 1e-10


def test_c4_adjoint_finite_differences_at_config():
    """The configuration's own check: 1M clump particles (seed 3), the 512^2
    parallel beam through the 30/45-degree frame, L = 0.5 ||Sigma - Sigma_t||^2
    with Sigma_t rendered from masses m (1 + 0.1 N(0,1)) and positions
    displaced by 0.002 N(0,1); plus a Shepard-normalised quantity column for
    the A-gradient.  dL/dm_b, dL/dA_b and dL/dr_b from the adjoint against
    central differences of the GPU FP64 forward on 64 random particles with a
    nonzero gradient.  The difference of the loss is taken as gout . (out(+) -
    out(-)) with gout = out - target at the base point, which equals
    L(+) - L(-) up to O(eps^3) and keeps the rounding at the level of the
    per-pixel differences.  m (eps = 1e-6 relative) and A (1e-6 absolute)
    enter smoothly: tight agreement.  Positions move pairs along the
    piecewise-linear line-kernel table (segments of 2/4095 in q); at the
    configuration's eps = 1e-6, with h down to ~4e-4 in dense clumps, a pair's
    difference quotient can span several segments, so it agrees to the table's
    slope steps; at eps = 1e-8 it agrees tightly."""
    import torch
    d = W.clumps(1_000_000, 3)
    h, rho = W.density_h(d)
    n = len(d["x"])
    rng = np.random.default_rng(1003)
    A = np.sin(4 * d["x"]) + d["z"] + 0.05 * rng.standard_normal(n)
    fr = W.c3_frame().as_array()
    prm = np.array([0.0, 1.0, 0.0, 1.0])
    npix = 512
    cat = CatalogC(scalars=[0, 1], shepard=[0, 1])

    def render(ctx):
        out = [torch.empty(npix * npix, dtype=torch.float64, device="cuda") for _ in range(2)]
        ctx.interp_beam(fr, prm, npix, npix, cat, strategy=L.PSB_SCATTER, prec=L.PSB_PREC_FP64, out=out)
        return out

    # target image
    dt = dict(d)
    dt["m"] = d["m"] * (1.0 + 0.1 * rng.standard_normal(n))
    for k in ("x", "y", "z"):
        dt[k] = d[k] + 0.002 * rng.standard_normal(n)
    ctx_t = make_ctx(dt, h, rho, [rho, A])
    tgt = render(ctx_t)
    ctx_t.close()
    # base point, cotangents and the adjoint
    ctx = Context(0)
    ctx.set_particles(d["x"], d["y"], d["z"], d["m"], h, rho, [rho, A])
    perm, _ = ctx.build()
    pos = np.empty(n, dtype=np.int64)
    pos[perm] = np.arange(n)  # leaf position of each particle
    base = render(ctx)
    gout = [torch.nan_to_num(b - t) for b, t in zip(base, tgt)]
    g = ctx.adjoint_beam(fr, prm, npix, npix, cat, [go.cpu().numpy() for go in gout], strategy=L.PSB_SCATTER)
    # particles whose gradient stands above the difference quotients'
    # rounding floor (a pixel value of ~100 carries ~1e-14 of rounding, which
    # an eps of 1e-12 in m turns into ~1e-2 of the quotient)
    gmax = np.abs(g["m"]).max()
    live = np.flatnonzero(np.abs(g["m"]) >= 1e-4 * gmax)
    assert len(live) > 1000
    picks = rng.choice(live, 64, replace=False)

    def dot(outs):
        return sum(float((go * torch.nan_to_num(o)).sum()) for go, o in zip(gout, outs))

    # values (m, A): the tree is unchanged, only the values are replaced
    leaf = {"m": d["m"][perm].copy(), "rho": rho[perm].copy(), "A": A[perm].copy(), "r": rho[perm].copy()}

    def values_fd(b, key, eps):
        res = []
        for sgn in (1.0, -1.0):
            arr = leaf[key].copy()
            arr[pos[b]] += sgn * eps
            mm = arr if key == "m" else leaf["m"]
            aa = arr if key == "A" else leaf["A"]
            ctx.set_values(mm, leaf["rho"], [leaf["r"], aa])
            res.append(dot(render(ctx)))
        return (res[0] - res[1]) / (2 * eps)

    sm, sa = np.abs(g["m"]).max(), np.abs(g["cols"][1]).max()
    for b in picks:
        fd = values_fd(b, "m", 1e-6 * d["m"][b])
        assert abs(fd - g["m"][b]) <= 1e-6 * abs(g["m"][b]) + 1e-8 * sm, ("m", b, fd, g["m"][b])
        fd = values_fd(b, "A", 1e-6)
        assert abs(fd - g["cols"][1][b]) <= 1e-6 * abs(g["cols"][1][b]) + 1e-8 * sa, ("A", b, fd, g["cols"][1][b])
    ctx.set_values(leaf["m"], leaf["rho"], [leaf["r"], leaf["A"]])

    # positions: a second context rebuilt for every displaced input
    ctx2 = Context(0)
    coords = {k: d[k].copy() for k in ("x", "y", "z")}

    def pos_fd(b, key, eps):
        res = []
        for sgn in (1.0, -1.0):
            c = coords[key].copy()
            c[b] += sgn * eps
            cc = dict(coords)
            cc[key] = c
            ctx2.set_particles(cc["x"], cc["y"], cc["z"], d["m"], h, rho, [rho, A])
            ctx2.build(want_perm=False)
            res.append(dot(render(ctx2)))
        return (res[0] - res[1]) / (2 * eps)

    loose = 0
    for key in ("x", "y", "z"):
        sc = np.abs(g[key]).max()
        for b in picks:
            fd8 = pos_fd(b, key, 1e-8)
            assert abs(fd8 - g[key][b]) <= 1e-4 * abs(g[key][b]) + 1e-6 * sc, (key, b, fd8, g[key][b])
            fd6 = pos_fd(b, key, 1e-6)
            if abs(fd6 - g[key][b]) > 2e-3 * abs(g[key][b]) + 1e-5 * sc:
                loose += 1
    # at eps = 1e-6 nearly every particle agrees to the table's slope steps
    assert loose <= 8, loose
