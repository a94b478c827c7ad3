"""Oracle pins on the reference's deterministic interpolation fixtures.

 * 4-particle fixture + 3 point samples, symmetric, nearest-particle h,
   scalar + divergence vs brute force at rtol 1e-10
   (test/point_samples_interpolation_tests.jl:53-79,
    test/grid_interpolation_test_common.jl:40-71)
 * line fixture + 3 lines, scatter, line-integrated scalars vs brute force at
   rtol 1e-10 (test/point_samples_interpolation_tests.jl:121-155,
   test/grid_interpolation_test_common.jl:108-144)
 * 12^3 lattice with variable h, analytic linear fields, all three
   strategies, the reference's atol/rtol
   (test/point_samples_interpolation_tests.jl:211-239,
    test/interpolation_analytic_test_common.jl:31-75)
 * uniform 8^3 and 12^3 lattices, constant h: mean errors of Shepard q,
   grad q, div v, curl v, rho and grad rho against the analytic fields,
   pooled over the three strategies (test/traversal_analytic.jl:48-101)
 * uniform vector field: divergence = curl = 0 to 1e-12
   (test/interpolation_tests.jl:305-336)
 * empty neighbourhoods: density 0, every other field NaN
   (test/interpolation_tests.jl:52-117)
"""
import math

import numpy as np
import pytest

import bruteforce as B
import oracle as O


def fixture_points():
    P = dict(x=np.array([0.15, 0.35, 0.55, 0.75]), y=np.array([0.20, 0.60, 0.25, 0.70]),
             z=np.array([0.25, 0.45, 0.80, 0.30]), h=np.array([0.28, 0.24, 0.26, 0.22]),
             rho=np.array([1.0, 0.95, 1.05, 1.1]), m=np.array([0.4, 0.45, 0.42, 0.38]))
    cols = [np.array([10.0, 11.0, 13.0, 12.0]), np.array([0.1, -0.2, 0.3, -0.1]),
            np.array([0.0, 0.25, -0.15, 0.2]), np.array([-0.05, 0.1, 0.2, -0.1])]
    return P, cols


def make_oracle(P, cols):
    return O.Oracle(P["x"], P["y"], P["z"], P["m"], P["h"], P["rho"], cols)


def test_point_fixture_symmetric_nearest_h():
    P, cols = fixture_points()
    orc = make_oracle(P, cols)
    s = (np.array([0.20, 0.40, 0.65]), np.array([0.25, 0.55, 0.50]), np.array([0.30, 0.50, 0.35]))
    cat = O.Catalog(scalars=[0], shepard=[1], divs=[1, 2, 3])
    out = orc.interp_points(*s, cat, strategy=O.SYMMETRIC, hmode=O.H_NEAREST)
    for i in range(3):
        p = np.array([s[0][i], s[1][i], s[2][i]])
        ha = B.nearest_h(P, p)
        ref = B.general(P, cols, p, ha, "symmetric", scalars=[0], shepard=[1], divs=[(1, 2, 3)])
        assert out[0][i] == pytest.approx(ref[0], rel=1e-10, abs=1e-12)
        assert out[1][i] == pytest.approx(ref[1], rel=1e-10, abs=1e-12)


@pytest.mark.parametrize("strategy,name", [(O.GATHER, "gather"), (O.SCATTER, "scatter"), (O.SYMMETRIC, "symmetric")])
def test_point_fixture_all_fields(strategy, name):
    P, cols = fixture_points()
    orc = make_oracle(P, cols)
    rng = np.random.default_rng(3)
    s = tuple(rng.uniform(0.1, 0.8, 20) for _ in range(3))
    spec = dict(scalars=[0, 1], shepard=[1, 0], grads=[0, -1], divs=[(1, 2, 3)], curls=[(1, 2, 3)])
    cat = O.Catalog(scalars=spec["scalars"], shepard=spec["shepard"], grads=spec["grads"],
                    divs=[c for t in spec["divs"] for c in t], curls=[c for t in spec["curls"] for c in t])
    out = orc.interp_points(*s, cat, strategy=strategy, hmode=O.H_NEAREST)
    for i in range(20):
        p = np.array([s[0][i], s[1][i], s[2][i]])
        ha = B.nearest_h(P, p)
        ref = B.general(P, cols, p, ha, name, **spec)
        got = [o[i] for o in out]
        for a, b in zip(got, ref):
            if math.isnan(b):
                assert math.isnan(a)
            else:
                assert a == pytest.approx(b, rel=1e-10, abs=1e-12)


def test_line_fixture_scatter():
    P, cols = fixture_points()
    cols = cols[:2]
    orc = make_oracle(P, cols)
    r2 = 1 / math.sqrt(2.0)
    o = (np.array([0.20, 0.40, 0.55]), np.array([0.25, 0.35, 0.45]), np.array([0.00, 0.10, 0.20]))
    d = (np.array([0.0, r2, 1.0]), np.array([0.0, 0.0, 0.0]), np.array([1.0, r2, 0.0]))
    out = orc.interp_lines(o, d, scalars=[0, 1], shepard=[1, 1], strategy=O.SCATTER)
    table = O.line_table()
    for i in range(3):
        ref = B.line_quantities(P, cols, [o[k][i] for k in range(3)], [d[k][i] for k in range(3)], 0.0, "scatter",
                                [0, 1], [1, 1], table)
        assert out[0][i] == pytest.approx(ref[0], rel=1e-10, abs=1e-12)
        assert out[1][i] == pytest.approx(ref[1], rel=1e-10, abs=1e-12)


def lattice(nx=12, eta=1.2, variable_h=True):
    dx = 1.0 / nx
    c = np.arange(dx / 2, 1.0 - dx / 2 + 1e-12, dx)
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")   # x outermost, z fastest, as the Julia loop
    x, y, z = X.ravel(), Y.ravel(), Z.ravel()
    n = len(x)
    if variable_h:
        h = eta * dx * (1.0 + 0.18 * (x - 0.5) - 0.10 * (y - 0.5) + 0.08 * (z - 0.5))
    else:
        h = np.full(n, eta * dx)
    P = dict(x=x, y=y, z=z, m=np.full(n, dx ** 3), h=h, rho=np.ones(n))
    cols = [x + y + z, x.copy(), y.copy(), z.copy()]
    return P, cols


@pytest.mark.parametrize("strategy", [O.GATHER, O.SCATTER, O.SYMMETRIC])
def test_analytic_linear_fields(strategy):
    P, cols = lattice()
    orc = make_oracle(P, cols)
    s = (np.array([0.35, 0.45, 0.55]), np.array([0.40, 0.50, 0.45]), np.array([0.45, 0.35, 0.50]))
    cat = O.Catalog(scalars=[0], shepard=[1], grads=[0], divs=[1, 2, 3], curls=[1, 2, 3])
    out = orc.interp_points(*s, cat, strategy=strategy, hmode=O.H_NEAREST)
    for i in range(3):
        p = [s[0][i], s[1][i], s[2][i]]
        assert out[0][i] == pytest.approx(sum(p), abs=2e-2, rel=1e-2)
        for k in (1, 2, 3):
            assert out[k][i] == pytest.approx(1.0, abs=6e-2, rel=1e-2)
        assert out[4][i] == pytest.approx(3.0, abs=1e-1, rel=2e-2)
        for k in (5, 6, 7):
            assert out[k][i] == pytest.approx(0.0, abs=5e-2)


# catalog of the analytic traversal regression: Shepard q, grad q, grad rho,
# div v, curl v (outputs 0 | 1-3 | 4-6 | 7 | 8-10)
ANALYTIC_CAT = dict(scalars=[0], shepard=[1], grads=[0, -1], divs=[1, 2, 3], curls=[1, 2, 3])
# mean-absolute-error bounds of test/traversal_analytic.jl:94-99
ANALYTIC_BOUNDS = dict(scalar=2e-2, grad=6e-2, div=1e-1, curl=5e-2, rho=5e-2, grad_rho=5e-2)


def analytic_refs(nx, eta=1.2, n=12, seed=0xA11CE):
    """n reference points at least 1.5 K h from the cube's faces (K = 2 for
    M4), as sample_reference_points (test/interpolation_analytic_test_common.jl:75-87),
    drawn from numpy's PCG64 instead of Julia's Xoshiro."""
    h = eta / nx
    lo, hi = 1.5 * 2.0 * h, 1.0 - 1.5 * 2.0 * h
    r = np.random.default_rng(seed).random((n, 3)) * (hi - lo) + lo
    return h, r[:, 0].copy(), r[:, 1].copy(), r[:, 2].copy()


def analytic_errors(outs, rho, sx, sy, sz):
    """Per-sample errors against q = x + y + z, grad q = (1,1,1), v = r
    (div 3, curl 0) and the uniform density 1 with zero gradient."""
    o = [np.asarray(a, dtype=np.float64) for a in outs]
    return dict(scalar=np.abs(o[0] - (sx + sy + sz)),
                grad=np.sqrt((o[1] - 1) ** 2 + (o[2] - 1) ** 2 + (o[3] - 1) ** 2),
                div=np.abs(o[7] - 3.0),
                curl=np.sqrt(o[8] ** 2 + o[9] ** 2 + o[10] ** 2),
                rho=np.abs(np.asarray(rho, dtype=np.float64) - 1.0),
                grad_rho=np.sqrt(o[4] ** 2 + o[5] ** 2 + o[6] ** 2))


@pytest.mark.parametrize("nx", [8, 12])
def test_traversal_analytic_mean_errors(nx):
    """test/traversal_analytic.jl:48-101: uniform lattice (eta 1.2, constant h),
    12 interior reference points, errors pooled over the three strategies."""
    P, cols = lattice(nx, variable_h=False)
    orc = make_oracle(P, cols)
    h, sx, sy, sz = analytic_refs(nx)
    cat = O.Catalog(**ANALYTIC_CAT)
    pooled = {k: [] for k in ANALYTIC_BOUNDS}
    for st in (O.GATHER, O.SCATTER, O.SYMMETRIC):
        outs = orc.interp_points(sx, sy, sz, cat, strategy=st, hmode=O.H_CONSTANT, hs=np.array([h]))
        rho = orc.density(sx, sy, sz, strategy=st, hmode=O.H_CONSTANT, hs=np.array([h]))
        for k, v in analytic_errors(outs, rho, sx, sy, sz).items():
            pooled[k].append(v)
    for k, bound in ANALYTIC_BOUNDS.items():
        err = np.concatenate(pooled[k])
        assert np.all(np.isfinite(err)), k
        assert float(np.mean(err)) <= bound, (k, float(np.mean(err)))


@pytest.mark.parametrize("strategy", [O.GATHER, O.SCATTER, O.SYMMETRIC])
def test_uniform_field_div_curl_vanish(strategy):
    x = np.array([0.0, 0.05, 0.11, -0.08])
    y = np.array([0.02, -0.03, 0.04, 0.01])
    z = np.array([0.0, 0.01, -0.02, 0.03])
    n = 4
    cols = [np.full(n, 1.0), np.full(n, -2.0), np.full(n, 0.5)]
    orc = O.Oracle(x, y, z, np.ones(n), np.full(n, 0.12), np.ones(n), cols)
    cat = O.Catalog(divs=[0, 1, 2], curls=[0, 1, 2])
    out = orc.interp_points(x[:1], y[:1], z[:1], cat, strategy=strategy, hmode=O.H_PER_SAMPLE, hs=[0.12])
    for o in out:
        assert abs(o[0]) <= 1e-12


def test_empty_neighbourhood_semantics():
    P, cols = fixture_points()
    orc = make_oracle(P, cols)
    far = (np.array([9.0]), np.array([9.0]), np.array([9.0]))
    cat = O.Catalog(scalars=[0], shepard=[1], grads=[0], divs=[1, 2, 3], curls=[1, 2, 3])
    out = orc.interp_points(*far, cat, strategy=O.SCATTER)
    assert all(math.isnan(o[0]) for o in out)
    assert orc.density(*far, strategy=O.SCATTER)[0] == 0.0
    lo = orc.interp_lines(far, (np.array([1.0]), np.array([0.0]), np.array([0.0])), scalars=[0], strategy=O.SCATTER)
    assert math.isnan(lo[0][0])


def test_density_kernel_matches_brute_force():
    P, cols = lattice(8)
    orc = make_oracle(P, cols)
    rng = np.random.default_rng(5)
    s = tuple(rng.uniform(0.1, 0.9, 10) for _ in range(3))
    ha = rng.uniform(0.1, 0.2, 10)
    got = orc.density(*s, strategy=O.GATHER, hmode=O.H_PER_SAMPLE, hs=ha)
    for i in range(10):
        p = np.array([s[0][i], s[1][i], s[2][i]])
        sel, d, r, hb = B._neighbours(P, p, ha[i], "gather")
        assert got[i] == pytest.approx(np.sum(P["m"][sel] * B.W(r, ha[i])), rel=1e-12)


@pytest.mark.parametrize("kid", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("strategy,name", [(O.GATHER, "gather"), (O.SCATTER, "scatter"), (O.SYMMETRIC, "symmetric")])
def test_other_kernels_points_vs_brute_force(kid, strategy, name):
    """M5, M6 and the Wendland kernels (kernels/*.jl): support K h, weights and
    gradients of each family, every output kind, against brute force."""
    rng = np.random.default_rng(40 + kid)
    n = 400
    P = dict(x=rng.random(n), y=rng.random(n), z=rng.random(n), m=rng.uniform(0.5, 1.5, n) / n,
             h=0.09 * rng.uniform(0.7, 1.4, n), rho=rng.uniform(0.8, 1.2, n))
    cols = [rng.uniform(1, 2, n), np.sin(3 * P["x"]) + P["y"], P["y"] - P["z"], P["x"] * P["z"]]
    orc = O.Oracle(P["x"], P["y"], P["z"], P["m"], P["h"], P["rho"], cols, kernel=kid)
    s = tuple(rng.uniform(0.1, 0.9, 25) for _ in range(3))
    spec = dict(scalars=[0, 1], shepard=[1, 0], grads=[0, -1], divs=[(1, 2, 3)], curls=[(1, 2, 3)])
    cat = O.Catalog(scalars=spec["scalars"], shepard=spec["shepard"], grads=spec["grads"],
                    divs=[c for t in spec["divs"] for c in t], curls=[c for t in spec["curls"] for c in t])
    out = orc.interp_points(*s, cat, strategy=strategy, hmode=O.H_NEAREST)
    B.set_kernel(kid)
    try:
        for i in range(25):
            p = np.array([s[0][i], s[1][i], s[2][i]])
            ref = B.general(P, cols, p, B.nearest_h(P, p), name, **spec)
            for a, b in zip([o[i] for o in out], ref):
                if math.isnan(b):
                    assert math.isnan(a)
                else:
                    assert a == pytest.approx(b, rel=1e-10, abs=1e-10 * max(1.0, abs(b)))
        # line-integrated scalars with the family's own table
        o = (rng.uniform(0.1, 0.9, 6), rng.uniform(0.1, 0.9, 6), np.zeros(6))
        d = (np.zeros(6), np.zeros(6), np.ones(6))
        lo = orc.interp_lines(o, d, scalars=[0, 1], shepard=[1, 0], strategy=O.SCATTER)
        table = O.line_table(kid)
        for i in range(6):
            ref = B.line_quantities(P, cols, [o[k][i] for k in range(3)], [d[k][i] for k in range(3)], 0.0,
                                    "scatter", [0, 1], [1, 0], table)
            assert lo[0][i] == pytest.approx(ref[0], rel=1e-10, abs=1e-12)
            assert lo[1][i] == pytest.approx(ref[1], rel=1e-10, abs=1e-12)
    finally:
        B.set_kernel(0)


@pytest.mark.parametrize("strategy,name", [(O.GATHER, "gather"), (O.SCATTER, "scatter"), (O.SYMMETRIC, "symmetric")])
def test_number_density_and_plain_density_gradient_vs_brute_force(strategy, name):
    """_number_density_kernel (scalar_interpolation.jl:86-166) and the standalone
    _gradient_density_kernel (gradient_interpolation.jl:1-170): sum W, and
    sum m gradW - rho(r) sum (m/rho_b) gradW with rho(r) = sum m W (NaN where
    rho(r) = 0), against brute force."""
    P, cols = lattice(8)
    P = dict(P)
    rng = np.random.default_rng(17)
    P["m"] = P["m"] * rng.uniform(0.5, 1.5, len(P["m"]))
    P["rho"] = rng.uniform(0.7, 1.3, len(P["m"]))
    orc = make_oracle(P, cols)
    s = tuple(np.append(rng.uniform(0.1, 0.9, 12), 9.0) for _ in range(3))  # the last sample has no neighbour
    ha = np.append(rng.uniform(0.1, 0.2, 12), 0.1)
    nd = orc.density(*s, strategy=strategy, hmode=O.H_PER_SAMPLE, hs=ha, number=True)
    gd = orc.gradient_density(*s, strategy=strategy, hmode=O.H_PER_SAMPLE, hs=ha)
    for i in range(13):
        p = np.array([s[0][i], s[1][i], s[2][i]])
        sel, d, r, hb = B._neighbours(P, p, ha[i], name)
        Wv, G = B._weights(d, r, hb, ha[i], name)
        assert nd[i] == pytest.approx(np.sum(Wv), rel=1e-12, abs=0)
        rho = np.sum(P["m"][sel] * Wv)
        if rho == 0:
            assert np.all(np.isnan(gd[:, i]))
            continue
        f_ = np.sum(P["m"][sel] * G, axis=1)
        b_ = np.sum(P["m"][sel] * G / P["rho"][sel], axis=1)
        ref = f_ - b_ * rho
        np.testing.assert_allclose(gd[:, i], ref, rtol=1e-10, atol=1e-12 * np.max(np.abs(f_)))
    assert nd[12] == 0.0
