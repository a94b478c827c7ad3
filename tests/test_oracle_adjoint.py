"""Oracle adjoint against central finite differences of the oracle forward.

The reference has no adjoint.  The oracle's vector-Jacobian product (the
checker of the GPU adjoint) is pinned here by central differences of the
restated forward pass for L = sum_k sum_s gout[k][s] out_k(s), with respect to
particle masses, columns and positions, for point samples (all three
strategies, every output kind, given h_a) and for line-integrated samples.
Position steps re-run the LBVH build on the perturbed coordinates.
"""
import numpy as np
import pytest

import oracle as O

CAT = dict(scalars=[0, 1, 3], shepard=[0, 1, 1], grads=[-1, 1], divs=[1, 2, 3], curls=[3, 2, 1])


def particles(n, seed):
    rng = np.random.default_rng(seed)
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    m = rng.uniform(0.5, 1.5, n) / n
    h = 1.3 * (1.0 / n) ** (1 / 3) * rng.uniform(0.7, 1.4, n)
    rho = rng.uniform(0.5, 2.0, n)
    cols = [rho.copy(), np.sin(3 * x) + y, -y + 0.3 * z, x * x + 0.2 * rng.standard_normal(n)]
    return [x, y, z, m, h, rho], cols


def loss_points(arrs, cols, s, cat, gout, strategy, hs):
    orc = O.Oracle(*arrs, cols=cols)
    out = orc.interp_points(*s, O.Catalog(**cat), strategy=strategy, hmode=O.H_PER_SAMPLE, hs=hs)
    return sum(float(np.sum(np.nan_to_num(o) * g)) for o, g in zip(out, gout))


def fd(fun, base, eps):
    return (fun(base + eps) - fun(base - eps)) / (2 * eps)


@pytest.mark.parametrize("strategy", [O.GATHER, O.SCATTER, O.SYMMETRIC])
def test_point_adjoint_matches_central_differences(strategy):
    arrs, cols = particles(500, 11)
    rng = np.random.default_rng(12)
    ns = 80
    s = tuple(rng.uniform(0.1, 0.9, ns) for _ in range(3))
    hs = rng.uniform(0.06, 0.1, ns)
    L = O.Catalog(**CAT).L
    gout = [rng.standard_normal(ns) for _ in range(L)]
    orc = O.Oracle(*arrs, cols=cols)
    g = orc.adjoint_points(*s, O.Catalog(**CAT), gout, strategy=strategy, hmode=O.H_PER_SAMPLE, hs=hs)
    # particles that sit inside some support
    cand = np.flatnonzero(np.abs(g["m"]) > 0)
    assert len(cand) > 50
    for b in rng.choice(cand, 6, replace=False):
        def with_arr(k, eps):
            a2 = [a.copy() for a in arrs]
            a2[k][b] += eps
            return loss_points(a2, cols, s, CAT, gout, strategy, hs)

        def with_col(c, eps):
            c2 = [cc.copy() for cc in cols]
            c2[c][b] += eps
            return loss_points(arrs, c2, s, CAT, gout, strategy, hs)

        em = 1e-6 * arrs[3][b]
        assert fd(lambda e: with_arr(3, e), 0.0, em) == pytest.approx(g["m"][b], rel=1e-5, abs=1e-7 * abs(g["m"]).max())
        for k, key in ((0, "x"), (1, "y"), (2, "z")):
            got = fd(lambda e: with_arr(k, e), 0.0, 1e-7)
            assert got == pytest.approx(g[key][b], rel=1e-4, abs=1e-6 * abs(g[key]).max()), (b, key)
        for c in range(len(cols)):
            got = fd(lambda e: with_col(c, e), 0.0, 1e-6)
            assert got == pytest.approx(g["cols"][c][b], rel=1e-5, abs=1e-8 * abs(g["cols"][c]).max() + 1e-14)


def test_line_adjoint_matches_central_differences():
    arrs, cols = particles(600, 21)
    rng = np.random.default_rng(22)
    nl = 120
    o = (rng.uniform(0.1, 0.9, nl), rng.uniform(0.1, 0.9, nl), np.full(nl, -0.2))
    d = rng.standard_normal((3, nl)) * 0.2
    d[2] = 1.0
    d /= np.linalg.norm(d, axis=0)
    scal, shep = [0, 1], [0, 1]
    gout = [rng.standard_normal(nl) for _ in scal]

    def loss(a2, c2):
        orc = O.Oracle(*a2, cols=c2)
        out = orc.interp_lines(o, tuple(d), scal, shepard=shep, strategy=O.SCATTER)
        return sum(float(np.sum(np.nan_to_num(v) * g)) for v, g in zip(out, gout))

    orc = O.Oracle(*arrs, cols=cols)
    g = orc.adjoint_lines(o, tuple(d), scal, gout, shepard=shep, strategy=O.SCATTER)
    cand = np.flatnonzero(np.abs(g["m"]) > 0)
    assert len(cand) > 50
    for b in rng.choice(cand, 6, replace=False):
        def with_arr(k, eps):
            a2 = [a.copy() for a in arrs]
            a2[k][b] += eps
            return loss(a2, cols)

        em = 1e-6 * arrs[3][b]
        assert fd(lambda e: with_arr(3, e), 0.0, em) == pytest.approx(g["m"][b], rel=1e-5)
        for k, key in ((0, "x"), (1, "y"), (2, "z")):
            # the table is piecewise linear: the step stays well inside one segment
            got = fd(lambda e: with_arr(k, e), 0.0, 1e-9)
            assert got == pytest.approx(g[key][b], rel=2e-4, abs=1e-5 * abs(g[key]).max()), (b, key)
        c2 = [cc.copy() for cc in cols]
        for c in (0, 1):
            base = cols[c][b]

            def with_col(eps, c=c):
                c3 = [cc.copy() for cc in cols]
                c3[c][b] = base + eps
                return loss(arrs, c3)

            assert fd(with_col, 0.0, 1e-6) == pytest.approx(g["cols"][c][b], rel=1e-5, abs=1e-12)
