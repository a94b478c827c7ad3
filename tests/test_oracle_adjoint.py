"""Oracle adjoint against central finite differences of the oracle forward.

The reference has no adjoint.  The oracle's vector-Jacobian product (the
checker of the GPU adjoint) is pinned here by central differences of the
restated forward pass for L = sum_k sum_s gout[k][s] out_k(s), with respect to
particle masses, columns and positions, for point samples (all three
strategies, every output kind, given h_a) and for line-integrated samples,
with the M4 kernel and with each of M5, M6 and Wendland C2/C4/C6.
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


def loss_points(arrs, cols, s, cat, gout, strategy, hs, kernel=O.M4):
    orc = O.Oracle(*arrs, cols=cols, kernel=kernel)
    out = orc.interp_points(*s, O.Catalog(**cat), strategy=strategy, hmode=O.H_PER_SAMPLE, hs=hs)
    return sum(float(np.sum(np.nan_to_num(o) * g)) for o, g in zip(out, gout))


def fd(fun, base, eps):
    return (fun(base + eps) - fun(base - eps)) / (2 * eps)


@pytest.mark.parametrize("strategy,kernel", [(O.GATHER, O.M4), (O.SCATTER, O.M4), (O.SYMMETRIC, O.M4),
                                             (O.SYMMETRIC, O.M5), (O.SYMMETRIC, O.M6), (O.GATHER, O.C2),
                                             (O.SYMMETRIC, O.C4), (O.SCATTER, O.C6)])
def test_point_adjoint_matches_central_differences(strategy, kernel):
    arrs, cols = particles(500, 11)
    rng = np.random.default_rng(12)
    ns = 80
    s = tuple(rng.uniform(0.1, 0.9, ns) for _ in range(3))
    hs = rng.uniform(0.06, 0.1, ns)
    L = O.Catalog(**CAT).L
    gout = [rng.standard_normal(ns) for _ in range(L)]
    orc = O.Oracle(*arrs, cols=cols, kernel=kernel)
    g = orc.adjoint_points(*s, O.Catalog(**CAT), gout, strategy=strategy, hmode=O.H_PER_SAMPLE, hs=hs)
    # particles that sit inside some support
    cand = np.flatnonzero(np.abs(g["m"]) > 0)
    assert len(cand) > 50
    for b in rng.choice(cand, 6, replace=False):
        def with_arr(k, eps):
            a2 = [a.copy() for a in arrs]
            a2[k][b] += eps
            return loss_points(a2, cols, s, CAT, gout, strategy, hs, kernel)

        def with_col(c, eps):
            c2 = [cc.copy() for cc in cols]
            c2[c][b] += eps
            return loss_points(arrs, c2, s, CAT, gout, strategy, hs, kernel)

        em = 1e-6 * arrs[3][b]
        assert fd(lambda e: with_arr(3, e), 0.0, em) == pytest.approx(g["m"][b], rel=1e-5, abs=1e-7 * abs(g["m"]).max())
        for k, key in ((0, "x"), (1, "y"), (2, "z")):
            got = fd(lambda e: with_arr(k, e), 0.0, 1e-7)
            assert got == pytest.approx(g[key][b], rel=1e-4, abs=1e-6 * abs(g[key]).max()), (b, key)
        for c in range(len(cols)):
            got = fd(lambda e: with_col(c, e), 0.0, 1e-6)
            assert got == pytest.approx(g["cols"][c][b], rel=1e-5, abs=1e-8 * abs(g["cols"][c]).max() + 1e-14)


@pytest.mark.parametrize("kernel", [O.M4, O.M5, O.C4])
def test_line_adjoint_matches_central_differences(kernel):
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
        orc = O.Oracle(*a2, cols=c2, kernel=kernel)
        out = orc.interp_lines(o, tuple(d), scal, shepard=shep, strategy=O.SCATTER)
        return sum(float(np.sum(np.nan_to_num(v) * g)) for v, g in zip(out, gout))

    orc = O.Oracle(*arrs, cols=cols, kernel=kernel)
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


class Dual:
    """Forward-mode dual numbers over numpy: value v (shape s) and
    derivatives d (shape s + (k,)) with respect to k seeded parameters."""

    __array_ufunc__ = None  # ndarray (op) Dual defers to the Dual's reflected operators

    def __init__(self, v, d):
        self.v = np.asarray(v, dtype=float)
        self.d = np.asarray(d, dtype=float)

    @staticmethod
    def _p(o, like):
        return o if isinstance(o, Dual) else Dual(np.broadcast_to(o, like.v.shape), np.zeros(like.d.shape))

    def __add__(self, o):
        o = Dual._p(o, self)
        return Dual(self.v + o.v, self.d + o.d)

    __radd__ = __add__

    def __sub__(self, o):
        o = Dual._p(o, self)
        return Dual(self.v - o.v, self.d - o.d)

    def __rsub__(self, o):
        return Dual._p(o, self) - self

    def __mul__(self, o):
        o = Dual._p(o, self)
        return Dual(self.v * o.v, self.d * o.v[..., None] + o.d * self.v[..., None])

    __rmul__ = __mul__

    def __truediv__(self, o):
        o = Dual._p(o, self)
        return Dual(self.v / o.v, (self.d * o.v[..., None] - o.d * self.v[..., None]) / (o.v ** 2)[..., None])

    def sqrt(self):
        s = np.sqrt(self.v)
        with np.errstate(divide="ignore", invalid="ignore"):
            g = np.where(s > 0, 0.5 / s, 0.0)
        return Dual(s, self.d * g[..., None])


def test_line_adjoint_matches_forward_mode_dual_numbers():
    """The configuration's ForwardDiff check, restated: forward-mode dual
    numbers through a brute-force column density and a Shepard-normalised
    quantity (the table lookup of line_integrated_kernel.jl:13-19 differentiated
    as ForwardDiff would: the slope of the segment) for 16 particles of a
    20,000-particle set, against the oracle's adjoint."""
    from partia_b200 import workloads as W
    rng = np.random.default_rng(61)
    n = 20_000
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    m = rng.uniform(0.5, 1.5, n) / n
    h = 1.3 * (1.0 / n) ** (1 / 3) * rng.uniform(0.7, 1.4, n)
    rho = rng.uniform(0.5, 2.0, n)
    A = np.sin(3 * x) + y + 0.1 * rng.standard_normal(n)
    cols = [rho.copy(), A]
    fr = W.c3_frame().as_array()
    npix = 40
    o = W.plane_coordinates(fr, (0.0, 1.0, npix), (0.0, 1.0, npix))
    mdir = fr[9:12]
    nl = npix * npix
    gout = [rng.standard_normal(nl), rng.standard_normal(nl)]
    orc = O.Oracle(x, y, z, m, h, rho, cols=cols)
    g = orc.adjoint_lines(o, tuple(np.full(nl, mdir[c]) for c in range(3)), [0, 1], gout, shepard=[0, 1],
                          strategy=O.SCATTER)
    Q, I = O.line_table()
    dq = Q[1] - Q[0]

    def weight(px, py, pz, mb, hb, rb):
        """(m/rho) W_line for one particle (Dual or float coordinates) and every line."""
        D = [px - o[0], py - o[1], pz - o[2]]
        Dm = D[0] * mdir[0] + D[1] * mdir[1] + D[2] * mdir[2]
        d2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2] - Dm * Dm
        v = d2.v if isinstance(d2, Dual) else d2
        d2 = d2 * np.where(v > 0, 1.0, 0.0)  # clamp at 0 as the reference's caller
        dperp = d2.sqrt() if isinstance(d2, Dual) else np.sqrt(d2)
        q = dperp * (1.0 / hb)
        idxf = q * (1.0 / dq) + 1.0
        iv = idxf.v if isinstance(idxf, Dual) else idxf
        i = np.clip(np.trunc(iv).astype(np.int64), 1, len(Q) - 1)
        t = idxf - i
        Wl = (I[i - 1] * (1.0 - t) + I[i] * t) * (1.0 / hb)
        qv = q.v if isinstance(q, Dual) else q
        return Wl * np.where(qv < 2.0, 1.0, 0.0) * mb * (1.0 / rb)

    # sums over every particle (values)
    S0 = np.zeros(nl)
    num = np.zeros(nl)
    den = np.zeros(nl)
    for b in range(n):
        w = weight(x[b], y[b], z[b], m[b], h[b], rho[b])
        S0 += w * cols[0][b]
        num += w * A[b]
        den += w
    ok = den > 0
    for b in rng.choice(np.flatnonzero(np.abs(g["m"]) > 0), 16, replace=False):
        # seeds: m, x, y, z, A of particle b
        e = np.eye(5)
        P = [Dual(np.full(nl, v), np.tile(e[k], (nl, 1))) for k, v in enumerate((m[b], x[b], y[b], z[b], A[b]))]
        w = weight(P[1], P[2], P[3], P[0], h[b], rho[b])
        w0 = weight(x[b], y[b], z[b], m[b], h[b], rho[b])
        # the sums with particle b's term as a dual
        s0 = Dual(S0 - w0 * cols[0][b], np.zeros((nl, 5))) + w * cols[0][b]
        nu = Dual(num - w0 * A[b], np.zeros((nl, 5))) + w * P[4]
        de = Dual(den - w0, np.zeros((nl, 5))) + w
        sh = nu / Dual(np.where(ok, de.v, 1.0), de.d)
        dL = (gout[0][:, None] * s0.d).sum(0) + (np.where(ok, gout[1], 0.0)[:, None] * sh.d).sum(0)
        got = [g["m"][b], g["x"][b], g["y"][b], g["z"][b], g["cols"][1][b]]
        for k in range(5):
            assert got[k] == pytest.approx(dL[k], rel=1e-8, abs=1e-10 * abs(dL).max()), (b, k, got[k], dL[k])
