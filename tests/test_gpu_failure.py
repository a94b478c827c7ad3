"""Failure detection and determinism on the GPU.

 * Bounded walks: psb_test_loop_escapes points every walk-ending escape link
   of the particle LBVH at the root (ids stay valid, so no access leaves its
   buffer).  Every traversal then cycles until its 4n + 8 step bound; each
   call kind must return PSB_ETRAVERSAL, and after psb_build_lbvh the
   context gives the results it gave before, bit for bit.  The oracle is
   checked on the same injection in tests/test_oracle_failure.py.
 * Determinism: the same call twice, and on a second context, gives the same
   bits (FP64 and FP32C forward, every sample source; the adjoint).  No float
   atomics are used anywhere, so this holds by construction.
"""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

if not has_gpu():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from partia_b200 import _lib as L  # noqa: E402
from partia_b200.engine import CatalogC, Context  # noqa: E402


def particles(n, seed):
    rng = np.random.default_rng(seed)
    r = 0.1 / np.sqrt(rng.uniform(0.05, 1.0, n) ** (-2 / 3) - 1)   # a Plummer-like core
    v = rng.standard_normal((3, n))
    v /= np.linalg.norm(v, axis=0)
    x, y, z = r * v
    m = np.full(n, 1.0 / n)
    h = 0.02 * (1 + 5 * r)
    rho = 1.0 / (1 + r * r)
    cols = [rho.copy(), -y, x, 0.1 * z + 0.01 * rng.standard_normal(n)]
    return [x, y, z, m, h, rho], cols


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(a[~np.isnan(a)], b[~np.isnan(b)])


CAT = dict(scalars=[0, 3], shepard=[0, 1], grads=[-1], divs=[1, 2, 3], curls=[1, 2, 3])


def calls(ctx, s, lines, axis):
    """One result per call kind (all through the C ABI)."""
    cat = CatalogC(**CAT)
    out = {}
    out["points"] = ctx.interp_points(*s, cat, strategy=L.PSB_SYMMETRIC)
    ctx.extra_flags = L.PSB_FLAG_SINGLE_KERNEL
    out["points_single"] = ctx.interp_points(*s, cat, strategy=L.PSB_GATHER, hmode=L.PSB_H_NEAREST,
                                             prec=L.PSB_PREC_FP32C)
    ctx.extra_flags = 0
    out["grid"] = ctx.interp_grid(axis, axis, axis, cat, strategy=L.PSB_SCATTER, prec=L.PSB_PREC_FP32C)
    out["lines"] = ctx.interp_lines(*lines, CatalogC(scalars=[0], shepard=[0]), strategy=L.PSB_SCATTER)
    out["density"] = [ctx.density(*s, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_CONSTANT, hs=0.03)]
    out["digest"] = list(ctx.digest(s, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST, fp32c=True))
    return out


def inputs(seed):
    rng = np.random.default_rng(seed)
    s = tuple(rng.uniform(-0.3, 0.3, 3000) for _ in range(3))
    o = tuple(rng.uniform(-0.3, 0.3, 500) for _ in range(3))
    d = np.zeros((3, 500))
    d[2] = 1.0
    o = (o[0], o[1], np.full(500, -2.0))
    return s, (o, tuple(d)), np.linspace(-0.3, 0.3, 24)


def test_bounded_walks_report_a_cycle_and_rebuild_recovers():
    arrs, cols = particles(2000, 31)
    ctx = Context(0)
    ctx.set_particles(*arrs, cols=cols)
    ctx.build(want_perm=False)
    s, lines, axis = inputs(32)
    ref = calls(ctx, s, lines, axis)
    gout = [np.ones(3000) for _ in range(CatalogC(**CAT).L)]
    gref = ctx.adjoint_points(*s, CatalogC(**CAT), gout, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST)

    assert ctx.lib.psb_test_loop_escapes(ctx.h) == L.PSB_OK
    cat = CatalogC(**CAT)
    attempts = [
        lambda: ctx.interp_points(*s, cat, strategy=L.PSB_SYMMETRIC),
        lambda: ctx.interp_points(*s, cat, strategy=L.PSB_SCATTER, prec=L.PSB_PREC_FP32C),
        lambda: ctx.interp_grid(axis, axis, axis, cat, strategy=L.PSB_GATHER, hmode=L.PSB_H_CONSTANT, hs=0.03),
        lambda: ctx.interp_lines(*lines, CatalogC(scalars=[0], shepard=[0]), strategy=L.PSB_SCATTER),
        lambda: ctx.density(*s, strategy=L.PSB_SCATTER),
        lambda: ctx.digest(s, strategy=L.PSB_GATHER, hmode=L.PSB_H_NEAREST),
        lambda: ctx.adjoint_points(*s, cat, gout, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST),
    ]
    for k, f in enumerate(attempts):
        with pytest.raises(L.PsbError) as e:
            f()
        assert e.value.code == L.PSB_ETRAVERSAL, k
        assert "bound" in str(e.value) or "traversal" in str(e.value), str(e.value)
    ctx.extra_flags = L.PSB_FLAG_SINGLE_KERNEL
    with pytest.raises(L.PsbError) as e:
        ctx.interp_points(*s, cat, strategy=L.PSB_GATHER, hmode=L.PSB_H_NEAREST, prec=L.PSB_PREC_FP32C)
    assert e.value.code == L.PSB_ETRAVERSAL
    ctx.extra_flags = 0

    ctx.build(want_perm=False)   # a correct tree again; the context is usable
    again = calls(ctx, s, lines, axis)
    for key in ref:
        for a, b in zip(ref[key], again[key]):
            assert same(a, b), key
    g = ctx.adjoint_points(*s, CatalogC(**CAT), gout, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST)
    for key in ("m", "x", "y", "z"):
        assert np.array_equal(g[key], gref[key])


@pytest.mark.parametrize("prec", [L.PSB_PREC_FP64, L.PSB_PREC_FP32C])
def test_runs_are_bit_identical(prec):
    arrs, cols = particles(200_000, 33)
    ctxs = []
    for _ in range(2):
        c = Context(0)
        c.set_particles(*arrs, cols=cols)
        c.build(want_perm=False)
        ctxs.append(c)
    rng = np.random.default_rng(34)
    s = tuple(rng.uniform(-0.4, 0.4, 300_000) for _ in range(3))
    axis = np.linspace(-0.4, 0.4, 64)
    cat = CatalogC(**CAT)
    res = []
    for c in (ctxs[0], ctxs[0], ctxs[1]):
        r = c.interp_points(*s, cat, strategy=L.PSB_SYMMETRIC, prec=prec)
        r += c.interp_grid(axis, axis, axis, cat, strategy=L.PSB_SYMMETRIC, prec=prec)
        res.append(r)
    for r in res[1:]:
        for a, b in zip(res[0], r):
            assert same(a, b)
    if prec == L.PSB_PREC_FP64:
        gout = [rng.standard_normal(64 ** 3) for _ in range(cat.L)]
        g = [c.adjoint_grid(axis, axis, axis, cat, gout, strategy=L.PSB_SYMMETRIC) for c in (ctxs[0], ctxs[0], ctxs[1])]
        for gi in g[1:]:
            for key in ("m", "x", "y", "z"):
                assert np.array_equal(g[0][key], gi[key]), key
            for a, b in zip(g[0]["cols"], gi["cols"]):
                assert np.array_equal(a, b)
