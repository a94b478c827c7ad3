"""The standalone kernels of single_point_interpolation/kernels/ on the GPU.

 * _number_density_kernel (scalar_interpolation.jl:86-166): psb_density with
   PSB_FLAG_NUMBER_DENSITY, sum_b W, 0 without neighbours;
 * the standalone _gradient_density_kernel (gradient_interpolation.jl:1-170):
   the density gradient of a catalog with PSB_FLAG_DENSITY_GRADIENT_PLAIN,
   sum m gradW - rho(r) sum (m/rho_b) gradW with rho(r) = sum m W, NaN where
   rho(r) = 0; the catalog's other fields are unchanged by the flag;
 * its adjoint against central finite differences of the GPU FP64 forward.
All three strategies, both h modes, FP64 (1e-12 of each field's max) and
FP32C (4e-6, rough random fields).
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

FP64_TOL = 1e-12
FP32C_TOL = 4e-6
STRATS = [(L.PSB_GATHER, O.GATHER), (L.PSB_SCATTER, O.SCATTER), (L.PSB_SYMMETRIC, O.SYMMETRIC)]


def rel_err(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    assert np.array_equal(np.isnan(a), np.isnan(b)), "NaN masks differ"
    fin = ~np.isnan(b)
    if not fin.any():
        return 0.0
    return float(np.max(np.abs(a[fin] - b[fin])) / max(np.max(np.abs(b[fin])), 1e-300))


def particles(n, seed):
    rng = np.random.default_rng(seed)
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    m = rng.uniform(0.5, 1.5, n) / n
    h = 1.2 * (1.0 / n) ** (1 / 3) * rng.uniform(0.5, 2.0, n)
    rho = rng.uniform(0.5, 2.0, n)
    cols = [rho.copy(), np.sin(3 * x) + y, -y + 0.1 * rng.standard_normal(n)]
    return [x, y, z, m, h, rho], cols


def samples(ns, seed):
    rng = np.random.default_rng(seed)
    s = [rng.uniform(-0.1, 1.1, ns) for _ in range(3)]
    s[0][:50] = 5.0   # far outside the particles: empty neighbour sets
    return tuple(s), rng.uniform(0.02, 0.06, ns)


@pytest.mark.parametrize("st,ost", STRATS)
@pytest.mark.parametrize("prec", [L.PSB_PREC_FP64, L.PSB_PREC_FP32C])
def test_number_density(st, ost, prec):
    arrs, cols = particles(30_000, 3)
    ctx = Context(0)
    ctx.set_particles(*arrs, cols=cols)
    ctx.build(want_perm=False)
    orc = O.Oracle(*arrs, cols=cols)
    s, hs = samples(4000, 4)
    got = ctx.density(*s, strategy=st, hmode=L.PSB_H_PER_SAMPLE, hs=hs, prec=prec, number=True)
    ref = orc.density(*s, strategy=ost, hmode=O.H_PER_SAMPLE, hs=hs, number=True)
    assert (ref == 0).any() and (ref > 0).any()
    assert np.array_equal(got == 0, ref == 0)
    assert rel_err(got, ref) <= (FP64_TOL if prec == L.PSB_PREC_FP64 else FP32C_TOL)
    # the flag leaves the mass-weighted density alone
    dm = ctx.density(*s, strategy=st, hmode=L.PSB_H_PER_SAMPLE, hs=hs, prec=prec)
    assert rel_err(dm, orc.density(*s, strategy=ost, hmode=O.H_PER_SAMPLE, hs=hs)) <= (
        FP64_TOL if prec == L.PSB_PREC_FP64 else FP32C_TOL)


@pytest.mark.parametrize("st,ost", STRATS)
@pytest.mark.parametrize("hmode", [L.PSB_H_NEAREST, L.PSB_H_PER_SAMPLE])
@pytest.mark.parametrize("prec", [L.PSB_PREC_FP64, L.PSB_PREC_FP32C])
def test_plain_density_gradient(st, ost, hmode, prec):
    arrs, cols = particles(30_000, 5)
    ctx = Context(0)
    ctx.set_particles(*arrs, cols=cols)
    ctx.build(want_perm=False)
    orc = O.Oracle(*arrs, cols=cols)
    s, hs = samples(4000, 6)
    if hmode == L.PSB_H_NEAREST:
        hs = None
    spec = dict(scalars=[0, 1], shepard=[0, 1], grads=[-1, 1], divs=[], curls=[])
    plain = ctx.interp_points(*s, CatalogC(**spec), strategy=st, hmode=hmode, hs=hs, prec=prec,
                              flags=L.PSB_FLAG_DENSITY_GRADIENT_PLAIN)
    ref = orc.gradient_density(*s, strategy=ost, hmode=hmode, hs=hs)
    tol = FP64_TOL if prec == L.PSB_PREC_FP64 else FP32C_TOL
    for d in range(3):
        assert rel_err(plain[2 + d], ref[d]) <= tol, d
    # every other field as without the flag, bit for bit
    base = ctx.interp_points(*s, CatalogC(**spec), strategy=st, hmode=hmode, hs=hs, prec=prec)
    for k in (0, 1, 5, 6, 7):
        a, b = plain[k], base[k]
        assert np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(a[~np.isnan(a)], b[~np.isnan(b)]), k
    # and the catalog form differs (Shepard-normalised density in the subtraction)
    fin = ~np.isnan(base[2])
    assert not np.allclose(base[2][fin], plain[2][fin])


def test_plain_density_gradient_adjoint_vs_finite_differences():
    arrs, cols = particles(3000, 7)
    x, y, z, m, h, rho = arrs
    ctx = Context(0)
    ctx.set_particles(*arrs, cols=cols)
    ctx.build(want_perm=False)
    rng = np.random.default_rng(8)
    ns = 1500
    s = tuple(rng.uniform(0.05, 0.95, ns) for _ in range(3))
    hs = rng.uniform(0.04, 0.07, ns)
    cat = CatalogC(grads=[-1])
    gout = [rng.standard_normal(ns) for _ in range(3)]
    flag = L.PSB_FLAG_DENSITY_GRADIENT_PLAIN
    g = ctx.adjoint_points(*s, cat, gout, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_PER_SAMPLE, hs=hs, flags=flag)

    def loss(a):
        c2 = Context(0)
        c2.set_particles(*a, cols=cols)
        c2.build(want_perm=False)
        out = c2.interp_points(*s, cat, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_PER_SAMPLE, hs=hs, flags=flag)
        c2.close()
        return sum(float(np.nansum(go * o)) for go, o in zip(gout, out))

    picks = np.argsort(-np.abs(g["m"]))[:6]
    for b in picks:
        for key, k, eps in (("m", 3, 1e-6 * m[b]), ("x", 0, 1e-7), ("y", 1, 1e-7), ("z", 2, 1e-7)):
            up = [a.copy() for a in arrs]
            dn = [a.copy() for a in arrs]
            up[k][b] += eps
            dn[k][b] -= eps
            fd = (loss(up) - loss(dn)) / (2 * eps)
            scale = np.max(np.abs(g[key]))
            assert abs(fd - g[key][b]) <= 1e-5 * scale + 1e-6 * abs(fd), (key, b, fd, g[key][b])
