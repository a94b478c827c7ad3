"""The CUDA-extension design kept as a baseline (psb_baseline_cudaext_points):
one thread per sample, per-thread DFS, tree and input copied from the host
every call (ext/CUDAExt/KernelInterpolation/grid_interpolation/drivers/
PointSamples_driver.jl:12-27, kernels/PointSamples_kernel.jl:1-68).  It must
give the oracle's fields (FP64, 1e-12 of each field's max, identical NaN
masks) and the library's accepted-pair count, for every strategy, with M4
and another kernel family."""
import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

if not has_gpu():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

import oracle as O  # noqa: E402
from partia_b200 import _lib as L  # noqa: E402
from partia_b200.engine import CatalogC, Context  # noqa: E402

TOL = 1e-12
SPEC = dict(scalars=[0, 1], shepard=[0, 1], grads=[-1, 1], divs=[1, 2, 3], curls=[1, 2, 3])


def rel_err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert np.array_equal(np.isnan(a), np.isnan(b)), "NaN masks differ"
    fin = ~np.isnan(b)
    return float(np.max(np.abs(a[fin] - b[fin])) / np.max(np.abs(b[fin]))) if fin.any() else 0.0


@pytest.mark.parametrize("kernel", [L.PSB_KERNEL_M4, L.PSB_KERNEL_M5])
@pytest.mark.parametrize("strategy,ost", [(L.PSB_GATHER, O.GATHER), (L.PSB_SCATTER, O.SCATTER),
                                          (L.PSB_SYMMETRIC, O.SYMMETRIC)])
def test_cudaext_design_matches_oracle_and_library(kernel, strategy, ost):
    rng = np.random.default_rng(44)
    n = 20_000
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    m = rng.uniform(0.5, 1.5, n) / n
    h = 1.2 * (1.0 / n) ** (1 / 3) * rng.uniform(0.5, 2.0, n)
    rho = rng.uniform(0.5, 2.0, n)
    cols = [rho.copy(), np.sin(3 * x) + y, -y + 0.1 * rng.standard_normal(n), x + 0.1 * rng.standard_normal(n)]
    ctx = Context(0)
    ctx.set_particles(x, y, z, m, h, rho, cols, kernel=kernel)
    perm, _ = ctx.build()
    tree = ctx.tree()
    parts = dict(x=x[perm], y=y[perm], z=z[perm], m=m[perm], h=h[perm], rho=rho[perm], cols=[c[perm] for c in cols])
    s = [rng.uniform(-0.05, 1.05, 7000) for _ in range(3)]
    s[0][:20] = 3.0  # no neighbours: NaN
    cat = CatalogC(**SPEC)
    got = ctx.baseline_cudaext_points(parts, tree, *s, cat, strategy=strategy)
    base_pairs = ctx.last_stats.pairs
    assert ctx.last_stats.launches == 1 and ctx.last_stats.h2d_ms > 0
    lib = ctx.interp_points(*s, cat, strategy=strategy, hmode=L.PSB_H_NEAREST, prec=L.PSB_PREC_FP64)
    assert ctx.last_stats.pairs == base_pairs
    orc = O.Oracle(x, y, z, m, h, rho, cols, kernel=kernel)
    ref = orc.interp_points(*s, O.Catalog(**SPEC), strategy=ost, hmode=O.H_NEAREST)
    for k in range(cat.L):
        assert rel_err(got[k], ref[k]) <= TOL, k
        assert rel_err(got[k], lib[k]) <= TOL, k
