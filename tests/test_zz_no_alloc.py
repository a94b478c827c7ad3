"""psb_interp_points_noalloc: the allocation-free point interpolation.

Called through the C ABI with device pointers and compared with
psb_interp_points (PSB_FLAG_DEVICE_PTRS) on the same inputs, on two calls in a
row (the second call runs on the scratch the first one left behind).  Also:
device free memory does not move across the calls after the first one on the
device, calls above the sample limit are rejected with PSB_EINVAL, and an
empty call succeeds.  The file sorts last so that the entry point is also
exercised after every other test has used the device; it passes alone in a
fresh process as well.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

if not has_gpu():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

import torch  # noqa: E402

from partia_b200 import _lib as L  # noqa: E402
from partia_b200.engine import CatalogC, Context  # noqa: E402

FP64_TOL = 1e-12
FP32C_TOL = 4e-6


def rel_err(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb), "NaN masks differ"
    fin = ~na
    if not fin.any():
        return 0.0
    scale = max(float(np.max(np.abs(b[fin]))), 1e-300)
    return float(np.max(np.abs(a[fin] - b[fin])) / scale)


def particles(n, seed, dtype):
    rng = np.random.default_rng(seed)
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    m = rng.uniform(0.5, 1.5, n) / n
    h = 1.2 * (1.0 / n) ** (1 / 3) * rng.uniform(0.5, 2.0, n)
    rho = rng.uniform(0.5, 2.0, n)
    cols = [rho.copy(), np.sin(3 * x) + y, -y + 0.1 * rng.standard_normal(n), x + 0.1 * rng.standard_normal(n)]
    return [a.astype(dtype) for a in (x, y, z, m, h, rho)], [c.astype(dtype) for c in cols]


def device_samples(ns, seed, tdt):
    g = torch.Generator(device="cpu").manual_seed(seed)
    s = [(torch.rand(ns, generator=g, dtype=torch.float64) * 1.2 - 0.1).to(tdt).cuda() for _ in range(3)]
    hs = (0.02 + 0.03 * torch.rand(ns, generator=g, dtype=torch.float64)).to(tdt).cuda()
    return s, hs


def noalloc(ctx, s, hmode, hs, strategy, cat, prec, outs):
    ptrs = (C.c_void_p * max(len(outs), 1))(*[o.data_ptr() for o in outs])
    st = L.Stats()
    rc = ctx.lib.psb_interp_points_noalloc(ctx.h, len(s[0]) if s else 0,
                                           *[a.data_ptr() if a is not None else None for a in s],
                                           hmode, hs.data_ptr() if hs is not None else None, strategy,
                                           C.byref(cat.c), prec, ptrs, C.byref(st))
    return rc, st


CAT = dict(scalars=[0, 1], shepard=[1, 0], grads=[1, -1], divs=[1, 2, 3], curls=[1, 2, 3])


@pytest.mark.parametrize("dtype,ns,strategy,hmode,prec", [
    (np.float64, 20_000, L.PSB_SYMMETRIC, L.PSB_H_NEAREST, L.PSB_PREC_FP64),
    (np.float64, 20_000, L.PSB_SYMMETRIC, L.PSB_H_NEAREST, L.PSB_PREC_FP32C),
    (np.float64, 50, L.PSB_GATHER, L.PSB_H_PER_SAMPLE, L.PSB_PREC_FP64),
    (np.float64, L.PSB_NOALLOC_MAX_SAMPLES, L.PSB_SCATTER, L.PSB_H_NEAREST, L.PSB_PREC_FP32C),
    (np.float32, 5_000, L.PSB_SYMMETRIC, L.PSB_H_PER_SAMPLE, L.PSB_PREC_FP32C),
])
def test_noalloc_matches_interp_points(dtype, ns, strategy, hmode, prec):
    arrs, cols = particles(30_000, 11, dtype)
    ctx = Context(0)
    ctx.set_particles(*arrs, cols=cols, dtype=dtype)
    ctx.build(want_perm=False)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    s, hs = device_samples(ns, 5, tdt)
    if hmode != L.PSB_H_PER_SAMPLE:
        hs = None
    cat = CatalogC(**CAT)
    ref = ctx.interp_points(*s, cat, strategy=strategy, hmode=hmode, hs=hs, prec=prec)
    torch.cuda.synchronize()
    ref = [r.cpu().numpy() for r in ref]
    outs = [torch.full((ns,), float("nan"), dtype=tdt, device="cuda") for _ in range(cat.L)]
    tol = FP64_TOL if prec == L.PSB_PREC_FP64 else FP32C_TOL
    if dtype == np.float32:
        tol = 2e-4
    free = []
    for call in range(2):
        for o in outs:
            o.fill_(float("nan"))
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        rc, st = noalloc(ctx, s, hmode, hs, strategy, cat, prec, outs)
        assert rc == L.PSB_OK, ctx.lib.psb_last_error(ctx.h)
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        assert st.pairs > 0
        for k, (o, r) in enumerate(zip(outs, ref)):
            assert rel_err(o.cpu().numpy(), r) <= tol, (call, k)
    # the second call allocates nothing (the first may load the library's
    # device image, which holds the scratch array)
    assert free[2] == free[3]


def test_noalloc_limits_and_empty():
    arrs, cols = particles(2_000, 3, np.float64)
    ctx = Context(0)
    ctx.set_particles(*arrs, cols=cols, dtype=np.float64)
    ctx.build(want_perm=False)
    cat = CatalogC(scalars=[0])
    one = torch.zeros(1, dtype=torch.float64, device="cuda")
    # over the limit: rejected before anything touches the sample arrays
    n_over = L.PSB_NOALLOC_MAX_SAMPLES + 1
    rc = ctx.lib.psb_interp_points_noalloc(ctx.h, n_over, one.data_ptr(), one.data_ptr(), one.data_ptr(),
                                           L.PSB_H_NEAREST, None, L.PSB_SYMMETRIC, C.byref(cat.c),
                                           L.PSB_PREC_FP64, (C.c_void_p * 1)(one.data_ptr()), None)
    assert rc == L.PSB_EINVAL
    assert b"262144" in ctx.lib.psb_last_error(ctx.h)
    # empty call
    rc = ctx.lib.psb_interp_points_noalloc(ctx.h, 0, None, None, None, L.PSB_H_NEAREST, None, L.PSB_SYMMETRIC,
                                           C.byref(cat.c), L.PSB_PREC_FP64, None, None)
    assert rc == L.PSB_OK
    # the context stays usable
    s, _ = device_samples(100, 1, torch.float64)
    out = [torch.empty(100, dtype=torch.float64, device="cuda")]
    rc, _ = noalloc(ctx, s, L.PSB_H_NEAREST, None, L.PSB_SYMMETRIC, cat, L.PSB_PREC_FP64, out)
    assert rc == L.PSB_OK
    ref = ctx.interp_points(*s, cat, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST)
    assert rel_err(out[0].cpu().numpy(), ref[0].cpu().numpy()) <= FP64_TOL
