"""torch.autograd.Function wrappers (partia_b200.autograd) over the adjoint
entry points: torch.autograd.gradcheck in FP64 on small cases, for the point,
structured-grid and parallel-beam forwards, with respect to masses, positions
and quantity columns (central differences of the library's own FP64 forward
against the Jacobian the backward returns)."""
import math

import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

if not has_gpu():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

import torch  # noqa: E402

from partia_b200 import _lib as L  # noqa: E402
from partia_b200 import autograd as AG  # noqa: E402
from partia_b200 import workloads as W  # noqa: E402
from partia_b200.engine import CatalogC  # noqa: E402


def particles(n, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    x, y, z = (torch.rand(n, generator=g, dtype=torch.float64) for _ in range(3))
    m = (0.5 + torch.rand(n, generator=g, dtype=torch.float64)) / n
    h = 1.6 * (1.0 / n) ** (1 / 3) * (0.7 + 0.6 * torch.rand(n, generator=g, dtype=torch.float64))
    rho = 0.8 + 0.4 * torch.rand(n, generator=g, dtype=torch.float64)
    A = torch.sin(3 * x) + y + 0.1 * torch.randn(n, generator=g, dtype=torch.float64)
    B = -y + 0.2 * z
    C = x * z
    cuda = lambda t: t.cuda()
    return [cuda(t) for t in (x, y, z, m, h, rho, A, B, C)]


def test_gradcheck_points():
    x, y, z, m, h, rho, A, B, C = particles(150, 1)
    g = torch.Generator(device="cpu").manual_seed(2)
    s = [(0.15 + 0.7 * torch.rand(40, generator=g, dtype=torch.float64)).cuda() for _ in range(3)]
    hs = (0.25 + 0.1 * torch.rand(40, generator=g, dtype=torch.float64)).cuda()
    cat = CatalogC(scalars=[0, 1], shepard=[0, 1], grads=[-1, 1], divs=[1, 2, 3], curls=[1, 2, 3])

    def f(m_, x_, y_, z_, A_, B_):
        return AG.interpolate_points(x_, y_, z_, m_, h, rho, [rho, A_, B_, C], s, cat,
                                     strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_PER_SAMPLE, hs=hs)

    inputs = [t.clone().requires_grad_(True) for t in (m, x, y, z, A, B)]
    assert torch.autograd.gradcheck(f, inputs, eps=1e-6, atol=1e-6, rtol=1e-4)


def test_gradcheck_grid_and_backward_values():
    x, y, z, m, h, rho, A, B, C = particles(120, 3)
    ax = np.linspace(0.2, 0.8, 4)
    cat = CatalogC(scalars=[1], shepard=[1], grads=[1])

    def f(m_, x_, A_):
        return AG.interpolate_grid(x_, y, z, m_, h, rho, [rho, A_], (ax, ax, ax), cat,
                                   strategy=L.PSB_GATHER, hmode=L.PSB_H_CONSTANT, hs=0.3)

    inputs = [t.clone().requires_grad_(True) for t in (m, x, A)]
    assert torch.autograd.gradcheck(f, inputs, eps=1e-6, atol=1e-6, rtol=1e-4)
    # a scalar loss: the gradient is the adjoint's
    mm, xx, AA = (t.clone().requires_grad_(True) for t in (m, x, A))
    out = f(mm, xx, AA)
    (out[0] ** 2).sum().backward()
    assert mm.grad is not None and xx.grad is not None and AA.grad is not None
    assert torch.isfinite(xx.grad).all()


def test_gradcheck_beam_column_density():
    x, y, z, m, h, rho, A, B, C = particles(150, 5)
    fr = W.c3_frame().as_array()
    prm = np.array([0.1, 0.9, 0.1, 0.9])
    cat = CatalogC(scalars=[0, 1], shepard=[0, 1])

    def f(m_, x_, z_, A_):
        return AG.interpolate_beam(x_, y, z_, m_, h, rho, [rho, A_], fr, prm, 6, 5, cat)

    # masses and the column enter linearly: the full gradcheck
    def f_lin(m_, A_):
        return f(m_, x, z, A_)

    assert torch.autograd.gradcheck(f_lin, [m.clone().requires_grad_(True), A.clone().requires_grad_(True)],
                                    eps=1e-6, atol=1e-8, rtol=1e-6)
    # positions: the line kernel is a piecewise-linear table in q, so a
    # central difference that straddles a table knot averages two slopes.
    # The backward's slope must match the forward or the backward one-sided
    # difference (the slope on one side of the knot), or lie between them.
    eps = 1e-7
    for which in ("x", "z"):
        pos = (x if which == "x" else z).clone().requires_grad_(True)
        out = (f(m, pos, z, A) if which == "x" else f(m, x, pos, A)).reshape(-1)
        ja = torch.stack([torch.autograd.grad(out[i], pos, retain_graph=True)[0] for i in range(out.numel())])
        base = out.detach()
        fwd = torch.empty_like(ja)
        bwd = torch.empty_like(ja)
        for j in range(pos.numel()):
            for sgn, dst in ((1.0, fwd), (-1.0, bwd)):
                q = pos.detach().clone()
                q[j] += sgn * eps
                o = (f(m, q, z, A) if which == "x" else f(m, x, q, A)).reshape(-1)
                dst[:, j] = sgn * (o - base) / eps
        tol = 2e-6 + 1e-3 * torch.maximum(fwd.abs(), bwd.abs())
        lo, hi = torch.minimum(fwd, bwd) - tol, torch.maximum(fwd, bwd) + tol
        ok = (ja >= lo) & (ja <= hi)
        assert bool(ok.all()), (which, int((~ok).sum()), float((ja - (fwd + bwd) / 2).abs().max()))


def test_h_and_rho_are_held_fixed():
    x, y, z, m, h, rho, A, B, C = particles(100, 7)
    hh = h.clone().requires_grad_(True)
    s = [(0.3 + 0.4 * torch.rand(10, dtype=torch.float64)).cuda() for _ in range(3)]
    out = AG.interpolate_points(x, y, z, m, hh, rho, [A], s, CatalogC(scalars=[0], shepard=[1]),
                                hmode=L.PSB_H_CONSTANT, hs=0.3)
    with pytest.raises(RuntimeError):
        out.sum().backward()
    assert math.isfinite(float(out.nansum()))
