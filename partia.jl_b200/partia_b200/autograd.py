"""torch.autograd.Function wrappers of the interpolation and its adjoint.

The reference has no derivatives.  The adjoint entry points of the library
(psb_adjoint_points / _grid / _beam) are the vector-Jacobian products a
ChainRulesCore.rrule of PointSamples_interpolation, StructuredGrid_interpolation
and LineSamples_interpolation needs; this module is the same rule for torch:
the forward runs the FP64 interpolation on CUDA tensors, the backward the
adjoint, and gradients flow to the particle masses, positions and quantity
columns.  Smoothing lengths and densities are held fixed (a gradient with
respect to them is refused), as is the sample h (hs, or the nearest
particle's h, which is piecewise constant in the positions).

    out = interpolate_points(x, y, z, m, h, rho, cols, (sx, sy, sz), catalog,
                             strategy=PSB_SYMMETRIC, hmode=PSB_H_PER_SAMPLE, hs=hs)
    loss = (out ** 2).sum(); loss.backward()   # x.grad, m.grad, cols[c].grad

Every tensor lives on one CUDA device; particle tensors are float64 (the
adjoint works on double particle data).  out has shape (L, ns) in catalog
order.  There is no CPU path.
"""
from __future__ import annotations

import itertools
import threading

import torch

from . import _lib as L
from .engine import CatalogC, Context

_engines: dict[int, "_Engine"] = {}
_lock = threading.Lock()
_tokens = itertools.count(1)


class _Engine:
    """One library context per device, re-loaded when another call's
    particles are on it (the backward of a call re-uploads its own)."""

    def __init__(self, device: int):
        self.ctx = Context(device)
        self.token = 0

    def load(self, token, x, y, z, m, h, rho, cols, kernel):
        if self.token == token:
            return self.ctx
        self.ctx.set_particles(x, y, z, m, h, rho, cols=list(cols), kernel=kernel)
        self.ctx.build(want_perm=False)
        self.token = token
        return self.ctx


def _engine(device: int) -> _Engine:
    with _lock:
        e = _engines.get(device)
        if e is None:
            e = _Engine(device)
            _engines[device] = e
        return e


def _check(t, name):
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64):
        raise TypeError(f"{name} must be a float64 CUDA tensor")
    return t.detach().contiguous()


class _Interp(torch.autograd.Function):
    """forward(spec, x, y, z, m, h, rho, *cols) -> (L, ns) outputs."""

    @staticmethod
    def forward(fctx, spec, x, y, z, m, h, rho, *cols):
        dev = x.device.index if x.device.index is not None else torch.cuda.current_device()
        parts = [_check(t, n) for t, n in zip((x, y, z, m, h, rho), ("x", "y", "z", "m", "h", "rho"))]
        cdet = [_check(c, f"cols[{k}]") for k, c in enumerate(cols)]
        token = next(_tokens)
        with torch.cuda.device(dev):
            eng = _engine(dev)
            ctx = eng.load(token, *parts, cdet, spec["kernel"])
            torch.cuda.current_stream().synchronize()
            outs = spec["run"](ctx)
        fctx.spec = spec
        fctx.token = token
        fctx.dev = dev
        fctx.ncol = len(cols)
        fctx.save_for_backward(*parts, *cdet)
        return torch.stack(outs)

    @staticmethod
    def backward(fctx, gout):
        spec = fctx.spec
        saved = fctx.saved_tensors
        parts, cols = saved[:6], list(saved[6:])
        if fctx.needs_input_grad[5] or fctx.needs_input_grad[6]:
            raise RuntimeError("gradients with respect to h and rho are not provided (they are held fixed)")
        with torch.cuda.device(fctx.dev):
            ctx = _engine(fctx.dev).load(fctx.token, *parts, cols, spec["kernel"])
            go = [torch.nan_to_num(g.detach(), nan=0.0).contiguous() for g in gout]
            torch.cuda.current_stream().synchronize()
            g = spec["adjoint"](ctx, go)
        grads = [None, g["x"], g["y"], g["z"], g["m"], None, None]
        grads += [g["cols"][k] if fctx.needs_input_grad[7 + k] else None for k in range(fctx.ncol)]
        return tuple(grads)


def _as_cat(catalog) -> CatalogC:
    if isinstance(catalog, CatalogC):
        return catalog
    return catalog.concise()   # a partia_b200.InterpolationCatalog


def interpolate_points(x, y, z, m, h, rho, cols, samples, catalog, strategy=L.PSB_SYMMETRIC,
                       hmode=L.PSB_H_PER_SAMPLE, hs=None, kernel=L.PSB_KERNEL_M4):
    """PointSamples_interpolation in FP64 with gradients for m, x, y, z and cols."""
    cat = _as_cat(catalog)
    s = [t.detach().double().contiguous() for t in samples]
    hsd = None if hs is None else torch.as_tensor(hs, dtype=torch.float64, device=s[0].device).reshape(-1)

    def run(ctx):
        return ctx.interp_points(*s, cat, strategy=strategy, hmode=hmode, hs=hsd, prec=L.PSB_PREC_FP64)

    def adjoint(ctx, go):
        return ctx.adjoint_points(*s, cat, go, strategy=strategy, hmode=hmode, hs=hsd)

    spec = dict(kernel=kernel, run=run, adjoint=adjoint)
    return _Interp.apply(spec, x, y, z, m, h, rho, *cols)


def interpolate_grid(x, y, z, m, h, rho, cols, axes, catalog, strategy=L.PSB_SYMMETRIC,
                     hmode=L.PSB_H_PER_SAMPLE, hs=None, kernel=L.PSB_KERNEL_M4):
    """StructuredGrid_interpolation (Cartesian axes, column-major samples)."""
    cat = _as_cat(catalog)
    ax = [torch.as_tensor(a, dtype=torch.float64).cpu().numpy() for a in axes]
    ns = len(ax[0]) * len(ax[1]) * len(ax[2])
    dev = x.device
    hsd = None if hs is None else torch.as_tensor(hs, dtype=torch.float64, device=dev).reshape(-1)

    def run(ctx):
        out = [torch.empty(ns, dtype=torch.float64, device=dev) for _ in range(cat.L)]
        return ctx.interp_grid(*ax, cat, strategy=strategy, hmode=hmode, hs=hsd, prec=L.PSB_PREC_FP64, out=out)

    def adjoint(ctx, go):
        return ctx.adjoint_grid(*ax, cat, go, strategy=strategy, hmode=hmode, hs=hsd, device=True)

    spec = dict(kernel=kernel, run=run, adjoint=adjoint)
    return _Interp.apply(spec, x, y, z, m, h, rho, *cols)


def interpolate_beam(x, y, z, m, h, rho, cols, frame, params, nx, ny, catalog, kernel=L.PSB_KERNEL_M4):
    """LineSamples_interpolation over a parallel beam (scatter), e.g. column density."""
    cat = _as_cat(catalog)
    fr = torch.as_tensor(frame, dtype=torch.float64).cpu().numpy()
    pa = torch.as_tensor(params, dtype=torch.float64).cpu().numpy()
    dev = x.device

    def run(ctx):
        out = [torch.empty(nx * ny, dtype=torch.float64, device=dev) for _ in range(cat.L)]
        return ctx.interp_beam(fr, pa, nx, ny, cat, strategy=L.PSB_SCATTER, prec=L.PSB_PREC_FP64, out=out)

    def adjoint(ctx, go):
        return ctx.adjoint_beam(fr, pa, nx, ny, cat, go, strategy=L.PSB_SCATTER, device=True)

    spec = dict(kernel=kernel, run=run, adjoint=adjoint)
    return _Interp.apply(spec, x, y, z, m, h, rho, *cols)
