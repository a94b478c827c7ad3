"""Thin object wrapper of one library context (one particle set + its LBVH).

Arrays are numpy arrays (host; the library copies them) or objects exposing
``data_ptr()`` on the context's device (e.g. torch CUDA tensors), which are
passed as device pointers with PSB_FLAG_DEVICE_PTRS.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


def _is_dev(a) -> bool:
    return hasattr(a, "data_ptr")


def _ptr(a):
    if a is None:
        return None
    if _is_dev(a):
        return a.data_ptr()
    return a.ctypes.data


def _ptr_array(arrs):
    t = (C.c_void_p * max(len(arrs), 1))()
    for k, a in enumerate(arrs):
        t[k] = _ptr(a)
    return t


class CatalogC:
    """InterpolationCatalogConcise with 0-based slots (grad slot -1: density)."""

    def __init__(self, scalars=(), shepard=None, grads=(), divs=(), curls=()):
        self.scalars = np.ascontiguousarray(scalars, dtype=np.int32)
        if shepard is None:
            shepard = [1] * len(self.scalars)
        self.shepard = np.ascontiguousarray(shepard, dtype=np.uint8)
        self.grads = np.ascontiguousarray(grads, dtype=np.int32)
        self.divs = np.ascontiguousarray(divs, dtype=np.int32).reshape(-1)
        self.curls = np.ascontiguousarray(curls, dtype=np.int32).reshape(-1)
        self.c = L.Catalog(len(self.scalars), self.scalars.ctypes.data, self.shepard.ctypes.data,
                           len(self.grads), self.grads.ctypes.data, len(self.divs) // 3, self.divs.ctypes.data,
                           len(self.curls) // 3, self.curls.ctypes.data)

    @property
    def L(self) -> int:
        return len(self.scalars) + 3 * len(self.grads) + len(self.divs) // 3 + len(self.curls)


class Context:
    """One psb_ctx on one GPU."""

    def __init__(self, device: int = 0):
        self.lib = L.load()
        h = C.c_void_p()
        rc = self.lib.psb_create(C.byref(h), int(device))
        if rc != 0:
            raise L.PsbError(rc, "psb_create failed (is a CUDA device visible?)")
        self.h = h
        self.device = int(device)
        # OR-ed into the flags of the interpolation calls (e.g. PSB_FLAG_SINGLE_KERNEL)
        self.extra_flags = 0
        self.dtype = np.dtype(np.float64)
        self.n = 0
        self.ncol = 0
        self.last_stats = L.Stats()
        self.builds = 0  # psb_build_lbvh calls made through this object
        self.kernel = L.PSB_KERNEL_M4
        self.generation = 0  # LBVH builds made through the Partia-API layer on this context

    def close(self):
        if getattr(self, "h", None):
            self.lib.psb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        L.check(self.h, rc)

    # ---- particles / build ----
    def set_particles(self, x, y, z, m, h, rho, cols=(), dtype=None, kernel=L.PSB_KERNEL_M4):
        dev = _is_dev(x)
        if dtype is None:
            dtype = (np.float64 if str(x.dtype).endswith("float64") else np.float32) if dev else np.asarray(x).dtype
        self.dtype = np.dtype(dtype)
        if not dev:
            cv = lambda a: np.ascontiguousarray(np.asarray(a, dtype=self.dtype))
            x, y, z, m, h, rho = (cv(a) for a in (x, y, z, m, h, rho))
            cols = [cv(c) for c in cols]
        self._keep = (x, y, z, m, h, rho, list(cols))
        n = len(x)
        dt = L.PSB_F64 if self.dtype == np.float64 else L.PSB_F32
        colp = _ptr_array(list(cols))
        self._chk(self.lib.psb_set_particles(self.h, n, dt, _ptr(x), _ptr(y), _ptr(z), _ptr(m), _ptr(h), _ptr(rho),
                                             len(cols), colp, int(kernel),
                                             L.PSB_FLAG_DEVICE_PTRS if dev else 0))
        self._keep = None
        self.n = n
        self.ncol = len(cols)
        self.kernel = int(kernel)

    def set_values(self, m, rho, cols=()):
        """New m, rho and columns (in the LBVH's leaf order) for the built tree."""
        dev = _is_dev(m)
        if not dev:
            cv = lambda a: np.ascontiguousarray(np.asarray(a, dtype=self.dtype))
            m, rho = cv(m), cv(rho)
            cols = [cv(c) for c in cols]
        cols = list(cols)
        for a in (m, rho, *cols):
            if len(a) != self.n:
                raise ValueError(f"value arrays must hold {self.n} entries (got {len(a)})")
        self._chk(self.lib.psb_set_values(self.h, _ptr(m), _ptr(rho), len(cols), _ptr_array(cols),
                                          L.PSB_FLAG_DEVICE_PTRS if dev else 0))
        self.ncol = len(cols)

    def build(self, want_perm=True, want_codes=False):
        perm = np.zeros(self.n, dtype=np.int64) if want_perm else None
        codes = np.zeros(self.n, dtype=np.uint64) if want_codes else None
        self._chk(self.lib.psb_build_lbvh(self.h, _ptr(perm), _ptr(codes)))
        self.builds += 1
        return perm, codes

    def tree(self):
        n = self.n
        tot, nint = 2 * n - 1, max(n - 1, 0)
        root = np.zeros(1, dtype=np.int32)
        l, r, e, p = (np.zeros(tot, dtype=np.int32) for _ in range(4))
        nmin, nmax, ns = np.zeros(3 * nint), np.zeros(3 * nint), np.zeros(nint)
        self._chk(self.lib.psb_get_tree(self.h, root.ctypes.data, l.ctypes.data, r.ctypes.data, e.ctypes.data,
                                        p.ctypes.data, nmin.ctypes.data, nmax.ctypes.data, ns.ctypes.data))
        return dict(root=int(root[0]), left=l, right=r, escape=e, parent=p,
                    node_min=nmin.reshape(3, nint), node_max=nmax.reshape(3, nint), node_scale=ns)

    # ---- helpers ----
    def _arr(self, a):
        if _is_dev(a):
            return a
        return np.ascontiguousarray(np.asarray(a, dtype=self.dtype))

    def _hs(self, hmode, hs, dev):
        """hs where the call's pointers live: on this context's GPU when the
        call passes device pointers, in host memory otherwise."""
        if hs is None:
            return None
        if dev:
            import torch
            tdt = torch.float64 if self.dtype == np.float64 else torch.float32
            return torch.as_tensor(hs, dtype=tdt).reshape(-1).to(f"cuda:{self.device}").contiguous()
        if _is_dev(hs):
            hs = hs.detach().cpu().numpy()
        return np.ascontiguousarray(np.atleast_1d(np.asarray(hs, dtype=self.dtype)))

    def _outs(self, ns, L_, like_dev, out=None):
        if out is not None:
            return out
        if like_dev:
            import torch
            tdt = torch.float64 if self.dtype == np.float64 else torch.float32
            return [torch.empty(ns, dtype=tdt, device="cuda") for _ in range(L_)]
        return [np.empty(ns, dtype=self.dtype) for _ in range(L_)]

    # ---- interpolation ----
    def interp_points(self, sx, sy, sz, cat: CatalogC, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST, hs=None,
                      prec=L.PSB_PREC_FP64, out=None, flags=0):
        sx, sy, sz = self._arr(sx), self._arr(sy), self._arr(sz)
        dev = _is_dev(sx)
        ns = len(sx)
        hsa = self._hs(hmode, hs, dev)
        outs = self._outs(ns, cat.L, dev, out)
        self._chk(self.lib.psb_interp_points(self.h, ns, _ptr(sx), _ptr(sy), _ptr(sz), hmode, _ptr(hsa), strategy,
                                             C.byref(cat.c), prec, _ptr_array(outs),
                                             (L.PSB_FLAG_DEVICE_PTRS if dev else 0) | self.extra_flags | flags,
                                             C.byref(self.last_stats)))
        return outs

    # ---- the reference's GPU design (baseline) ----
    def baseline_cudaext_points(self, parts, tree, sx, sy, sz, cat: CatalogC, strategy=L.PSB_SYMMETRIC, kernel=None):
        """psb_baseline_cudaext_points: parts = dict of host arrays x y z m h rho
        and cols (leaf order), tree = Context.tree() of the same particles;
        samples and outputs are host arrays (copied every call)."""
        f64 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64))
        arrs = [f64(parts[k]) for k in ("x", "y", "z", "m", "h", "rho")]
        cols = [f64(c) for c in parts.get("cols", ())]
        s = [f64(a) for a in (sx, sy, sz)]
        ns = len(s[0])
        outs = [np.empty(ns, dtype=np.float64) for _ in range(cat.L)]
        t = {k: np.ascontiguousarray(tree[k]) for k in ("left", "escape")}
        nmin = np.ascontiguousarray(tree["node_min"], dtype=np.float64)
        nmax = np.ascontiguousarray(tree["node_max"], dtype=np.float64)
        nsc = np.ascontiguousarray(tree["node_scale"], dtype=np.float64)
        kern = self.kernel if kernel is None else int(kernel)
        self._chk(self.lib.psb_baseline_cudaext_points(
            self.h, len(arrs[0]), *[_ptr(a) for a in arrs], len(cols), _ptr_array(cols), kern, int(tree["root"]),
            _ptr(t["left"]), _ptr(t["escape"]), _ptr(nmin), _ptr(nmax), _ptr(nsc), ns, *[_ptr(a) for a in s],
            strategy, C.byref(cat.c), _ptr_array(outs), C.byref(self.last_stats)))
        return outs

    # ---- adjoint ----
    def _grad_outs(self, like_dev):
        n = self.n
        if like_dev:
            import torch
            mk = lambda: torch.zeros(n, dtype=torch.float64, device="cuda")
        else:
            mk = lambda: np.zeros(n, dtype=np.float64)
        g = dict(m=mk(), x=mk(), y=mk(), z=mk(), cols=[mk() for _ in range(self.ncol)])
        return g

    def _gout(self, gout, dev):
        if dev:
            return list(gout)
        return [np.ascontiguousarray(np.asarray(g, dtype=np.float64)) for g in gout]

    def adjoint_points(self, sx, sy, sz, cat: CatalogC, gout, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST,
                       hs=None, flags=0):
        """dL/dm, dL/dA_c, dL/dx.. for L = sum_k sum_s gout[k][s] out_k(s), in the particles' given order."""
        sx, sy, sz = self._arr(sx), self._arr(sy), self._arr(sz)
        dev = _is_dev(sx)
        hsa = self._hs(hmode, hs, dev)
        go = self._gout(gout, dev)
        g = self._grad_outs(dev)
        self._chk(self.lib.psb_adjoint_points(self.h, len(sx), _ptr(sx), _ptr(sy), _ptr(sz), hmode, _ptr(hsa),
                                              strategy, C.byref(cat.c), _ptr_array(go), _ptr(g["m"]),
                                              _ptr_array(g["cols"]), _ptr(g["x"]), _ptr(g["y"]), _ptr(g["z"]),
                                              (L.PSB_FLAG_DEVICE_PTRS if dev else 0) | flags,
                                              C.byref(self.last_stats)))
        return g

    def adjoint_grid(self, ax, ay, az, cat: CatalogC, gout, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST,
                     hs=None, device=False):
        ax, ay, az = (np.ascontiguousarray(np.asarray(a, dtype=np.float64)) for a in (ax, ay, az))
        hsa = self._hs(hmode, hs, device)
        go = self._gout(gout, device)
        g = self._grad_outs(device)
        self._chk(self.lib.psb_adjoint_grid(self.h, ax.ctypes.data, len(ax), ay.ctypes.data, len(ay),
                                            az.ctypes.data, len(az), hmode, _ptr(hsa), strategy, C.byref(cat.c),
                                            _ptr_array(go), _ptr(g["m"]), _ptr_array(g["cols"]), _ptr(g["x"]),
                                            _ptr(g["y"]), _ptr(g["z"]), L.PSB_FLAG_DEVICE_PTRS if device else 0,
                                            C.byref(self.last_stats)))
        return g

    def adjoint_beam(self, frame, params, nx, ny, cat: CatalogC, gout, strategy=L.PSB_SCATTER,
                     hmode=L.PSB_H_PER_SAMPLE, hs=None, device=False):
        fr = np.ascontiguousarray(np.asarray(frame, dtype=np.float64).reshape(12))
        pa = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(4))
        hsa = self._hs(hmode, hs, device)
        go = self._gout(gout, device)
        g = self._grad_outs(device)
        self._chk(self.lib.psb_adjoint_beam(self.h, fr.ctypes.data, pa.ctypes.data, nx, ny, hmode, _ptr(hsa),
                                            strategy, C.byref(cat.c), _ptr_array(go), _ptr(g["m"]),
                                            _ptr_array(g["cols"]), _ptr(g["x"]), _ptr(g["y"]), _ptr(g["z"]),
                                            L.PSB_FLAG_DEVICE_PTRS if device else 0, C.byref(self.last_stats)))
        return g

    def interp_grid(self, ax, ay, az, cat: CatalogC, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST, hs=None,
                    prec=L.PSB_PREC_FP64, out=None, device_out=False):
        ax, ay, az = (np.ascontiguousarray(np.asarray(a, dtype=self.dtype)) for a in (ax, ay, az))
        ns = len(ax) * len(ay) * len(az)
        dev = device_out or (out is not None and _is_dev(out[0]))
        hsa = self._hs(hmode, hs, dev)
        outs = self._outs(ns, cat.L, dev, out)
        self._chk(self.lib.psb_interp_grid(self.h, ax.ctypes.data, len(ax), ay.ctypes.data, len(ay),
                                           az.ctypes.data, len(az), hmode, _ptr(hsa), strategy, C.byref(cat.c), prec,
                                           _ptr_array(outs), (L.PSB_FLAG_DEVICE_PTRS if dev else 0) | self.extra_flags,
                                           C.byref(self.last_stats)))
        return outs

    def interp_box(self, frame, params, nx, ny, nz, cat: CatalogC, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST,
                   hs=None, prec=L.PSB_PREC_FP64, out=None, device_out=False):
        fr = np.ascontiguousarray(np.asarray(frame, dtype=self.dtype).reshape(12))
        pa = np.ascontiguousarray(np.asarray(params, dtype=self.dtype).reshape(6))
        ns = nx * ny * nz
        dev = device_out or (out is not None and _is_dev(out[0]))
        hsa = self._hs(hmode, hs, dev)
        outs = self._outs(ns, cat.L, dev, out)
        self._chk(self.lib.psb_interp_box(self.h, fr.ctypes.data, pa.ctypes.data, nx, ny, nz, hmode, _ptr(hsa),
                                          strategy, C.byref(cat.c), prec, _ptr_array(outs),
                                          (L.PSB_FLAG_DEVICE_PTRS if dev else 0) | self.extra_flags, C.byref(self.last_stats)))
        return outs

    def interp_lines(self, o, d, cat: CatalogC, strategy=L.PSB_SCATTER, hmode=L.PSB_H_PER_SAMPLE, hs=None,
                     prec=L.PSB_PREC_FP64, out=None):
        arrs = [self._arr(a) for a in (*o, *d)]
        dev = _is_dev(arrs[0])
        nl = len(arrs[0])
        hsa = self._hs(hmode, hs, dev)
        outs = self._outs(nl, cat.L, dev, out)
        self._chk(self.lib.psb_interp_lines(self.h, nl, *[_ptr(a) for a in arrs], hmode, _ptr(hsa), strategy,
                                            C.byref(cat.c), prec, _ptr_array(outs),
                                            (L.PSB_FLAG_DEVICE_PTRS if dev else 0) | self.extra_flags, C.byref(self.last_stats)))
        return outs

    def interp_beam(self, frame, params, nx, ny, cat: CatalogC, strategy=L.PSB_SCATTER, hmode=L.PSB_H_PER_SAMPLE,
                    hs=None, prec=L.PSB_PREC_FP64, out=None, device_out=False):
        fr = np.ascontiguousarray(np.asarray(frame, dtype=self.dtype).reshape(12))
        pa = np.ascontiguousarray(np.asarray(params, dtype=self.dtype).reshape(4))
        dev = device_out or (out is not None and _is_dev(out[0]))
        hsa = self._hs(hmode, hs, dev)
        outs = self._outs(nx * ny, cat.L, dev, out)
        self._chk(self.lib.psb_interp_beam(self.h, fr.ctypes.data, pa.ctypes.data, nx, ny, hmode, _ptr(hsa), strategy,
                                           C.byref(cat.c), prec, _ptr_array(outs),
                                           (L.PSB_FLAG_DEVICE_PTRS if dev else 0) | self.extra_flags, C.byref(self.last_stats)))
        return outs

    def density(self, sx, sy, sz, strategy=L.PSB_GATHER, hmode=L.PSB_H_PER_SAMPLE, hs=None, prec=L.PSB_PREC_FP64,
                out=None, number=False):
        """sum m W (_density_kernel), or sum W (_number_density_kernel) with number=True."""
        sx, sy, sz = self._arr(sx), self._arr(sy), self._arr(sz)
        dev = _is_dev(sx)
        hsa = self._hs(hmode, hs, dev)
        o = out if out is not None else self._outs(len(sx), 1, dev)[0]
        flags = (L.PSB_FLAG_DEVICE_PTRS if dev else 0) | self.extra_flags
        if number:
            flags |= L.PSB_FLAG_NUMBER_DENSITY
        self._chk(self.lib.psb_density(self.h, len(sx), _ptr(sx), _ptr(sy), _ptr(sz), hmode, _ptr(hsa), strategy, prec,
                                       _ptr(o), flags, C.byref(self.last_stats)))
        return o

    def digest(self, a, d=None, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST, hs=None, fp32c=False):
        kind = 0 if d is None else 1
        arrs = [self._arr(v) for v in a]
        darrs = [self._arr(v) for v in d] if d is not None else [None, None, None]
        ns = len(arrs[0])
        hsa = self._hs(hmode, hs, False)
        cnt = np.zeros(ns, dtype=np.int64)
        hsh = np.zeros(ns, dtype=np.uint64)
        ha = np.zeros(ns, dtype=self.dtype)
        flags = L.PSB_FLAG_FP32C_DECISIONS if fp32c else 0
        self._chk(self.lib.psb_neighbor_digest(self.h, kind, ns, *[_ptr(v) for v in arrs], *[_ptr(v) for v in darrs],
                                               hmode, _ptr(hsa), strategy, cnt.ctypes.data, hsh.ctypes.data,
                                               ha.ctypes.data, flags))
        return cnt, hsh, ha
