"""ctypes wrapper of the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA library and the timed CPU
baseline.  Product code never imports this module; only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline legs do.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle_partia.so")
_lib = None

GATHER, SCATTER, SYMMETRIC = 0, 1, 2
# kernel families (kernel_function/kernels/*.jl), numbered as psb_kernel
M4, M5, M6, C2, C4, C6 = 0, 1, 2, 3, 4, 5
H_NEAREST, H_PER_SAMPLE, H_CONSTANT = 0, 1, 2

_vp = C.c_void_p
_i64 = C.c_int64


def build() -> str:
    """Compile the oracle with its Makefile (a few seconds)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "oracle.cpp")
        ):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_threads.restype = C.c_int
        for name in ("orc_W", "orc_line_kernel"):
            getattr(L, name).argtypes = [C.c_double, C.c_double]
            getattr(L, name).restype = C.c_double
        for name in ("orc_Wf", "orc_line_kernelf"):
            getattr(L, name).argtypes = [C.c_float, C.c_float]
            getattr(L, name).restype = C.c_float
        for name in ("orc_f", "orc_df"):
            getattr(L, name).argtypes = [C.c_double]
            getattr(L, name).restype = C.c_double
        for name in ("orc_support", "orc_norm3"):
            getattr(L, name).argtypes = []
            getattr(L, name).restype = C.c_double
        L.orc_set_kernel.argtypes = [C.c_int]
        L.orc_set_kernel.restype = C.c_int
        L.orc_gradW.argtypes = [C.c_double] * 4 + [_vp]
        L.orc_gradW.restype = None
        L.orc_line_table.argtypes = [_vp, _vp]
        L.orc_line_table.restype = None
        L.orc_create.argtypes = [_i64, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int, _vp]
        L.orc_create.restype = _vp
        L.orc_destroy.argtypes = [_vp]
        L.orc_destroy.restype = None
        L.orc_build.argtypes = [_vp, _vp, _vp]
        L.orc_build.restype = C.c_int
        L.orc_test_loop_escapes.argtypes = [_vp]
        L.orc_test_loop_escapes.restype = C.c_int
        L.orc_get_tree.argtypes = [_vp] * 9
        L.orc_get_tree.restype = C.c_int
        L.orc_interp_points.argtypes = [_vp, _i64, _vp, _vp, _vp, C.c_int, _vp, C.c_int,
                                        C.c_int, _vp, _vp, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, _vp]
        L.orc_interp_points.restype = C.c_int
        L.orc_interp_lines.argtypes = [_vp, _i64, _vp, C.c_int, _vp, C.c_int, C.c_int, _vp, _vp, _vp]
        L.orc_interp_lines.restype = C.c_int
        L.orc_density.argtypes = [_vp, _i64, _vp, _vp, _vp, C.c_int, _vp, C.c_int, _vp, C.c_int]
        L.orc_density.restype = C.c_int
        L.orc_neighbor_digest.argtypes = [_vp, C.c_int, _i64, _vp, C.c_int, _vp, C.c_int, _vp, _vp, _vp]
        L.orc_neighbor_digest.restype = C.c_int
        L.orc_brute_digest.argtypes = [_vp, C.c_int, _i64, _vp, _vp, C.c_int, _vp, _vp]
        L.orc_brute_digest.restype = C.c_int
        L.orc_brute_nearest.argtypes = [_vp, _i64, _vp, _vp, _vp, _vp]
        L.orc_brute_nearest.restype = C.c_int
        L.orc_morton_codes.argtypes = [_i64, C.c_int, _vp, _vp, _vp, _vp]
        L.orc_morton_codes.restype = C.c_int
        L.orc_adjoint_points.argtypes = [_vp, _i64, _vp, _vp, _vp, C.c_int, _vp, C.c_int,
                                         C.c_int, _vp, _vp, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, _vp,
                                         _vp, _vp, _vp, _vp, _vp]
        L.orc_adjoint_points.restype = C.c_int
        L.orc_adjoint_lines.argtypes = [_vp, _i64, _vp, C.c_int, _vp, C.c_int, C.c_int, _vp, _vp, _vp,
                                        _vp, _vp, _vp, _vp, _vp]
        L.orc_adjoint_lines.restype = C.c_int
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    return lib().orc_set_threads(int(n))


def _p(a) -> int:
    return a.ctypes.data if a is not None else None


def _ptr_array(arrs):
    t = (C.c_void_p * max(len(arrs), 1))()
    for k, a in enumerate(arrs):
        t[k] = a.ctypes.data
    return t


def set_kernel(kernel: int):
    """Kernel family of the following oracle calls (M4 ... C6)."""
    if lib().orc_set_kernel(int(kernel)) != 0:
        raise ValueError(f"unknown kernel {kernel}")


def W(r, h, kernel=M4):
    set_kernel(kernel)
    return lib().orc_W(float(r), float(h))


def f(q, kernel=M4):
    set_kernel(kernel)
    return lib().orc_f(float(q))


def df(q, kernel=M4):
    set_kernel(kernel)
    return lib().orc_df(float(q))


def support(kernel=M4):
    set_kernel(kernel)
    return lib().orc_support()


def norm3(kernel=M4):
    set_kernel(kernel)
    return lib().orc_norm3()


def gradW(dx, dy, dz, h, kernel=M4):
    set_kernel(kernel)
    g = np.zeros(3)
    lib().orc_gradW(float(dx), float(dy), float(dz), float(h), g.ctypes.data)
    return g


def line_kernel(r, h, kernel=M4):
    set_kernel(kernel)
    return lib().orc_line_kernel(float(r), float(h))


def line_table(kernel=M4):
    set_kernel(kernel)
    Q = np.zeros(4096)
    I = np.zeros(4096)
    lib().orc_line_table(Q.ctypes.data, I.ctypes.data)
    return Q, I


def morton_codes(x, y, z):
    x = np.ascontiguousarray(x)
    dt = 0 if x.dtype == np.float64 else 1
    y = np.ascontiguousarray(y, dtype=x.dtype)
    z = np.ascontiguousarray(z, dtype=x.dtype)
    out = np.zeros(len(x), dtype=np.uint64)
    lib().orc_morton_codes(len(x), dt, _p(x), _p(y), _p(z), _p(out))
    return out


class Catalog:
    """Concise catalog with 0-based slots (grad slot -1 = density gradient)."""

    def __init__(self, scalars=(), shepard=None, grads=(), divs=(), curls=()):
        self.scalars = np.asarray(scalars, dtype=np.int32)
        if shepard is None:
            shepard = [1] * len(self.scalars)
        self.shepard = np.asarray(shepard, dtype=np.uint8)
        self.grads = np.asarray(grads, dtype=np.int32)
        self.divs = np.asarray(divs, dtype=np.int32).reshape(-1)
        self.curls = np.asarray(curls, dtype=np.int32).reshape(-1)

    @property
    def L(self):
        return len(self.scalars) + 3 * len(self.grads) + len(self.divs) // 3 + len(self.curls)


class Oracle:
    """One particle set + its LBVH, restated on the CPU."""

    def __init__(self, x, y, z, m, h, rho, cols=(), dtype=np.float64, kernel=M4):
        self.kernel = int(kernel)
        set_kernel(self.kernel)
        self.dtype = np.dtype(dtype)
        cv = lambda a: np.ascontiguousarray(np.asarray(a, dtype=self.dtype))
        self._keep = [cv(a) for a in (x, y, z, m, h, rho)]
        self._cols = [cv(c) for c in cols]
        self.n = len(self._keep[0])
        self._colptr = _ptr_array(self._cols)
        self.ctx = lib().orc_create(self.n, 0 if self.dtype == np.float64 else 1,
                                    *[_p(a) for a in self._keep], len(self._cols), self._colptr)
        self.perm = np.zeros(self.n, dtype=np.int64)
        self.codes = np.zeros(self.n, dtype=np.uint64)
        rc = lib().orc_build(self.ctx, _p(self.perm), _p(self.codes))
        if rc != 0:
            raise ValueError(f"oracle build failed ({rc})")

    def test_loop_escapes(self):
        """Failure injection: every walk-ending escape link points at the root."""
        rc = lib().orc_test_loop_escapes(self.ctx)
        if rc != 0:
            raise ValueError(f"oracle escape injection failed ({rc})")

    def rebuild(self):
        """orc_build again on the (already Morton-ordered) particles."""
        rc = lib().orc_build(self.ctx, None, None)
        if rc != 0:
            raise ValueError(f"oracle build failed ({rc})")

    def __del__(self):
        if getattr(self, "ctx", None):
            lib().orc_destroy(self.ctx)
            self.ctx = None

    def tree(self):
        n = self.n
        tot, nint = 2 * n - 1, max(n - 1, 0)
        root = np.zeros(1, dtype=np.int32)
        l, r, e, p = (np.zeros(tot, dtype=np.int32) for _ in range(4))
        nmin = np.zeros(3 * nint)
        nmax = np.zeros(3 * nint)
        ns = np.zeros(nint)
        rc = lib().orc_get_tree(self.ctx, _p(root), _p(l), _p(r), _p(e), _p(p), _p(nmin), _p(nmax), _p(ns))
        assert rc == 0
        return dict(root=int(root[0]), left=l, right=r, escape=e, parent=p,
                    node_min=nmin.reshape(3, nint), node_max=nmax.reshape(3, nint), node_scale=ns)

    def _s(self, a):
        return np.ascontiguousarray(np.asarray(a, dtype=self.dtype))

    def interp_points(self, sx, sy, sz, cat: Catalog, strategy=SYMMETRIC, hmode=H_NEAREST, hs=None):
        sx, sy, sz = self._s(sx), self._s(sy), self._s(sz)
        ns = len(sx)
        hsa = None if hs is None else self._s(np.atleast_1d(hs))
        outs = [np.zeros(ns, dtype=self.dtype) for _ in range(cat.L)]
        optr = _ptr_array(outs)
        set_kernel(self.kernel)
        rc = lib().orc_interp_points(self.ctx, ns, _p(sx), _p(sy), _p(sz), hmode, _p(hsa), strategy,
                                     len(cat.scalars), _p(cat.scalars), _p(cat.shepard),
                                     len(cat.grads), _p(cat.grads), len(cat.divs) // 3, _p(cat.divs),
                                     len(cat.curls) // 3, _p(cat.curls), optr)
        if rc != 0:
            raise RuntimeError(f"oracle interp_points failed ({rc})")
        return outs

    def interp_lines(self, o, d, scalars, shepard=None, strategy=SCATTER, hmode=H_PER_SAMPLE, hs=None):
        arrs = [self._s(a) for a in (*o, *d)]
        nl = len(arrs[0])
        cat = Catalog(scalars=scalars, shepard=shepard)
        hsa = None if hs is None else self._s(np.atleast_1d(hs))
        outs = [np.zeros(nl, dtype=self.dtype) for _ in range(len(cat.scalars))]
        set_kernel(self.kernel)
        rc = lib().orc_interp_lines(self.ctx, nl, _ptr_array(arrs), hmode, _p(hsa), strategy,
                                    len(cat.scalars), _p(cat.scalars), _p(cat.shepard), _ptr_array(outs))
        if rc != 0:
            raise RuntimeError(f"oracle interp_lines failed ({rc})")
        return outs

    def _grad_bufs(self):
        g = dict(m=np.zeros(self.n), x=np.zeros(self.n), y=np.zeros(self.n), z=np.zeros(self.n),
                 cols=[np.zeros(self.n) for _ in self._cols])
        return g, _ptr_array(g["cols"])

    def adjoint_points(self, sx, sy, sz, cat: Catalog, gout, strategy=SYMMETRIC, hmode=H_NEAREST, hs=None):
        """dL/dm, dL/dA_c, dL/dx for L = sum_k sum_s gout[k][s] out_k(s) (double particles), in the
        order the particles were given."""
        sx, sy, sz = self._s(sx), self._s(sy), self._s(sz)
        hsa = None if hs is None else self._s(np.atleast_1d(hs))
        go = [np.ascontiguousarray(g, dtype=np.float64) for g in gout]
        g, cptr = self._grad_bufs()
        set_kernel(self.kernel)
        rc = lib().orc_adjoint_points(self.ctx, len(sx), _p(sx), _p(sy), _p(sz), hmode, _p(hsa), strategy,
                                      len(cat.scalars), _p(cat.scalars), _p(cat.shepard),
                                      len(cat.grads), _p(cat.grads), len(cat.divs) // 3, _p(cat.divs),
                                      len(cat.curls) // 3, _p(cat.curls), _ptr_array(go),
                                      _p(g["m"]), cptr, _p(g["x"]), _p(g["y"]), _p(g["z"]))
        if rc != 0:
            raise RuntimeError(f"oracle adjoint_points failed ({rc})")
        return g

    def adjoint_lines(self, o, d, scalars, gout, shepard=None, strategy=SCATTER, hmode=H_PER_SAMPLE, hs=None):
        arrs = [self._s(a) for a in (*o, *d)]
        cat = Catalog(scalars=scalars, shepard=shepard)
        hsa = None if hs is None else self._s(np.atleast_1d(hs))
        go = [np.ascontiguousarray(g, dtype=np.float64) for g in gout]
        g, cptr = self._grad_bufs()
        set_kernel(self.kernel)
        rc = lib().orc_adjoint_lines(self.ctx, len(arrs[0]), _ptr_array(arrs), hmode, _p(hsa), strategy,
                                     len(cat.scalars), _p(cat.scalars), _p(cat.shepard), _ptr_array(go),
                                     _p(g["m"]), cptr, _p(g["x"]), _p(g["y"]), _p(g["z"]))
        if rc != 0:
            raise RuntimeError(f"oracle adjoint_lines failed ({rc})")
        return g

    def density(self, sx, sy, sz, strategy=GATHER, hmode=H_PER_SAMPLE, hs=None, number=False):
        """_density_kernel (sum m W), or _number_density_kernel (sum W) with number=True."""
        sx, sy, sz = self._s(sx), self._s(sy), self._s(sz)
        hsa = None if hs is None else self._s(np.atleast_1d(hs))
        out = np.zeros(len(sx), dtype=self.dtype)
        set_kernel(self.kernel)
        rc = lib().orc_density(self.ctx, len(sx), _p(sx), _p(sy), _p(sz), hmode, _p(hsa), strategy, _p(out),
                               1 if number else 0)
        if rc != 0:
            raise RuntimeError(f"oracle density failed ({rc})")
        return out

    def gradient_density(self, sx, sy, sz, strategy=GATHER, hmode=H_PER_SAMPLE, hs=None):
        """_gradient_density_kernel: sum m gradW - rho(r) sum (m/rho_b) gradW, NaN where rho(r) = 0."""
        sx, sy, sz = self._s(sx), self._s(sy), self._s(sz)
        hsa = None if hs is None else self._s(np.atleast_1d(hs))
        out = np.zeros(3 * len(sx), dtype=self.dtype)
        set_kernel(self.kernel)
        rc = lib().orc_density(self.ctx, len(sx), _p(sx), _p(sy), _p(sz), hmode, _p(hsa), strategy, _p(out), 2)
        if rc != 0:
            raise RuntimeError(f"oracle gradient density failed ({rc})")
        return out.reshape(3, len(sx))

    def digest(self, a, d=None, strategy=SYMMETRIC, hmode=H_NEAREST, hs=None):
        kind = 0 if d is None else 1
        arrs = [self._s(v) for v in a] + ([self._s(v) for v in d] if d is not None else [])
        ns = len(arrs[0])
        hsa = None if hs is None else self._s(np.atleast_1d(hs))
        cnt = np.zeros(ns, dtype=np.int64)
        hsh = np.zeros(ns, dtype=np.uint64)
        ha = np.zeros(ns, dtype=self.dtype)
        set_kernel(self.kernel)
        rc = lib().orc_neighbor_digest(self.ctx, kind, ns, _ptr_array(arrs), hmode, _p(hsa), strategy,
                                       _p(cnt), _p(hsh), _p(ha))
        if rc != 0:
            raise RuntimeError(f"oracle digest failed ({rc})")
        return cnt, hsh, ha

    def brute_digest(self, a, ha, d=None, strategy=SYMMETRIC):
        kind = 0 if d is None else 1
        arrs = [self._s(v) for v in a] + ([self._s(v) for v in d] if d is not None else [])
        ns = len(arrs[0])
        haa = self._s(np.broadcast_to(np.asarray(ha), (ns,)))
        cnt = np.zeros(ns, dtype=np.int64)
        hsh = np.zeros(ns, dtype=np.uint64)
        set_kernel(self.kernel)
        lib().orc_brute_digest(self.ctx, kind, ns, _ptr_array(arrs), _p(haa), strategy, _p(cnt), _p(hsh))
        return cnt, hsh

    def brute_nearest(self, sx, sy, sz):
        sx, sy, sz = (np.ascontiguousarray(v, dtype=np.float64) for v in (sx, sy, sz))
        idx = np.zeros(len(sx), dtype=np.int64)
        lib().orc_brute_nearest(self.ctx, len(sx), _p(sx), _p(sy), _p(sz), _p(idx))
        return idx


def mix64(v: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser, vectorised (the neighbour-digest hash)."""
    v = np.asarray(v, dtype=np.uint64).copy()
    with np.errstate(over="ignore"):
        v += np.uint64(0x9E3779B97F4A7C15)
        v = (v ^ (v >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        v = (v ^ (v >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        v = v ^ (v >> np.uint64(31))
    return v
