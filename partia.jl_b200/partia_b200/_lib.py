"""ctypes binding of libpartia_b200.so (include/partia_b200.h).

The library is the only compute path: if it is missing or fails to load, every
call raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
# the in-tree build, unless PARTIA_B200_LIB names another build of the same ABI
LIB_PATH = os.environ.get("PARTIA_B200_LIB") or os.path.join(_HERE, "_lib", "libpartia_b200.so")
HEADER_PATH = os.path.normpath(os.path.join(_HERE, "..", "..", "include", "partia_b200.h"))

PSB_OK = 0
PSB_EINVAL = -1
PSB_EDIM = -2
PSB_ENOMEM = -3
PSB_ECUDA = -4
PSB_ETRAVERSAL = -5
PSB_EUNSUPPORTED = -6
PSB_ESTATE = -7

PSB_F64, PSB_F32 = 0, 1
PSB_KERNEL_M4, PSB_KERNEL_M5, PSB_KERNEL_M6, PSB_KERNEL_C2, PSB_KERNEL_C4, PSB_KERNEL_C6 = 0, 1, 2, 3, 4, 5
PSB_GATHER, PSB_SCATTER, PSB_SYMMETRIC = 0, 1, 2
PSB_PREC_FP64, PSB_PREC_FP32C = 0, 1
PSB_H_NEAREST, PSB_H_PER_SAMPLE, PSB_H_CONSTANT = 0, 1, 2
PSB_FLAG_DEVICE_PTRS = 1
PSB_FLAG_FP32C_DECISIONS = 0x100
PSB_FLAG_SINGLE_KERNEL = 0x200
PSB_FLAG_LUT1000_F32 = 0x400
PSB_FLAG_DENSITY_GRADIENT_PLAIN = 0x800
PSB_FLAG_NUMBER_DENSITY = 0x1000
PSB_NOALLOC_MAX_SAMPLES = 262144


class PsbError(RuntimeError):
    """A negative status returned by the library."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Catalog(C.Structure):
    _fields_ = [
        ("n_scalar", C.c_int32), ("scalar_slots", C.c_void_p), ("scalar_shepard", C.c_void_p),
        ("n_grad", C.c_int32), ("grad_slots", C.c_void_p),
        ("n_div", C.c_int32), ("div_slots", C.c_void_p),
        ("n_curl", C.c_int32), ("curl_slots", C.c_void_p),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("total_ms", C.c_double), ("h2d_ms", C.c_double), ("order_ms", C.c_double),
        ("nearest_ms", C.c_double), ("interp_ms", C.c_double), ("d2h_ms", C.c_double),
        ("pairs", C.c_int64), ("exact_retests", C.c_int64), ("warp_steps", C.c_int64), ("spans", C.c_int64),
        ("span_tests", C.c_int64), ("body_iters", C.c_int64), ("launches", C.c_int32),
        ("reserved", C.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


_vp, _i64, _i32, _u32 = C.c_void_p, C.c_int64, C.c_int32, C.c_uint32
_SIGS = {
    "psb_abi_version": ([], _i32),
    "psb_create": ([C.POINTER(_vp), C.c_int], C.c_int),
    "psb_destroy": ([_vp], C.c_int),
    "psb_last_error": ([_vp], C.c_char_p),
    "psb_set_stream": ([_vp, _vp], C.c_int),
    "psb_set_particles": ([_vp, _i64, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _vp, C.c_int, _u32], C.c_int),
    "psb_build_lbvh": ([_vp, _vp, _vp], C.c_int),
    "psb_set_values": ([_vp, _vp, _vp, _i32, _vp, _u32], C.c_int),
    "psb_test_loop_escapes": ([_vp], C.c_int),
    "psb_test_adjoint_pool": ([_vp, C.c_int64, C.c_int32], C.c_int),
    "psb_baseline_cudaext_points": ([_vp, _i64] + [_vp] * 6 + [_i32, _vp, C.c_int, _i32] + [_vp] * 5 +
                                    [_i64, _vp, _vp, _vp, C.c_int, _vp, _vp, _vp], C.c_int),
    "psb_get_tree": ([_vp] * 9, C.c_int),
    "psb_interp_points": ([_vp, _i64, _vp, _vp, _vp, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, _u32, _vp], C.c_int),
    "psb_adjoint_points": ([_vp, _i64, _vp, _vp, _vp, C.c_int, _vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                            _u32, _vp], C.c_int),
    "psb_adjoint_grid": ([_vp, _vp, _i64, _vp, _i64, _vp, _i64, C.c_int, _vp, C.c_int, _vp, _vp, _vp, _vp, _vp,
                          _vp, _vp, _u32, _vp], C.c_int),
    "psb_adjoint_beam": ([_vp, _vp, _vp, _i64, _i64, C.c_int, _vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                          _u32, _vp], C.c_int),
    "psb_interp_points_noalloc": ([_vp, _i64, _vp, _vp, _vp, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, _vp],
                                  C.c_int),
    "psb_interp_grid": ([_vp, _vp, _i64, _vp, _i64, _vp, _i64, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, _u32, _vp],
                        C.c_int),
    "psb_interp_box": ([_vp, _vp, _vp, _i64, _i64, _i64, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, _u32, _vp],
                       C.c_int),
    "psb_interp_lines": ([_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, _u32,
                          _vp], C.c_int),
    "psb_interp_beam": ([_vp, _vp, _vp, _i64, _i64, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, _u32, _vp], C.c_int),
    "psb_density": ([_vp, _i64, _vp, _vp, _vp, C.c_int, _vp, C.c_int, C.c_int, _vp, _u32, _vp], C.c_int),
    "psb_neighbor_digest": ([_vp, _i32, _i64, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int, _vp, C.c_int, _vp, _vp, _vp,
                             _u32], C.c_int),
}

_lib = None


def header_symbols(path: str = HEADER_PATH) -> list[str]:
    """Every function declared in include/partia_b200.h."""
    text = open(path).read()
    return sorted(set(re.findall(r"^\s*(?:int|int32_t|const char\*)\s+(psb_\w+)\s*\(", text, re.M)))


def load():
    """Load the CUDA library (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libpartia_b200.so not found at {LIB_PATH}; build it with `make -C partia.jl_b200/csrc` "
            "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    for name, (args, res) in _SIGS.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def check(ctx, rc: int):
    if rc != PSB_OK:
        msg = load().psb_last_error(ctx)
        raise PsbError(rc, msg.decode() if msg else "")
