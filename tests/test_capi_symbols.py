"""The C-ABI library loads and exports every function include/partia_b200.h
declares; host-only calls behave without a GPU."""
import ctypes as C
import os
import subprocess

import pytest

from partia_b200 import _lib as L


def test_library_built_and_exports_header_symbols():
    assert os.path.exists(L.LIB_PATH), "build with make -C partia.jl_b200/csrc"
    lib = L.load()
    declared = L.header_symbols()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(declared) <= exported
    # nothing else is exported from the product library
    assert {s for s in exported if s.startswith("psb_")} == set(declared)


def test_abi_version_and_null_context_handling():
    lib = L.load()
    assert lib.psb_abi_version() == 1
    assert lib.psb_destroy(None) == L.PSB_OK
    assert lib.psb_last_error(None) == b"null context"
    assert lib.psb_build_lbvh(None, None, None) == L.PSB_EINVAL
    assert lib.psb_create(None, 0) == L.PSB_EINVAL


def test_header_compiles_as_c():
    src = '#include "partia_b200.h"\nint main(void){ psb_stats s; psb_catalog c; (void)s; (void)c; return 0; }\n'
    inc = os.path.dirname(L.HEADER_PATH)
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", inc, "-x", "c", "-", "-fsyntax-only"],
                       input=src, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_struct_layouts_match_python_binding():
    # psb_stats / psb_catalog sizes as seen by C
    src = ('#include <stdio.h>\n#include "partia_b200.h"\n'
           'int main(void){ printf("%zu %zu\\n", sizeof(psb_stats), sizeof(psb_catalog)); return 0; }\n')
    inc = os.path.dirname(L.HEADER_PATH)
    exe = "/tmp/psb_sizes"
    r = subprocess.run(["gcc", "-std=c99", "-I", inc, "-x", "c", "-", "-o", exe], input=src, capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    a, b = map(int, subprocess.run([exe], capture_output=True, text=True).stdout.split())
    assert a == C.sizeof(L.Stats) and b == C.sizeof(L.Catalog)


def test_flag_constants_match_header():
    import re
    with open(L.HEADER_PATH) as f:
        hdr = f.read()
    names = re.findall(r"#define\s+(PSB_FLAG_\w+)\s", hdr)
    assert len(names) >= 4
    for name in names:
        m = re.search(r"#define\s+%s\s+(0x[0-9a-fA-F]+|\d+)u" % name, hdr)
        assert m and int(m.group(1), 0) == getattr(L, name), name


def test_julia_binding_calls_only_declared_symbols():
    """The Julia package (partia.jl_b200/julia/PartiaB200) ccalls only functions
    the header declares, and binds every driver entry point Partia's CUDA
    extension methods need.  (Julia is not in this image; this checks the
    source against the ABI.)"""
    import re
    root = os.path.join(os.path.dirname(os.path.dirname(L.HEADER_PATH)), "partia.jl_b200", "julia", "PartiaB200")
    srcs = []
    for d, _, files in os.walk(root):
        srcs += [open(os.path.join(d, f)).read() for f in files if f.endswith(".jl")]
    called = set(re.findall(r"ccall\(\(:(psb_\w+), libpsb\)", "\n".join(srcs)))
    declared = set(L.header_symbols())
    assert called <= declared, called - declared
    assert {"psb_create", "psb_destroy", "psb_last_error", "psb_set_particles", "psb_set_values", "psb_build_lbvh",
            "psb_interp_points", "psb_interp_lines", "psb_adjoint_points"} <= called
    proj = open(os.path.join(root, "Project.toml")).read()
    assert "Partia" in proj and "ChainRulesCore" in proj
