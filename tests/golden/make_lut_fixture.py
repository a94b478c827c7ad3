"""Sample the reference's line-integrated kernel tables into a small golden fixture.

Reads src/julia/KernelInterpolation/table/line_integrated_kernel_tables.jl of a
Partia.jl checkout (first argument, else $PARTIA_REFERENCE_DIR) and writes, for
each kernel family, every 64th entry of _<K>_Q and _<K>_Inorm (64 + the last
entry) and the grid spacing Q[2] - Q[1] to line_table_samples.json next to
this script.  The full tables are not copied.
"""
import json
import os
import sys

import numpy as np

KERNELS = ["M4_spline", "M5_spline", "M6_spline", "C2_Wendland", "C4_Wendland", "C6_Wendland"]


def parse_table(root, name):
    path = os.path.join(root, "src/julia/KernelInterpolation/table/line_integrated_kernel_tables.jl")
    src = open(path).read()
    i = src.index(f"const {name} = SVector{{4096,Float64}}(")
    j = src.index(")", i + 40)
    body = src[i:j].split("(", 1)[1]
    return np.array([float(t) for t in body.replace("\n", "").split(",") if t.strip()])


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PARTIA_REFERENCE_DIR", "")
    if not root or not os.path.isdir(root):
        sys.exit("usage: make_lut_fixture.py <Partia.jl checkout>  (or set PARTIA_REFERENCE_DIR)")
    idx = list(range(0, 4096, 64)) + [4095]
    out = {"source": "table/line_integrated_kernel_tables.jl (_<K>_Q, _<K>_Inorm)", "index0": idx, "kernels": {}}
    for k in KERNELS:
        Q = parse_table(root, f"_{k}_Q")
        I = parse_table(root, f"_{k}_Inorm")
        out["kernels"][k] = {"Q": [repr(float(Q[i])) for i in idx], "Inorm": [repr(float(I[i])) for i in idx],
                             "dq": repr(float(Q[1] - Q[0]))}
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "line_table_samples.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
