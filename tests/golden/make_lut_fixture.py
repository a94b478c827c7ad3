"""Sample the reference's M4 line-integrated table into a small golden fixture.

Reads src/julia/KernelInterpolation/table/line_integrated_kernel_tables.jl of a
Partia.jl checkout (first argument, default /root/reference) and writes every
64th entry of _M4_spline_Q and _M4_spline_Inorm (64 + the last entry) to
m4_line_table_samples.json next to this script.  The full table is not copied.
"""
import json
import os
import sys

import numpy as np


def parse_table(root, name):
    path = os.path.join(root, "src/julia/KernelInterpolation/table/line_integrated_kernel_tables.jl")
    src = open(path).read()
    i = src.index(f"const {name} = SVector{{4096,Float64}}(")
    j = src.index(")", i + 40)
    body = src[i:j].split("(", 1)[1]
    return np.array([float(t) for t in body.replace("\n", "").split(",") if t.strip()])


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    Q = parse_table(root, "_M4_spline_Q")
    I = parse_table(root, "_M4_spline_Inorm")
    idx = list(range(0, 4096, 64)) + [4095]
    out = {"source": "table/line_integrated_kernel_tables.jl (_M4_spline_Q, _M4_spline_Inorm)",
           "index0": idx, "Q": [repr(float(Q[k])) for k in idx], "Inorm": [repr(float(I[k])) for k in idx],
           "dq": repr(float(Q[1] - Q[0]))}
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "m4_line_table_samples.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
