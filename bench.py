"""Benchmark of the SPH interpolation hot path on B200.

Workload (one step): the Plummer-sphere configuration -- N = 2,000,000
particles (a = 0.1, truncated at 10a, seed 1), symmetric strategy with
nearest-particle h, outputs rho, grad rho, div A, curl A (8 fields) on the
128^3 StructuredGrid over [-0.5, 0.5]^3, FP32C arithmetic (float pair sums with
compensated accumulation; double inclusion test and finalisation).  The FP64
path is timed beside it.

value: samples/s with particles, LBVH and outputs resident in HBM (grid
coordinates generated on the device), device time from CUDA events.
e2e:   the same metric through the C ABI with host buffers: the host sample
coordinates (pinned) are copied in and the 8 output fields copied out inside
the timed region every step, timed with the host clock around each call
(a pageable-buffer variant is reported beside it).

Multi-GPU: samples shard over ranks (each rank owns a contiguous slab of
z-planes of the grid, the slabs cut for equal estimated pair counts from a
coarse neighbour-digest pass; the particle set and its LBVH are replicated);
there is no data-path collective, and the total work is fixed (strong
scaling).  --impl reference times the CPU restatement of the
reference's multithreaded CPU path (oracle/, "port") on the host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "partia.jl_b200"))

METRIC = "samples/s & HBM-roofline frac: FP32 vs FP64 path at stated err; grad/fwd time"
UNIT = "samples/s"
NGRID = 128
CATALOG = dict(scalars=[0], shepard=[0], grads=[0], divs=[1, 2, 3], curls=[1, 2, 3])  # cols: rho, Ax, Ay, Az
L_OUT = 8
NCOL_USED = 4


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """DRAM bytes per launch of the point kernel from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "split_c2_traffic.json")) as f:
            return json.load(f)
    except Exception:
        return None


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region through NVML (read-only queries, every 10 ms); nvidia-smi when NVML
    is unavailable."""

    REASONS = [("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown")]

    def __init__(self, cuda_index=0):
        self.cuda_index = cuda_index
        self.samples = []   # (sm_mhz, max_mhz, [reasons])
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        self._h = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            props = torch.cuda.get_device_properties(cuda_index)
            try:
                self._h = pynvml.nvmlDeviceGetHandleByUUID("GPU-" + str(props.uuid))
            except Exception:
                bus = "%08x:%02x:%02x.0" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
                self._h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            self._nvml = pynvml
        except Exception:
            self._nvml = None

    def _sample_nvml(self):
        nv = self._nvml
        sm = nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(self._h, nv.NVML_CLOCK_SM)
        bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
        rs = [name for name, const in self.REASONS if bits & getattr(nv, const, 0)]
        self.samples.append((float(sm), float(mx), rs))

    def _sample_smi(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        out = subprocess.run(["nvidia-smi", "-i", str(self.cuda_index), f"--query-gpu={q}",
                              "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
        v = [x.strip() for x in out.stdout.strip().split(",")]
        if len(v) >= 6:
            rs = [self.REASONS[k][0] for k in range(4) if v[2 + k].lower() == "active"]
            self.samples.append((float(v[0]), float(v[1]), rs))

    def _run(self):
        while not self._stop.is_set():
            try:
                self._sample_nvml() if self._nvml else self._sample_smi()
            except Exception:
                pass
            self._stop.wait(0.01 if self._nvml else 0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [s[0] for s in self.samples]
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(s[1] for s in self.samples),
                "sm_mhz_min": min(sm), "reasons": sorted({r for s in self.samples for r in s[2]}),
                "samples": len(self.samples), "source": "nvml" if self._nvml else "nvidia-smi"}


def bench_config():
    """The workload description both arms print (the driver compares them)."""
    return {"workload": f"plummer-2M symmetric rho,grad rho,div A,curl A on {NGRID}^3 grid",
            "N": 2_000_000, "samples": NGRID ** 3, "fields": L_OUT, "strategy": "symmetric",
            "h": "nearest particle", "l2": "flushed (256 MB write) between GPU steps"}


def host_cpu():
    """nproc and the CPU model name of this host (lscpu)."""
    model = None
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for ln in out.splitlines():
            if ln.startswith("Model name:"):
                model = ln.split(":", 1)[1].strip()
                break
    except Exception:
        pass
    return {"nproc": os.cpu_count(), "model": model}


def roofline_block(b_alg, ms, what):
    """HBM-roofline fraction of an algorithmic byte count moved in ms."""
    hbm, kind = peaks()
    achieved = b_alg / (ms / 1e3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "peak_kind": kind, "alg_bytes": int(b_alg), "ms": ms, "bytes": what}


def make_workload():
    from partia_b200 import workloads as W
    from partia_b200 import linrange
    d = W.plummer_c2()
    axis = linrange(-0.5, 0.5, NGRID)
    return d, axis


def timed_call(fn, stream, steps, warmup):
    """Median device time (ms) of fn() over `steps` calls after `warmup`, CUDA events on `stream`."""
    import torch
    for _ in range(warmup):
        fn()
    ms = []
    for _ in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    return float(np.median(ms))


def cudaext_leg(ctx, d, axis, steps, warmup, ours):
    """The reference's CUDA-extension design on the same workload
    (psb_baseline_cudaext_points: one thread per sample, per-thread DFS, FP64;
    particles, tree and samples copied from pageable host memory and the 8
    fields copied back in every call).  Its LBVH comes from this library's
    build (the reference builds it on the CPU, which is not timed here)."""
    import torch
    from partia_b200.engine import CatalogC
    perm, _ = ctx.build(want_perm=True)
    tree = ctx.tree()
    parts = {k: np.ascontiguousarray(d[k][perm]) for k in ("x", "y", "z", "m", "h", "rho")}
    parts["cols"] = [np.ascontiguousarray(d[k][perm]) for k in ("rho", "Ax", "Ay", "Az")]
    n = len(axis)
    X, Y, Z = np.meshgrid(axis, axis, axis, indexing="ij")
    s = [np.ascontiguousarray(a.ravel(order="F")) for a in (X, Y, Z)]
    cat = CatalogC(**CATALOG)
    for _ in range(warmup):
        ctx.baseline_cudaext_points(parts, tree, *s, cat)
    host, kern, tot = [], [], []
    for _ in range(steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.baseline_cudaext_points(parts, tree, *s, cat)
        host.append(time.perf_counter() - t0)
        kern.append(ctx.last_stats.interp_ms)
        tot.append(ctx.last_stats.total_ms)
    pairs = int(ctx.last_stats.pairs)
    kms, hms = float(np.median(kern)), 1e3 * float(np.median(host))
    ns = n ** 3
    return {"design": "one thread per sample (256/block), per-thread stackless DFS for nearest h and the FP64 "
                      "general kernel; particles, tree and samples H2D and outputs D2H in every call "
                      "(ext/CUDAExt/.../PointSamples_driver.jl:12-27, kernels/PointSamples_kernel.jl:1-68)",
            "kernel_ms": kms, "e2e_ms": hms, "event_ms": float(np.median(tot)), "pairs": pairs,
            "samples_per_s_device": ns / (kms / 1e3), "samples_per_s_e2e": ns / (hms / 1e3),
            "not_timed": "the reference's CPU LBVH build (the tree is this library's, uploaded every call)",
            "vs_cudaext_design": {"device_fp32c": kms / ours["fp32c_ms"], "device_fp64": kms / ours["fp64_ms"],
                                  "e2e": hms / ours["e2e_ms"]}}


def lines_and_adjoint(steps, warmup, n_lines=8_000_000, npix_lines=1024):
    """The line-integrated configurations (clump particles, parallel beam through
    the 30/45-degree frame over [0,1]^2, scatter, column density = plain scalar
    rho): forward throughput of 8M particles x 1024^2 lines in FP32C and FP64,
    and the adjoint of 0.5 ||Sigma - Sigma_target||^2 for 1M particles x 512^2
    lines against its forward.  Particles and outputs stay on the device."""
    import torch
    from partia_b200 import _lib as L, workloads as W
    from partia_b200.engine import CatalogC, Context
    stream = torch.cuda.Stream()
    fr = W.c3_frame().as_array()
    prm = np.array([0.0, 1.0, 0.0, 1.0])
    cat = CatalogC(scalars=[0], shepard=[0])
    res = {}

    def context(d, h, rho):
        ctx = Context(0)
        L.load().psb_set_stream(ctx.h, stream.cuda_stream)
        ctx.set_particles(d["x"], d["y"], d["z"], d["m"], h, rho, [rho])
        ctx.build(want_perm=False)
        return ctx

    # 8M particles, 1024^2 lines
    d = W.clumps(n_lines, 2)
    h, rho = W.density_h(d)
    ctx = context(d, h, rho)
    npix = npix_lines
    out32 = [torch.empty(npix * npix, dtype=torch.float64, device="cuda")]
    out64 = [torch.empty(npix * npix, dtype=torch.float64, device="cuda")]
    f32 = lambda: ctx.interp_beam(fr, prm, npix, npix, cat, strategy=L.PSB_SCATTER, prec=L.PSB_PREC_FP32C, out=out32)
    f64 = lambda: ctx.interp_beam(fr, prm, npix, npix, cat, strategy=L.PSB_SCATTER, prec=L.PSB_PREC_FP64, out=out64)
    t32 = timed_call(f32, stream, steps, warmup)
    pairs = ctx.last_stats.pairs
    t64 = timed_call(f64, stream, max(2, steps // 2), 1)
    a, b = out32[0], out64[0]
    fin = torch.isfinite(b)
    err = ((a[fin] - b[fin]).abs().max() / b[fin].abs().max()).item()
    # the 1000-entry float table of the line integral, against the 4096-entry FP64 result
    ctx.extra_flags = L.PSB_FLAG_LUT1000_F32
    t1000 = timed_call(f32, stream, steps, warmup)
    ctx.extra_flags = 0
    err1000 = ((out32[0][fin] - b[fin]).abs().max() / b[fin].abs().max()).item()
    res["lines"] = {"workload": f"clumps-{n_lines / 1e6:g}M column density, {npix}^2 parallel beam, scatter",
                    "N": n_lines,
                    "lines": npix * npix, "pairs": int(pairs), "fp32c_ms": t32, "fp64_ms": t64,
                    "lines_per_s": npix * npix / (t32 / 1e3), "fp64_lines_per_s": npix * npix / (t64 / 1e3),
                    "speedup_fp32c_vs_fp64": t64 / t32, "fp32c_rel_err_vs_fp64": err,
                    "lut1000_f32": {"fp32c_ms": t1000, "rel_err_vs_fp64_lut4096": err1000},
                    # beam lines are generated on the device (S_in = 0); 1 output of 8 B per line;
                    # the FP32C pair record is x, y, z, h, m, rho + 1 column in float (28 B)
                    "roofline": roofline_block(npix * npix * 8 + int(pairs) * (6 + 1) * 4, t32,
                                               "lines x 8 B out + pairs x 28 B (FP32C records)")}
    ctx.close()
    del out32, out64

    # 1M particles, 512^2 lines: forward and adjoint
    d = W.clumps(1_000_000, 3)
    h, rho = W.density_h(d)
    ctx = context(d, h, rho)
    rng = np.random.default_rng(1003)
    dt = dict(d)
    dt["m"] = d["m"] * (1.0 + 0.1 * rng.standard_normal(len(d["m"])))
    for k in ("x", "y", "z"):
        dt[k] = d[k] + 0.002 * rng.standard_normal(len(d[k]))
    npix = 512
    tgt = [torch.empty(npix * npix, dtype=torch.float64, device="cuda")]
    ctx_t = context(dt, h, rho)
    ctx_t.interp_beam(fr, prm, npix, npix, cat, strategy=L.PSB_SCATTER, prec=L.PSB_PREC_FP64, out=tgt)
    ctx_t.close()
    sig = [torch.empty(npix * npix, dtype=torch.float64, device="cuda")]
    fwd = lambda: ctx.interp_beam(fr, prm, npix, npix, cat, strategy=L.PSB_SCATTER, prec=L.PSB_PREC_FP32C, out=sig)
    tf = timed_call(fwd, stream, steps, warmup)
    fwd64 = lambda: ctx.interp_beam(fr, prm, npix, npix, cat, strategy=L.PSB_SCATTER, prec=L.PSB_PREC_FP64, out=sig)
    tf64 = timed_call(fwd64, stream, max(2, steps // 2), 1)
    gout = [torch.nan_to_num(sig[0] - tgt[0])]
    bwd = lambda: ctx.adjoint_beam(fr, prm, npix, npix, cat, gout, strategy=L.PSB_SCATTER, device=True)
    tb = timed_call(bwd, stream, steps, warmup)
    res["adjoint"] = {"workload": "clumps-1M column density, 512^2 parallel beam, loss 0.5||Sigma - Sigma_target||^2",
                      "N": 1_000_000, "lines": npix * npix, "pairs": int(ctx.last_stats.pairs),
                      "forward_fp32c_ms": tf, "forward_fp64_ms": tf64, "backward_ms": tb,
                      "grad_fwd_time_ratio": tb / tf, "grad_fwd_time_ratio_vs_fp64": tb / tf64,
                      "gradients": "dL/dm, dL/drho-column, dL/dx (FP64)"}
    ctx.close()
    return res


def large_leg(steps, warmup, oracle_check=True, n=64_000_000, ng=256):
    """The large mixed configuration: 64M float32 particles (70% exponential
    disc, 30% Plummer halo; h and rho from the density sum), rho, Shepard z^2,
    grad rho and curl v on a 256^3 grid over [-1,1]^3 plus four randomly
    oriented 128^3 boxes over [-0.5,0.5]^3 (25.2M samples), symmetric,
    nearest-particle h.  FP32C against the all-FP64 path on the same particle
    values (the float32 data converted to double on the device), and the
    float32-storage path (the reference's Float32 semantics) beside them."""
    import math
    import torch
    from partia_b200 import _lib as L, workloads as W, linrange
    from partia_b200.engine import CatalogC, Context
    stream = torch.cuda.Stream()
    d = W.disc_halo_c5(n)
    h, rho = W.density_h(d)
    cols = [rho, d["vx"], d["vy"], d["vz"], d["z2"]]
    cat = CatalogC(scalars=[0, 4], shepard=[0, 1], grads=[0], curls=[1, 2, 3])
    rng = np.random.default_rng(4)
    frames = []
    for _ in range(4):
        fr = W.Frame((0.0, 0.0, 0.0), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0))
        fr.rotate(*rng.uniform(-math.pi, math.pi, 3))
        frames.append(fr.as_array())
    bprm = np.array([-0.5, 0.5, -0.5, 0.5, -0.5, 0.5])
    nb = ng // 2
    ax = linrange(-1.0, 1.0, ng)
    res = {}
    outs = {}
    ns = ng ** 3 + len(frames) * nb ** 3
    runs = {torch.float32: [("float32_storage", L.PSB_PREC_FP32C)],
            torch.float64: [("fp32c", L.PSB_PREC_FP32C), ("fp64", L.PSB_PREC_FP64)]}
    for dt, legs in runs.items():
        ctx = Context(0)
        L.load().psb_set_stream(ctx.h, stream.cuda_stream)
        dev = [torch.from_numpy(a).cuda().to(dt) for a in (d["x"], d["y"], d["z"], d["m"], h, rho)]
        dcols = [torch.from_numpy(c).cuda().to(dt) for c in cols]
        ctx.set_particles(*dev, cols=dcols)
        ctx.build(want_perm=False)
        del dev, dcols
        go = [torch.empty(ng ** 3, dtype=dt, device="cuda") for _ in range(8)]
        bo = [[torch.empty(nb ** 3, dtype=dt, device="cuda") for _ in range(8)] for _ in frames]
        for label, prec in legs:
            pairs = [0]

            def step():
                ctx.interp_grid(ax, ax, ax, cat, strategy=L.PSB_SYMMETRIC, prec=prec, out=go)
                p = ctx.last_stats.pairs
                for fa, o in zip(frames, bo):
                    ctx.interp_box(fa, bprm, nb, nb, nb, cat, strategy=L.PSB_SYMMETRIC, prec=prec, out=o)
                    p += ctx.last_stats.pairs
                pairs[0] = p

            t = timed_call(step, stream, steps, warmup)
            res[label] = {"ms": t, "samples_per_s": ns / (t / 1e3), "pairs": int(pairs[0])}
            outs[label] = [torch.cat([go[k].double()] + [o[k].double() for o in bo]) for k in range(8)]
        if dt == torch.float64:
            res["adjoint"] = large_adjoint(ctx, ax, stream, steps, warmup, torch.from_numpy(cols[4]).cuda().double(),
                                           torch.from_numpy(d["m"]).cuda().double())
        ctx.close()
        del go, bo
        torch.cuda.empty_cache()
    names = ["rho", "z2", "grad_rho_x", "grad_rho_y", "grad_rho_z", "curl_v_x", "curl_v_y", "curl_v_z"]

    def errs(a_, b_):
        e = {}
        for k in range(8):
            a, b = a_[k], b_[k]
            fin = torch.isfinite(b) & torch.isfinite(a)
            e[names[k]] = ((a[fin] - b[fin]).abs().max() / b[fin].abs().max()).item()
        return e
    ora = oracle_subset(d, h, rho, cols, ax, frames, bprm, nb, outs, names) if oracle_check else None
    res["float32_storage"]["note"] = ("particle data kept in float32; inclusion tests and nearest-particle h in float "
                                      "arithmetic, as the reference computes with Float32 inputs")
    res["fp32c"]["particles"] = res["fp64"]["particles"] = "the float32 values converted to double on the device"
    return {"workload": f"disc+halo {n / 1e6:g}M, {ng}^3 grid + 4 oriented {nb}^3 boxes, symmetric, nearest h",
            "N": n, "samples": ns, "fp32c": res["fp32c"], "fp64": res["fp64"],
            "float32_storage": res["float32_storage"],
            "speedup_fp32c_vs_fp64": res["fp64"]["ms"] / res["fp32c"]["ms"],
            "fp32c_rel_err_vs_fp64": errs(outs["fp32c"], outs["fp64"]),
            "float32_storage_rel_err_vs_fp64": errs(outs["float32_storage"], outs["fp64"]),
            "oracle_subset": ora, "adjoint": res["adjoint"],
            # grid and box samples are generated on the device (S_in = 0); 8 outputs of 8 B;
            # the FP32C pair record is x, y, z, h, m, rho + 5 columns in float (44 B)
            "roofline": roofline_block(ns * 8 * 8 + res["fp32c"]["pairs"] * (6 + 5) * 4, res["fp32c"]["ms"],
                                       "samples x 64 B out + pairs x 44 B (FP32C records)")}


def kernel_families(d, axis, steps, warmup):
    """The Plummer workload (8 fields, symmetric, nearest h, 128^3 grid) with
    each kernel family of kernels/*.jl: FP32C and FP64 device time, accepted
    pairs (the support K h sets the neighbour count) and the largest FP32C vs
    FP64 field error; and the adjoint of L = sum_k <gout_k, out_k> (seeded
    normal gout, all 8 fields, the gradients with respect to m_b, A_b and r_b)
    against the FP32C forward.  Every field is linear in the columns, so
    sum_c <dL/dA_c, A_c> = L at any size: its relative residual is reported."""
    import torch
    from partia_b200 import _lib as L
    from partia_b200.engine import CatalogC, Context
    stream = torch.cuda.Stream()
    cat = CatalogC(**CATALOG)
    colsd = [torch.from_numpy(np.ascontiguousarray(d[k])).cuda() for k in ("rho", "Ax", "Ay", "Az")]
    gen = torch.Generator(device="cuda").manual_seed(7)
    names = ["M4_spline", "M5_spline", "M6_spline", "C2_Wendland", "C4_Wendland", "C6_Wendland"]
    ns = len(axis) ** 3
    res = {}
    for kid, name in enumerate(names):
        ctx = Context(0)
        L.load().psb_set_stream(ctx.h, stream.cuda_stream)
        ctx.set_particles(d["x"], d["y"], d["z"], d["m"], d["h"], d["rho"], [d["rho"], d["Ax"], d["Ay"], d["Az"]],
                          kernel=kid)
        ctx.build(want_perm=False)
        outs = {p: [torch.empty(ns, dtype=torch.float64, device="cuda") for _ in range(L_OUT)]
                for p in (L.PSB_PREC_FP32C, L.PSB_PREC_FP64)}
        t = {}
        for prec in outs:
            def step(prec=prec):
                ctx.interp_grid(axis, axis, axis, cat, strategy=L.PSB_SYMMETRIC, prec=prec, out=outs[prec])
            t[prec] = timed_call(step, stream, steps, warmup)
        errs, nan_diff = [], 0
        for a, b in zip(outs[L.PSB_PREC_FP32C], outs[L.PSB_PREC_FP64]):
            fa, fb = torch.isfinite(a), torch.isfinite(b)
            nan_diff += int((fa != fb).sum())
            both = fa & fb
            errs.append(((a[both] - b[both]).abs().max() / b[both].abs().max()).item() if both.any() else 0.0)
        pairs = int(ctx.last_stats.pairs)
        gout = [torch.randn(ns, generator=gen, device="cuda", dtype=torch.float64) for _ in range(L_OUT)]
        g = {}

        def bwd():
            g.update(ctx.adjoint_grid(axis, axis, axis, cat, gout, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST,
                                      device=True))
        t_bwd = timed_call(bwd, stream, 3, 2)
        lhs = float(sum((gc * c).sum() for gc, c in zip(g["cols"], colsd)))
        rhs = float(sum((go * torch.nan_to_num(o, nan=0.0)).sum() for go, o in zip(gout, outs[L.PSB_PREC_FP64])))
        res[name] = {"fp32c_ms": t[L.PSB_PREC_FP32C], "fp64_ms": t[L.PSB_PREC_FP64],
                     "samples_per_s": ns / (t[L.PSB_PREC_FP32C] / 1e3),
                     "speedup_fp32c_vs_fp64": t[L.PSB_PREC_FP64] / t[L.PSB_PREC_FP32C],
                     "pairs": pairs, "max_fp32c_rel_err_vs_fp64": max(errs),
                     "nan_mask_differences": nan_diff,
                     "adjoint_ms": t_bwd, "grad_fwd_time_ratio": t_bwd / t[L.PSB_PREC_FP32C],
                     "adjoint_linearity_in_A_rel_residual": abs(lhs - rhs) / abs(rhs)}
        ctx.close()
    return res


def oracle_subset(d, h, rho, cols, ax, frames, bprm, nb, outs, names, nsub=100_000):
    """The FP64 CPU oracle over all particles (the float32 values in double) on
    a random subset of the grid and box samples; relative error of each GPU
    field (FP64 and FP32C) against it, over the subset's finite values."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    nthr = O.set_threads(os.cpu_count() or 1)
    f64 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    t0 = time.time()
    orc = O.Oracle(f64(d["x"]), f64(d["y"]), f64(d["z"]), f64(d["m"]), f64(h), f64(rho), [f64(c) for c in cols])
    build_s = time.time() - t0
    ng = len(ax)
    ng3, nb3 = ng ** 3, nb ** 3
    rng = np.random.default_rng(41)
    idx = np.sort(rng.choice(ng3 + len(frames) * nb3, nsub, replace=False))
    sx, sy, sz = np.empty(nsub), np.empty(nsub), np.empty(nsub)
    g = idx < ng3
    i, r = idx[g] % ng, idx[g] // ng
    sx[g], sy[g], sz[g] = ax[i], ax[r % ng], ax[r // ng]
    lo, hi = bprm[0], bprm[1]
    dq = (hi - lo) / float(nb - 1)
    for bi, fa in enumerate(frames):  # box_coordinates' arithmetic at the chosen indices
        sel = (idx >= ng3 + bi * nb3) & (idx < ng3 + (bi + 1) * nb3)
        k = idx[sel] - ng3 - bi * nb3
        xi, eta, ze = (lo + (k % nb) * dq, lo + ((k // nb) % nb) * dq, lo + (k // (nb * nb)) * dq)
        x0, rr, u, f = fa[0:3], fa[3:6], fa[6:9], fa[9:12]
        sx[sel], sy[sel], sz[sel] = (x0[c] + xi * rr[c] + eta * u[c] + ze * f[c] for c in range(3))
    t0 = time.time()
    ref = orc.interp_points(sx, sy, sz, O.Catalog(scalars=[0, 4], shepard=[0, 1], grads=[0], curls=[1, 2, 3]),
                            strategy=O.SYMMETRIC, hmode=O.H_NEAREST)
    interp_s = time.time() - t0
    ti = torch.from_numpy(idx).cuda()
    out = {"samples": nsub, "threads": nthr, "oracle_build_s": build_s, "oracle_interp_s": interp_s}
    for label in ("fp64", "fp32c"):
        e, nan_diff = {}, 0
        for k in range(8):
            a = outs[label][k][ti].cpu().numpy()
            b = np.asarray(ref[k])
            nan_diff += int(np.count_nonzero(np.isnan(a) != np.isnan(b)))
            fin = np.isfinite(b) & np.isfinite(a)
            e[names[k]] = float(np.max(np.abs(a[fin] - b[fin])) / np.max(np.abs(b[fin])))
        out[label + "_rel_err_vs_oracle"] = e
        out[label + "_nan_mask_differences"] = nan_diff
    del orc
    return out


def large_adjoint(ctx, ax, stream, steps, warmup, a_col, m):
    """Gradient of the 256^3 grid scalar's L2 norm, L = ||S||_2 with S the
    Shepard-normalised z^2, with respect to every particle input (A_b, m_b,
    r_b), against the FP32C forward of the same output.  S is linear in A and
    invariant under a common scaling of the masses, so <dL/dA, A> = <gout, S>
    and <dL/dm, m> = 0 hold at any size; both residuals are reported."""
    import torch
    from partia_b200 import _lib as L
    from partia_b200.engine import CatalogC
    cat = CatalogC(scalars=[4], shepard=[1])
    ng3 = len(ax) ** 3
    s32 = [torch.empty(ng3, dtype=torch.float64, device="cuda")]
    s64 = [torch.empty(ng3, dtype=torch.float64, device="cuda")]

    def fwd():
        ctx.interp_grid(ax, ax, ax, cat, strategy=L.PSB_SYMMETRIC, prec=L.PSB_PREC_FP32C, out=s32)

    def fwd64():
        ctx.interp_grid(ax, ax, ax, cat, strategy=L.PSB_SYMMETRIC, prec=L.PSB_PREC_FP64, out=s64)

    t_fwd = timed_call(fwd, stream, steps, warmup)
    t_fwd64 = timed_call(fwd64, stream, steps, warmup)
    S = torch.nan_to_num(s64[0], nan=0.0)
    gout = [S / torch.linalg.vector_norm(S)]
    g = {}

    def bwd():
        g.update(ctx.adjoint_grid(ax, ax, ax, cat, gout, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST,
                                  device=True))

    t_bwd = timed_call(bwd, stream, steps, warmup)
    pairs = int(ctx.last_stats.pairs)
    gA, gm = g["cols"][4], g["m"]
    lhs, rhs = float((gA * a_col).sum()), float((gout[0] * S).sum())
    return {"output": f"Shepard z^2 on the {len(ax)}^3 grid, L = ||S||_2", "gradients": "dL/dA_b, dL/dm_b, dL/dr_b (FP64)",
            "forward_fp32c_ms": t_fwd, "forward_fp64_ms": t_fwd64, "backward_ms": t_bwd,
            "grad_fwd_time_ratio": t_bwd / t_fwd, "grad_fwd_time_ratio_vs_fp64": t_bwd / t_fwd64, "pairs": pairs,
            "linearity_in_A_rel_residual": abs(lhs - rhs) / abs(rhs),
            "mass_scaling_rel_residual": abs(float((gm * m).sum())) / float((gm * m).abs().sum())}


def cpu_reference(args, d, axis, steps, warmup, threads=None):
    """Oracle port on the host cores over a bounded random sample of grid points."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    nthr = O.set_threads(threads or (os.cpu_count() or 1))
    t0 = time.time()
    orc = O.Oracle(d["x"], d["y"], d["z"], d["m"], d["h"], d["rho"], [d["rho"], d["Ax"], d["Ay"], d["Az"]])
    build_s = time.time() - t0
    rng = np.random.default_rng(12345)
    cat = O.Catalog(**CATALOG)
    # calibrate the sample size to ~args.cpu_seconds of work per step
    probe = 512
    idx = rng.integers(0, NGRID ** 3, probe)
    i, r = idx % NGRID, idx // NGRID
    s = (axis[i], axis[r % NGRID], axis[r // NGRID])
    t0 = time.time()
    orc.interp_points(*s, cat, strategy=O.SYMMETRIC, hmode=O.H_NEAREST)
    per = max((time.time() - t0) / probe, 1e-7)
    ns = int(min(max(args.cpu_seconds / per, 2000), NGRID ** 3))
    times = []
    for k in range(warmup + steps):
        idx = rng.integers(0, NGRID ** 3, ns)
        i, r = idx % NGRID, idx // NGRID
        s = (axis[i], axis[r % NGRID], axis[r // NGRID])
        t0 = time.time()
        orc.interp_points(*s, cat, strategy=O.SYMMETRIC, hmode=O.H_NEAREST)
        dt = time.time() - t0
        if k >= warmup:
            times.append(dt)
    val = ns / float(np.median(times))
    return dict(value=val, unit=UNIT, cores=nthr, kind="port", host=host_cpu(),
                sample=f"{ns} random grid points of the {NGRID}^3 grid per step (of {NGRID ** 3:,}), FP64 oracle, "
                       f"median of {steps} steps after {warmup} warm-up; LBVH build {build_s:.2f} s not timed"), times


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    d, axis = make_workload()
    steps = max(args.steps, 5)
    args.cpu_seconds = max(1.0, min(args.cpu_seconds, 150.0 / (steps + 1)))  # whole run within a few minutes
    cb, times = cpu_reference(args, d, axis, steps, 1)
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.median(times)),
            "higher_is_better": True, "scaling": "strong" if args.gpus > 1 else "weak", "vs_baseline": None,
            "dtype": "f64", "precision": "FP64 (CPU restatement of the reference's algorithm)",
            "data": "synthetic (seeded Plummer sphere, N=2e6, numpy PCG64 seed 1)",
            "config": bench_config(),
            "sampled": "each step times a random subset of the grid's samples and reports it as a rate "
                       "(see cpu_baseline.sample)",
            "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    global NGRID
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--grid", type=int, default=NGRID, help="grid points per axis (128 = the workload; smaller "
                    "values only for profiling captures)")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=4.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-lines", action="store_true", help="skip the line-integrated and adjoint legs")
    ap.add_argument("--no-large", action="store_true", help="skip the 64M-particle leg")
    ap.add_argument("--no-kernels", action="store_true", help="skip the kernel-family leg")
    ap.add_argument("--no-cudaext", action="store_true", help="skip the CUDA-extension design baseline leg")
    ap.add_argument("--lines-n", type=int, default=8_000_000,
                    help="particles of the line-integrated leg (8M = the workload; fewer only for profiling captures)")
    ap.add_argument("--lines-npix", type=int, default=1024,
                    help="beam pixels per side of the line-integrated leg (1024 = the workload)")
    ap.add_argument("--large-n", type=int, default=64_000_000,
                    help="particles of the large leg (64M = the workload; fewer only for profiling captures)")
    ap.add_argument("--large-grid", type=int, default=256,
                    help="grid points per axis of the large leg (256 = the workload; boxes take half)")
    args = ap.parse_args()
    NGRID = args.grid
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist

    from partia_b200 import _lib as L
    from partia_b200.engine import CatalogC, Context

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)

    d, axis = make_workload()
    ctx = Context(local)
    stream = torch.cuda.Stream(device=dev)
    L.load().psb_set_stream(ctx.h, stream.cuda_stream)
    cols = [d["rho"], d["Ax"], d["Ay"], d["Az"]]
    ctx.set_particles(d["x"], d["y"], d["z"], d["m"], d["h"], d["rho"], cols)
    ctx.build(want_perm=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.build(want_perm=False)  # second build: module loading excluded
    torch.cuda.synchronize()
    build_ms = (time.perf_counter() - t0) * 1e3
    cat = CatalogC(**CATALOG)

    # this rank's slab of z-planes (samples shard; particles and LBVH are
    # replicated): slabs of equal estimated pair count from a coarse digest
    # pass, which every rank computes identically
    z0, z1 = 0, NGRID
    if world > 1:
        from partia_b200.sharding import plane_pair_estimates, weighted_slabs
        plane_w = plane_pair_estimates(ctx, axis, axis, axis, stride=8)
        z0, z1 = weighted_slabs(plane_w, world)[rank]
    az = axis[z0:z1]
    ns = NGRID * NGRID * len(az)
    outs = [torch.empty(ns, dtype=torch.float64, device=dev) for _ in range(L_OUT)]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step(prec):
        ctx.interp_grid(axis, axis, az, cat, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST, prec=prec, out=outs)
        return ctx.last_stats

    def timed(prec, steps, warmup):
        for _ in range(warmup):
            step(prec)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        kern_ms, pairs = [], 0
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))  # evict L2 between steps
                ev[k][0].record(stream)
            st = step(prec)
            with torch.cuda.stream(stream):
                ev[k][1].record(stream)
            kern_ms.append(st.interp_ms)
            pairs = st.pairs
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        step_ms = [a.elapsed_time(b) for a, b in ev]
        return float(np.sum(step_ms)), step_ms, kern_ms, pairs

    with ClockSampler(local) as clk:
        tot32, steps32, kern32, pairs = timed(L.PSB_PREC_FP32C, args.steps, args.warmup)
    launches_per_step = ctx.last_stats.launches
    ctx_steps = ctx.last_stats.warp_steps
    ctx_spans, ctx_span_tests = ctx.last_stats.spans, ctx.last_stats.span_tests
    tot = torch.tensor([tot32], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tot, op=dist.ReduceOp.MAX)
    total_samples = NGRID ** 3 if world > 1 else ns
    value = total_samples * args.steps / (tot.item() / 1e3)

    # FP64 path and accuracy of FP32C against it
    fp64 = None
    errs = None
    if not args.no_fp64:
        tot64, _, kern64, _ = timed(L.PSB_PREC_FP64, max(2, args.steps // 2), 1)
        v64 = ns * max(2, args.steps // 2) / (tot64 / 1e3)
        step(L.PSB_PREC_FP32C)
        o32 = [o.clone() for o in outs]
        step(L.PSB_PREC_FP64)
        errs = {}
        names = ["rho", "grad_rho_x", "grad_rho_y", "grad_rho_z", "div_A", "curl_A_x", "curl_A_y", "curl_A_z"]
        for k in range(L_OUT):
            a, b = o32[k].double(), outs[k].double()
            fin = torch.isfinite(b)
            scale = b[fin].abs().max().item()
            errs[names[k]] = (a[fin] - b[fin]).abs().max().item() / scale if scale > 0 else 0.0
        fp64 = {"value": v64, "unit": UNIT, "kernel_ms": float(np.median(kern64)),
                "ms": tot64 / max(2, args.steps // 2),
                "speedup_fp32c_vs_fp64": value / v64 if world == 1 else None}

    # e2e through the C ABI with host buffers (pinned), copies inside the timed region
    X, Y, Z = np.meshgrid(axis, axis, az, indexing="ij")
    hx = torch.from_numpy(X.ravel(order="F").copy()).pin_memory()
    hy = torch.from_numpy(Y.ravel(order="F").copy()).pin_memory()
    hz = torch.from_numpy(Z.ravel(order="F").copy()).pin_memory()
    hout = [torch.empty(ns, dtype=torch.float64).pin_memory() for _ in range(L_OUT)]
    hxn, hyn, hzn = hx.numpy(), hy.numpy(), hz.numpy()
    houtn = [o.numpy() for o in hout]

    def e2e_step():
        ctx.interp_points(hxn, hyn, hzn, cat, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST,
                          prec=L.PSB_PREC_FP32C, out=houtn)
        return ctx.last_stats

    def e2e_timed(fn):
        """Host-clock seconds of each call (after a synchronise), plus the
        library's own event span of the call."""
        for _ in range(max(1, args.warmup)):
            fn()
        torch.cuda.synchronize()
        host_s, lib_ms = [], []
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st = fn()
            host_s.append(time.perf_counter() - t0)
            lib_ms.append(st.total_ms)
        tot = torch.tensor([float(np.sum(host_s))], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(tot, op=dist.ReduceOp.MAX)
        return total_samples * args.steps / tot.item(), float(np.median(host_s)) * 1e3, float(np.median(lib_ms))

    e2e_val, e2e_host_ms, e2e_lib_ms = e2e_timed(e2e_step)
    # the same call with pageable numpy buffers (what a Julia caller passes)
    pxn, pyn, pzn = (np.array(a, copy=True) for a in (hxn, hyn, hzn))
    poutn = [np.empty(ns, dtype=np.float64) for _ in range(L_OUT)]

    def e2e_pageable():
        ctx.interp_points(pxn, pyn, pzn, cat, strategy=L.PSB_SYMMETRIC, hmode=L.PSB_H_NEAREST,
                          prec=L.PSB_PREC_FP32C, out=poutn)
        return ctx.last_stats

    e2e_pg_val, e2e_pg_host_ms, e2e_pg_lib_ms = e2e_timed(e2e_pageable)
    for a, b in zip(houtn, poutn):
        assert np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(a[~np.isnan(a)], b[~np.isnan(b)]), \
            "pageable and pinned host calls disagree"

    # roofline of the point kernel (algorithmic bytes per launch)
    hbm, peak_kind = peaks()
    kern_ms = float(np.median(kern32))
    # grid coordinates are generated on the device (S_in = 0); outputs are
    # written in the input element type (f64, 8 B); the FP32C pair record is
    # (x, y, z, h, m, rho + the catalog's columns) in float
    b_alg = ns * (0 + L_OUT * 8) + pairs * (6 + NCOL_USED) * 4
    achieved = b_alg / (kern_ms / 1e3) / 1e9
    tr = ncu_traffic()

    cudaext = None
    if world == 1 and not args.no_cudaext:
        ours = {"fp32c_ms": tot32 / args.steps, "fp64_ms": (fp64 or {}).get("ms", float("nan")),
                "e2e_ms": e2e_host_ms}
        cudaext = cudaext_leg(ctx, d, axis, 3, 1, ours)

    extra = None
    if world == 1 and not args.no_lines:
        extra = lines_and_adjoint(max(3, args.steps // 4), 2, args.lines_n, args.lines_npix)
    kern = None
    if world == 1 and not args.no_kernels:
        kern = kernel_families(d, axis, max(3, args.steps // 4), 2)
    large = None
    if world == 1 and not args.no_large:
        large = large_leg(3, 1, oracle_check=not args.no_cpu, n=args.large_n, ng=args.large_grid)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu, _ = cpu_reference(args, d, axis, 5, 1)
        except Exception as e:  # the oracle build needs g++
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "port", "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot.item() / args.steps, "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "f32c",
            "precision": "FP32C (float pair sums with compensated accumulation; double inclusion test and "
                         "finalisation)",
            "data": "synthetic (seeded Plummer sphere, N=2e6, numpy PCG64 seed 1)",
            "config": bench_config(),
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": 3 * 8 * ns,
                    "d2h_bytes_per_step": L_OUT * 8 * ns,
                    "timing": "host clock (time.perf_counter) around each psb_interp_points call, after a "
                              "synchronise; pinned host buffers",
                    "host_ms_per_call": e2e_host_ms, "library_event_ms_per_call": e2e_lib_ms,
                    "pageable": {"value": e2e_pg_val, "unit": UNIT, "host_ms_per_call": e2e_pg_host_ms,
                                 "library_event_ms_per_call": e2e_pg_lib_ms}},
            "gpu_launches": int(args.steps * launches_per_step),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_kind": peak_kind,
                         "traffic": (tr or {}).get("bytes_per_launch") if tr else None,
                         "kernel": "k_collect + k_bodies <double,FP32C,SYMMETRIC,4> (pair lists, pair sums)", "kernel_ms": kern_ms,
                         "pairs_per_launch": int(pairs), "alg_bytes_per_launch": int(b_alg),
                         "warp_steps_per_launch": int(ctx_steps), "span_visits_per_launch": int(ctx_spans),
                         "samples_per_span_visit": ctx_span_tests / max(ctx_spans, 1)},
            "fp64": fp64, "fp32c_rel_err_vs_fp64": errs,
            "grad_fwd_time_ratio": extra["adjoint"]["grad_fwd_time_ratio"] if extra else None,
            "cudaext_design": cudaext,
            "lines": extra["lines"] if extra else None, "adjoint": extra["adjoint"] if extra else None,
            "large": large,
            "kernel_families": kern,
            "build_ms": build_ms,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    ctx.close()


if __name__ == "__main__":
    main()
