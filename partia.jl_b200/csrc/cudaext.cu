// cudaext.cu -- the reference's CUDA-extension design, kept as the GPU
// baseline this library is measured against (psb_baseline_cudaext_points).
//
// Partia's CUDA extension (ext/CUDAExt/KernelInterpolation/grid_interpolation/
// drivers/PointSamples_driver.jl:12-27, kernels/PointSamples_kernel.jl:1-68)
// builds the LBVH on the CPU, copies the whole input and the whole tree to
// the device on every call (to_CuVector), launches one thread per sample in
// blocks of 256, and copies the outputs back.  Each thread runs
// LBVH_find_nearest_h and then the general interpolation kernel, both as its
// own stackless DFS over the double node boxes, with no shared memory and no
// cooperation between threads.  This file restates that structure in CUDA C++
// with the library's FP64 arithmetic, so that the warp-tile design can be
// compared with it on the same GPU: the host supplies the tree (as the CPU
// build would) and everything crosses the host link in every call.  The
// device buffers are kept between calls, as CUDA.jl's memory pool keeps its
// allocations.
#include <cstring>
#include <vector>

#include "launch.hpp"
#include "psb_host.hpp"

namespace psb {
namespace {

template <int ST, int KC>
__global__ void __launch_bounds__(256) k_cudaext_points(const Args<double> A) {
    const TreeView<double>& tv = A.tv;
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= A.src.ns) return;
    const double p[3] = {A.src.a[0][k], A.src.a[1][k], A.src.a[2][k]};
    const int64_t n = tv.n;
    const int64_t bound = 4 * n + 8;
    bool ok = true;
    // one thread's stackless DFS (LinearBVHTraversalMacros.jl:26-108): prune
    // an internal node when reject(ni), visit leaves in DFS order
    auto walk = [&](auto reject, auto leaf) {
        if (tv.root == 0) {
            for (int64_t li = 0; li < n; ++li) leaf(li);
            return;
        }
        int32_t node = tv.root;
        int64_t steps = 0;
        while (node != 0) {
            if (++steps > bound || node < 0 || (int64_t)node > 2 * n - 1) {
                ok = false;
                return;
            }
            if (node >= n) {
                leaf((int64_t)node - n);
                node = tv.escape[node - 1];
                continue;
            }
            const int ni = node - 1;
            node = reject(ni) ? tv.escape[ni] : tv.left[ni];
        }
    };
    const double K = tv.Kd;
    double ha = 0.0;
    if (ST != ST_SCATTER) {  // LBVH_find_nearest_h (LinearBVHQueries.jl:118-140)
        double best = INFINITY;
        int64_t bi = -1;
        walk([&](int ni) { return ex_d2_pbox<double>(p, tv, ni) > best; },
             [&](int64_t li) {
                 const double d2 = ex_d2_pp<double>(p, tv.x[li], tv.y[li], tv.z[li]);
                 if (d2 < best) { best = d2; bi = li; }
             });
        ha = bi >= 0 ? tv.h[bi] : (double)NAN;
    }
    const double ra = X<double>::mul(K, ha), ra2 = X<double>::mul(ra, ra);
    const double sig = tv.sig;
    const bool m4 = tv.kern == KERN_M4;
    const int kc = A.rec.kc;
    const bool need_dg = A.rec.need_dg != 0;
    double ia = 0.0, sa3 = 0.0, sa4 = 0.0;
    if (ST != ST_SCATTER) {
        ia = 1.0 / ha;
        sa3 = sig * ia * ia * ia;
        sa4 = sa3 * ia;
    }
    PlainD S1, G[3], Sw[KC], Sg[KC][3], Dm, Dg[3];
    double a0[KC];
    S1.zero(); Dm.zero();
    for (int d = 0; d < 3; ++d) { G[d].zero(); Dg[d].zero(); }
    for (int c = 0; c < KC; ++c) {
        Sw[c].zero();
        a0[c] = 0.0;
        for (int d = 0; d < 3; ++d) Sg[c][d].zero();
    }
    unsigned long long npairs = 0;
    auto fdf = [&](double q, double& f, double& df) {
        if (m4) m4_fdf<double>(q, f, df);
        else kern_fdf<double>(tv.kern, q, f, df);
    };
    walk([&](int ni) {
             const double d2n = ex_d2_pbox<double>(p, tv, ni);
             return d2n > ex_r2<ST, double>(ra2, tv.nscale[ni], K);
         },
         [&](int64_t li) {
             const double hb = tv.h[li];
             const double d2 = ex_d2_pp<double>(p, tv.x[li], tv.y[li], tv.z[li]);
             if (!(d2 <= ex_r2<ST, double>(ra2, hb, K))) return;
             ++npairs;
             const double dx = p[0] - tv.x[li], dy = p[1] - tv.y[li], dz = p[2] - tv.z[li];
             const double r = sqrt(d2);
             const double invr = d2 > 0.0 ? 1.0 / r : 0.0;
             double W = 0.0, cg = 0.0, f, df;
             if (ST != ST_SCATTER) {
                 fdf(r * ia, f, df);
                 W = sa3 * f;
                 cg = sa4 * df * invr;
             }
             if (ST != ST_GATHER) {
                 const double ib = 1.0 / hb, sb3 = sig * ib * ib * ib;
                 fdf(r * ib, f, df);
                 const double Wb = sb3 * f, cb = sb3 * ib * df * invr;
                 if (ST == ST_SCATTER) { W = Wb; cg = cb; }
                 else { W = 0.5 * (W + Wb); cg = 0.5 * (cg + cb); }
             }
             const double mb = tv.m[li], mr = mb / tv.rho[li];
             const double w = mr * W, gc = mr * cg;
             const double gx = gc * dx, gy = gc * dy, gz = gc * dz;
             S1.add(w);
             G[0].add(gx); G[1].add(gy); G[2].add(gz);
             for (int c = 0; c < KC; ++c) {
                 if (c < kc) {
                     const double a = A.colT[c][li];
                     Sw[c].add(a * w);
                     Sg[c][0].add(a * gx); Sg[c][1].add(a * gy); Sg[c][2].add(a * gz);
                 }
             }
             if (need_dg) {
                 Dm.add(mb * W);
                 const double mc = mb * cg;
                 Dg[0].add(mc * dx); Dg[1].add(mc * dy); Dg[2].add(mc * dz);
             }
         });
    write_interp_outputs<double, PlainD, double, KC>(A, k, S1, G, Sw, Sg, Dm, Dg, a0);
    if (A.stats) atomicAdd(&A.stats[0], npairs);
    if (!ok) atomicOr(A.err, PSB_DERR_TRAVERSAL);
}

template <int ST>
void launch_st(const Args<double>& A, int kc, unsigned g, cudaStream_t s) {
    if (kc <= 1) k_cudaext_points<ST, 1><<<g, 256, 0, s>>>(A);
    else if (kc <= 2) k_cudaext_points<ST, 2><<<g, 256, 0, s>>>(A);
    else if (kc <= 4) k_cudaext_points<ST, 4><<<g, 256, 0, s>>>(A);
    else k_cudaext_points<ST, 8><<<g, 256, 0, s>>>(A);
}

inline size_t al256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

int make_recipe(psb_ctx* c, const psb_catalog* cat, bool line, Recipe& rec, std::vector<int>& colu);

}  // namespace psb

using namespace psb;

extern "C" __attribute__((visibility("default"))) int psb_baseline_cudaext_points(
    psb_ctx* c, int64_t n, const double* x, const double* y, const double* z, const double* m, const double* h,
    const double* rho, int32_t ncol, const double* const* cols, psb_kernel kernel, int32_t root, const int32_t* left,
    const int32_t* escape, const double* node_min, const double* node_max, const double* node_scale, int64_t ns,
    const double* sx, const double* sy, const double* sz, psb_strategy strategy, const psb_catalog* cat,
    double* const* out, psb_stats* stats) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    DeviceGuard dg(c->device);
    if (n < 1) return fail(c, PSB_EINVAL, "particle count must be positive");
    if (ns < 0) return fail(c, PSB_EINVAL, "sample count must be non-negative");
    if (ncol < 0 || (ncol > 0 && !cols)) return fail(c, PSB_EINVAL, "bad column arrays");
    if ((int)kernel < 0 || (int)kernel >= KERN_COUNT) return fail(c, PSB_EINVAL, "unknown kernel");
    if (strategy < 0 || strategy > 2) return fail(c, PSB_EINVAL, "unknown interpolation strategy");
    if (!x || !y || !z || !m || !h || !rho || !left || !escape) return fail(c, PSB_EINVAL, "NULL input array");
    if (n >= 2 && (!node_min || !node_max || !node_scale)) return fail(c, PSB_EINVAL, "NULL node array");
    if (root != (n >= 2 ? 1 : 0)) return fail(c, PSB_EINVAL, "root must be 1 (n >= 2) or 0");
    if (ns > 0 && (!sx || !sy || !sz)) return fail(c, PSB_EINVAL, "sample arrays must not be NULL");
    Args<double> A;
    memset((void*)&A, 0, sizeof(A));
    std::vector<int> colu;
    psb_ctx tmp;  // the recipe checks column slots against ncol
    tmp.ncol = ncol;
    int rc = make_recipe(&tmp, cat, false, A.rec, colu);
    if (rc) return fail(c, rc, tmp.err);
    const int L = A.rec.L;
    if (ns > 0 && L > 0 && !out) return fail(c, PSB_EINVAL, "output pointer array must not be NULL");
    for (int k = 0; ns > 0 && k < L; ++k)
        if (!out[k]) return fail(c, PSB_EINVAL, "an output pointer is NULL");
    cudaStream_t s = c->stream;
    const int64_t nint = n - 1, tot = 2 * n - 1;
    // one input buffer (particles, used columns, tree, samples) and one output buffer
    const size_t b_part = al256(8 * (size_t)n), b_id = al256(4 * (size_t)tot), b_node = al256(8 * (size_t)(nint > 0 ? nint : 1));
    const size_t b_smp = al256(8 * (size_t)(ns > 0 ? ns : 1));
    const size_t in_bytes = b_part * (6 + colu.size()) + 2 * b_id + 7 * b_node + 3 * b_smp;
    char* din = (char*)scratch(c, 90, in_bytes);
    char* dout = (char*)scratch(c, 91, b_smp * (L > 0 ? L : 1));
    unsigned long long* dstats = (unsigned long long*)scratch(c, 92, 8 * sizeof(unsigned long long));
    if (!din || !dout || !dstats) return fail(c, PSB_ENOMEM, "device buffers of the baseline");
    char* q = din;
    cudaError_t ce = cudaSuccess;
    auto put = [&](const void* src, size_t bytes, size_t room) -> void* {
        void* d = q;
        if (bytes && ce == cudaSuccess) ce = cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, s);
        q += room;
        return d;
    };
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[0], s), "event");
    TreeView<double>& tv = A.tv;
    tv.n = n;
    tv.root = root;
    tv.x = (const double*)put(x, 8 * n, b_part);
    tv.y = (const double*)put(y, 8 * n, b_part);
    tv.z = (const double*)put(z, 8 * n, b_part);
    tv.m = (const double*)put(m, 8 * n, b_part);
    tv.h = (const double*)put(h, 8 * n, b_part);
    tv.rho = (const double*)put(rho, 8 * n, b_part);
    for (size_t k = 0; k < colu.size(); ++k) A.colT[k] = (const double*)put(cols[colu[k]], 8 * n, b_part);
    tv.left = (const int32_t*)put(left, 4 * tot, b_id);
    tv.escape = (const int32_t*)put(escape, 4 * tot, b_id);
    for (int d = 0; d < 3; ++d) tv.nmin[d] = (const double*)put(node_min ? node_min + d * nint : nullptr, 8 * nint, b_node);
    for (int d = 0; d < 3; ++d) tv.nmax[d] = (const double*)put(node_max ? node_max + d * nint : nullptr, 8 * nint, b_node);
    tv.nscale = (const double*)put(node_scale, 8 * nint, b_node);
    A.src.kind = SRC_ARRAYS;
    A.src.ns = ns;
    A.src.a[0] = (const double*)put(sx, 8 * ns, b_smp);
    A.src.a[1] = (const double*)put(sy, 8 * ns, b_smp);
    A.src.a[2] = (const double*)put(sz, 8 * ns, b_smp);
    PSB_CUDA_TRY(c, ce, "input H2D");
    tv.kern = (int)kernel;
    tv.Kd = kern_support((int)kernel);
    tv.Kf = (float)tv.Kd;
    tv.sig = kern_norm3((int)kernel);
    for (int k = 0; k < L; ++k) A.out[k] = (double*)(dout + b_smp * k);
    A.err = c->d_err;
    A.stats = dstats;
    PSB_CUDA_TRY(c, cudaMemsetAsync(dstats, 0, 8 * sizeof(unsigned long long), s), "memset");
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[1], s), "event");
    if (ns > 0) {
        const unsigned g = (unsigned)((ns + 255) / 256);
        const int kc = A.rec.kc;
        if (strategy == PSB_GATHER) launch_st<ST_GATHER>(A, kc, g, s);
        else if (strategy == PSB_SCATTER) launch_st<ST_SCATTER>(A, kc, g, s);
        else launch_st<ST_SYMMETRIC>(A, kc, g, s);
        PSB_CUDA_TRY(c, cudaGetLastError(), "baseline kernel launch");
    }
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[2], s), "event");
    for (int k = 0; ns > 0 && k < L; ++k)
        PSB_CUDA_TRY(c, cudaMemcpyAsync(out[k], A.out[k], 8 * ns, cudaMemcpyDeviceToHost, s), "output D2H");
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[3], s), "event");
    unsigned long long hst[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    unsigned herr = 0;
    PSB_CUDA_TRY(c, cudaMemcpyAsync(hst, dstats, sizeof(hst), cudaMemcpyDeviceToHost, s), "stats D2H");
    PSB_CUDA_TRY(c, cudaMemcpyAsync(&herr, c->d_err, sizeof(herr), cudaMemcpyDeviceToHost, s), "error D2H");
    PSB_CUDA_TRY(c, cudaStreamSynchronize(s), "synchronize");
    if (herr) {
        cudaMemsetAsync(c->d_err, 0, sizeof(unsigned), s);
        cudaStreamSynchronize(s);
        return device_error(c, herr);
    }
    if (stats) {
        float ms = 0.f;
        memset(stats, 0, sizeof(*stats));
        cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
        stats->h2d_ms = ms;
        cudaEventElapsedTime(&ms, c->ev[1], c->ev[2]);
        stats->interp_ms = ms;
        cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]);
        stats->d2h_ms = ms;
        cudaEventElapsedTime(&ms, c->ev[0], c->ev[3]);
        stats->total_ms = ms;
        stats->pairs = (int64_t)hst[0];
        stats->launches = ns > 0 ? 1 : 0;
    }
    return PSB_OK;
}
