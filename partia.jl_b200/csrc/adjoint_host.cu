// adjoint_host.cu -- host drivers of the adjoint entry points: stage the
// samples and the output cotangents, obtain the sum cotangents (directly, or
// from the FP64 forward pass in its sum-cotangent mode), build the LBVH over
// the samples (points) and run the particle-centric kernels, then return dL/dm, dL/dA_c and dL/dx per particle
// in the order the particles were given to psb_set_particles.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "k_adjoint.cuh"
#include "psb_ctx.hpp"
#include "psb_host.hpp"

extern "C" int psb_create(psb_ctx** out, int device);
extern "C" int psb_set_stream(psb_ctx* c, void* stream);
extern "C" int psb_set_particles(psb_ctx* c, int64_t n, psb_dtype dt, const void* x, const void* y, const void* z,
                                 const void* m, const void* h, const void* rho, int32_t ncol, const void* const* cols,
                                 psb_kernel kernel, uint32_t flags);

namespace psb {

int make_recipe(psb_ctx* c, const psb_catalog* cat, bool line, Recipe& rec, std::vector<int>& colu);

// Sort keys of the particle tiles for the adjoint's walk, heaviest first:
// a tile's walk and pairs grow with its particles' supports, and the tiles of
// large-h particles in the outskirts hold many times the mean tile's pairs.
// Cost: the sum of h^3 over the tile's particles whose support reaches the
// samples' box (box = min x, y, z, max x, y, z; K the support).  The key is
// the cost's power of two only, and the radix sort is stable: tiles of like
// cost keep their Morton order, and with it the walk's locality in the
// sample tree.
__global__ void k_adj_tile_keys(const double* x, const double* y, const double* z, const double* h, int64_t n,
                                int64_t ntiles, double K, double b0, double b1, double b2, double b3, double b4,
                                double b5, uint64_t* keys, uint32_t* vals) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    double c = 0.0;
    for (int64_t b = t * 32; b < t * 32 + 32 && b < n; ++b) {
        const double r = K * h[b];
        const double dx = fmax(fmax(b0 - x[b], x[b] - b3), 0.0), dy = fmax(fmax(b1 - y[b], y[b] - b4), 0.0),
                     dz = fmax(fmax(b2 - z[b], z[b] - b5), 0.0);
        if (dx <= r && dy <= r && dz <= r) c += h[b] * h[b] * h[b];
    }
    const int e = c > 0.0 ? ilogb(c) + 1100 : 0;  // 0 .. ~2100, larger for more cost
    keys[t] = (uint64_t)(4095 - e);
    vals[t] = (uint32_t)t;
}

// pass: 0 = k_adj_points (whole tiles, or the listed ones), 1 = its pair-list
// form (COL), 2 = k_adj_bodies (grid over list blocks), 3 = k_adj_combine
template <int KC, bool SCAL, int KF>
static void launch_adj_points_ks(const AdjArgs& a, int st, int pass, unsigned g, cudaStream_t s) {
    if (pass == 1) {
        if (st == ST_GATHER) k_adj_points<ST_GATHER, 1, true, KF, true><<<g, 128, 0, s>>>(a);
        else if (st == ST_SCATTER) k_adj_points<ST_SCATTER, 1, true, KF, true><<<g, 128, 0, s>>>(a);
        else k_adj_points<ST_SYMMETRIC, 1, true, KF, true><<<g, 128, 0, s>>>(a);
    } else if (pass == 2) {
        if (st == ST_GATHER) k_adj_bodies<ST_GATHER, KC, SCAL, KF><<<g, 128, 0, s>>>(a);
        else if (st == ST_SCATTER) k_adj_bodies<ST_SCATTER, KC, SCAL, KF><<<g, 128, 0, s>>>(a);
        else k_adj_bodies<ST_SYMMETRIC, KC, SCAL, KF><<<g, 128, 0, s>>>(a);
    } else if (pass == 3) {
        k_adj_combine<KC><<<g, 128, 0, s>>>(a);
    } else {
        if (st == ST_GATHER) k_adj_points<ST_GATHER, KC, SCAL, KF><<<g, 128, 0, s>>>(a);
        else if (st == ST_SCATTER) k_adj_points<ST_SCATTER, KC, SCAL, KF><<<g, 128, 0, s>>>(a);
        else k_adj_points<ST_SYMMETRIC, KC, SCAL, KF><<<g, 128, 0, s>>>(a);
    }
}
// kf: 0 = the M4 code, 1 = the other kernel families
template <int KC>
static void launch_adj_points_k(const AdjArgs& a, int st, bool scal, int kf, int pass, unsigned g, cudaStream_t s) {
    if (kf == 0) {
        if (scal) launch_adj_points_ks<KC, true, 0>(a, st, pass, g, s);
        else launch_adj_points_ks<KC, false, 0>(a, st, pass, g, s);
    } else {
        if (scal) launch_adj_points_ks<KC, true, 1>(a, st, pass, g, s);
        else launch_adj_points_ks<KC, false, 1>(a, st, pass, g, s);
    }
}
static void launch_adj_rows(int kcl, bool scal, const double* lam, int64_t ns, int kc, const TreeView<double>& sv,
                            double* rec, cudaStream_t s) {
    const unsigned g = (unsigned)((ns + 255) / 256);
    if (scal) {
        if (kcl == 1) k_adj_rows<1, true><<<g, 256, 0, s>>>(lam, ns, kc, sv, rec);
        else if (kcl == 2) k_adj_rows<2, true><<<g, 256, 0, s>>>(lam, ns, kc, sv, rec);
        else if (kcl == 4) k_adj_rows<4, true><<<g, 256, 0, s>>>(lam, ns, kc, sv, rec);
        else k_adj_rows<8, true><<<g, 256, 0, s>>>(lam, ns, kc, sv, rec);
    } else {
        if (kcl == 1) k_adj_rows<1, false><<<g, 256, 0, s>>>(lam, ns, kc, sv, rec);
        else if (kcl == 2) k_adj_rows<2, false><<<g, 256, 0, s>>>(lam, ns, kc, sv, rec);
        else if (kcl == 4) k_adj_rows<4, false><<<g, 256, 0, s>>>(lam, ns, kc, sv, rec);
        else k_adj_rows<8, false><<<g, 256, 0, s>>>(lam, ns, kc, sv, rec);
    }
}
static void launch_adj_points(const AdjArgs& a, int kcl, int st, bool scal, int kf, int pass, unsigned g,
                              cudaStream_t s) {
    if (kcl == 1) launch_adj_points_k<1>(a, st, scal, kf, pass, g, s);
    else if (kcl == 2) launch_adj_points_k<2>(a, st, scal, kf, pass, g, s);
    else if (kcl == 4) launch_adj_points_k<4>(a, st, scal, kf, pass, g, s);
    else launch_adj_points_k<8>(a, st, scal, kf, pass, g, s);
}
template <int KC>
static void launch_adj_beam_k(const AdjArgs& a, int st, unsigned g, cudaStream_t s) {
    if (st == ST_GATHER) k_adj_beam<ST_GATHER, KC><<<g, 128, 0, s>>>(a);
    else if (st == ST_SCATTER) k_adj_beam<ST_SCATTER, KC><<<g, 128, 0, s>>>(a);
    else k_adj_beam<ST_SYMMETRIC, KC><<<g, 128, 0, s>>>(a);
}

// Sum cotangents that do not depend on the forward sums: a catalog of
// scalars without Shepard normalisation (lambda_Sw_c = the sum of the output
// cotangents of column c, every other cotangent zero).
__global__ void k_direct_cotangents(const Recipe rec, const double* const* gout, int64_t ns, int nq, bool line,
                                    double* lam) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ns) return;
    for (int q = 0; q < nq; ++q) lam[q * ns + k] = 0.0;
    const int base = line ? 1 : 8;  // Sw_c sits at q = 1 + c (lines) or 8 + c (points)
    for (int o = 0; o < rec.L; ++o) lam[(base + rec.a0[o]) * ns + k] += gout[o][k];
}

// h_a of every sample from hs (per sample, or one constant)
__global__ void k_fill_ha(const double* hs, bool per_sample, int64_t ns, double* ha) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < ns) ha[k] = per_sample ? hs[k] : hs[0];
}

// clears the adjoint hook of the context on every exit path
struct AdjHook {
    psb_ctx* c;
    ~AdjHook() {
        c->adj_gout = nullptr;
        c->adj_lam = nullptr;
        c->adj_lam_stride = 0;
        c->adj_ha = nullptr;
    }
};

int run_adjoint(psb_ctx* c, const SampleReq& rq0, int hmode, const void* hs, int st, const psb_catalog* cat,
                const void* const* gout, double* gm, double* const* gcols, double* gx, double* gy, double* gz,
                uint32_t flags, psb_stats* stats) {
    if (!c->built) return fail(c, PSB_ESTATE, "psb_build_lbvh must run before the adjoint");
    if (c->dt != PSB_F64) return fail(c, PSB_EUNSUPPORTED, "the adjoint needs double particle data");
    if (st < 0 || st > 2) return fail(c, PSB_EINVAL, "unknown interpolation strategy");
    if (hmode < 0 || hmode > 2) return fail(c, PSB_EINVAL, "unknown smoothing-length mode");
    const bool line = rq0.line;
    if (line && st != ST_SCATTER && hmode == PSB_H_NEAREST)
        return fail(c, PSB_EINVAL, "line samples need hs for itpGather and itpSymmetric");
    const bool dev = (flags & PSB_FLAG_DEVICE_PTRS) != 0;
    cudaStream_t s = c->stream;
    const int64_t n = c->n;
    int64_t ns = rq0.ns;
    if (rq0.kind == SRC_GRID) ns = rq0.nx * rq0.ny * rq0.nz;
    if (rq0.kind == SRC_BEAM) ns = rq0.nx * rq0.ny;
    if (ns < 0) return fail(c, PSB_EINVAL, "sample count must be non-negative");

    Recipe rec;
    std::vector<int> colu;
    int rc = make_recipe(c, cat, line, rec, colu);
    if (rc) return rc;
    const int L = rec.L, kc = rec.kc;
    if (L > 0 && ns > 0 && !gout) return fail(c, PSB_EINVAL, "gout must not be NULL");
    for (int k = 0; ns > 0 && k < L; ++k)
        if (!gout[k]) return fail(c, PSB_EINVAL, "a gout array is NULL");
    if (!gm || !gx || !gy || !gz) return fail(c, PSB_EINVAL, "gradient outputs must not be NULL");
    const bool need_h = st != ST_SCATTER && hmode != PSB_H_NEAREST;
    if (need_h && !hs) return fail(c, PSB_EINVAL, "hs must not be NULL for this strategy and hmode");
    if (dev) {  // pointers used in device copies, memsets and kernels
        int rc = PSB_OK;
        for (int q = 0; !rc && ns > 0 && rq0.kind == SRC_ARRAYS && q < (line ? 6 : 3); ++q)
            rc = check_device_ptr(c, rq0.a[q], "a sample coordinate array");
        if (!rc && ns > 0 && need_h) rc = check_device_ptr(c, hs, "hs");
        for (int k = 0; !rc && ns > 0 && k < L; ++k) rc = check_device_ptr(c, gout[k], "a gout array");
        for (const double* p : {gm, gx, gy, gz})
            if (!rc && n > 0) rc = check_device_ptr(c, p, "a gradient output");
        for (int k = 0; !rc && n > 0 && gcols && k < c->ncol; ++k) rc = check_device_ptr(c, gcols[k], "a column gradient");
        if (rc) return rc;
    }
    if (rq0.kind == SRC_BEAM) {
        if (rq0.nx < 2 || rq0.ny < 2) return fail(c, PSB_EUNSUPPORTED, "the beam adjoint needs nx, ny >= 2");
        const double* f = (const double*)rq0.frame;
        const double* pr = (const double*)rq0.params;
        if (pr[1] == pr[0] || pr[3] == pr[2]) return fail(c, PSB_EINVAL, "degenerate beam extent");
        auto dot = [&](int a, int b) { return f[a] * f[b] + f[a + 1] * f[b + 1] + f[a + 2] * f[b + 2]; };
        if (std::fabs(dot(3, 3) - 1) > 1e-9 || std::fabs(dot(6, 6) - 1) > 1e-9 || std::fabs(dot(9, 9) - 1) > 1e-9 ||
            std::fabs(dot(3, 6)) > 1e-9 || std::fabs(dot(3, 9)) > 1e-9 || std::fabs(dot(6, 9)) > 1e-9)
            return fail(c, PSB_EUNSUPPORTED, "the beam adjoint needs an orthonormal frame");
    }
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[0], s), "event");
    int launches = 0;

    // ---- gradient outputs (device) ----
    const int ng = 4 + kc;
    double* gdev = (double*)scratch(c, 27, sizeof(double) * (size_t)ng * (n > 0 ? n : 1));
    if (!gdev) return fail(c, PSB_ENOMEM, "scratch allocation failed (gradients)");
    double* g_m = dev ? gm : gdev;
    double* g_x = dev ? gx : gdev + n;
    double* g_y = dev ? gy : gdev + 2 * n;
    double* g_z = dev ? gz : gdev + 3 * n;
    double* g_c[MAX_KC] = {};
    for (int q = 0; q < kc; ++q) g_c[q] = dev ? (gcols ? gcols[colu[q]] : nullptr) : gdev + (4 + q) * n;
    PSB_CUDA_TRY(c, cudaMemsetAsync(gdev, 0, sizeof(double) * (size_t)ng * (n > 0 ? n : 1), s), "memset");
    if (dev) {
        for (double* p : {gm, gx, gy, gz}) PSB_CUDA_TRY(c, cudaMemsetAsync(p, 0, sizeof(double) * n, s), "memset");
        for (int k = 0; gcols && k < c->ncol; ++k)
            if (gcols[k]) PSB_CUDA_TRY(c, cudaMemsetAsync(gcols[k], 0, sizeof(double) * n, s), "memset");
    }

    if (ns > 0 && n > 0) {
        // ---- samples, hs and gout on the device ----
        SampleReq rq = rq0;
        double* xyz = nullptr;
        if (!line) {
            xyz = (double*)scratch(c, 25, sizeof(double) * 3 * (size_t)ns);
            if (!xyz) return fail(c, PSB_ENOMEM, "scratch allocation failed (samples)");
            if (rq0.kind == SRC_ARRAYS) {
                const cudaMemcpyKind kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
                for (int q = 0; q < 3; ++q)
                    PSB_CUDA_TRY(c, cudaMemcpyAsync(xyz + q * ns, rq0.a[q], sizeof(double) * ns, kind, s), "sample copy");
            } else {  // grid axes (host) -> coordinates of every sample
                double* ax = (double*)scratch(c, 29, sizeof(double) * (rq0.nx + rq0.ny + rq0.nz));
                if (!ax) return fail(c, PSB_ENOMEM, "scratch allocation failed (axes)");
                PSB_CUDA_TRY(c, cudaMemcpyAsync(ax, rq0.ax, sizeof(double) * rq0.nx, cudaMemcpyHostToDevice, s), "axis H2D");
                PSB_CUDA_TRY(c, cudaMemcpyAsync(ax + rq0.nx, rq0.ay, sizeof(double) * rq0.ny, cudaMemcpyHostToDevice, s), "axis H2D");
                PSB_CUDA_TRY(c, cudaMemcpyAsync(ax + rq0.nx + rq0.ny, rq0.az, sizeof(double) * rq0.nz, cudaMemcpyHostToDevice, s), "axis H2D");
                SampleSrc<double> G;
                memset((void*)&G, 0, sizeof(G));
                G.kind = SRC_GRID;
                G.ax = ax; G.ay = ax + rq0.nx; G.az = ax + rq0.nx + rq0.ny;
                G.nx = rq0.nx; G.ny = rq0.ny; G.nz = rq0.nz;
                k_sample_xyz<<<(unsigned)((ns + 255) / 256), 256, 0, s>>>(G, ns, xyz, xyz + ns, xyz + 2 * ns);
                PSB_CUDA_TRY(c, cudaGetLastError(), "sample coordinate kernel");
                ++launches;
            }
            rq = SampleReq();
            rq.kind = SRC_ARRAYS;
            rq.ns = ns;
            rq.a[0] = xyz; rq.a[1] = xyz + ns; rq.a[2] = xyz + 2 * ns;
        }
        const int64_t nh = need_h ? (hmode == PSB_H_PER_SAMPLE ? ns : 1) : 0;
        double* hsd = nullptr;
        std::vector<double> hs_host;
        if (need_h) {
            hsd = (double*)scratch(c, 28, sizeof(double) * nh);
            if (!hsd) return fail(c, PSB_ENOMEM, "scratch allocation failed (hs)");
            PSB_CUDA_TRY(c, cudaMemcpyAsync(hsd, hs, sizeof(double) * nh, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s),
                         "hs copy");
            if (line) {
                hs_host.resize(nh);
                PSB_CUDA_TRY(c, cudaMemcpyAsync(hs_host.data(), hsd, sizeof(double) * nh, cudaMemcpyDeviceToHost, s), "hs D2H");
            }
        }
        double* god = (double*)scratch(c, 21, sizeof(double) * (size_t)(L > 0 ? L : 1) * ns);
        const double** gptr = (const double**)scratch(c, 22, sizeof(void*) * (L > 0 ? L : 1));
        const int nq = line ? 1 + kc : 8 + 4 * kc;
        double* lam = (double*)scratch(c, 23, sizeof(double) * (size_t)nq * ns);
        double* ha = (double*)scratch(c, 24, sizeof(double) * ns);
        if (!god || !gptr || !lam || !ha) return fail(c, PSB_ENOMEM, "scratch allocation failed (cotangents)");
        std::vector<const double*> gp(L > 0 ? L : 1);
        for (int k = 0; k < L; ++k) {
            PSB_CUDA_TRY(c, cudaMemcpyAsync(god + (size_t)k * ns, gout[k], sizeof(double) * ns,
                                            dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s), "gout copy");
            gp[k] = god + (size_t)k * ns;
        }
        PSB_CUDA_TRY(c, cudaMemcpyAsync(gptr, gp.data(), sizeof(void*) * (L > 0 ? L : 1), cudaMemcpyHostToDevice, s),
                     "gout table copy");
        PSB_CUDA_TRY(c, cudaMemsetAsync(ha, 0, sizeof(double) * ns, s), "memset");
        PSB_CUDA_TRY(c, cudaStreamSynchronize(s), "synchronize");  // host staging buffers are released below

        // ---- sum cotangents: directly from gout when the catalog allows and
        // h_a needs no nearest search, else a forward pass in FP64 ----
        bool direct = true, scal = true;
        for (int o = 0; o < L; ++o) {
            if (rec.op[o] != OP_SCALAR || rec.a1[o]) direct = false;
            if (rec.op[o] != OP_SCALAR) scal = false;
        }
        if (!line && st != ST_SCATTER && hmode == PSB_H_NEAREST) direct = false;
        if (direct) {
            const unsigned gb = (unsigned)((ns + 255) / 256);
            k_direct_cotangents<<<gb, 256, 0, s>>>(rec, gptr, ns, nq, line, lam);
            if (need_h) k_fill_ha<<<gb, 256, 0, s>>>(hsd, hmode == PSB_H_PER_SAMPLE, ns, ha);
            PSB_CUDA_TRY(c, cudaGetLastError(), "cotangent kernel");
            launches += need_h ? 2 : 1;
        } else {
            AdjHook hook{c};
            c->adj_gout = gptr;
            c->adj_lam = lam;
            c->adj_lam_stride = ns;
            c->adj_ha = ha;
            psb_stats fst;
            memset(&fst, 0, sizeof(fst));
            // (a grid runs as a grid: its sample index is that of the coordinate arrays)
            rc = run(c, rq0.kind == SRC_GRID ? rq0 : rq, hmode, need_h ? (const void*)hsd : nullptr, st, cat,
                     PREC_FP64, nullptr, PSB_FLAG_DEVICE_PTRS | (flags & PSB_FLAG_DENSITY_GRADIENT_PLAIN), &fst,
                     WHAT_INTERP, nullptr, nullptr, nullptr);
            if (rc) return rc;
            launches += fst.launches;
        }

        AdjArgs J;
        memset((void*)&J, 0, sizeof(J));
        J.pt = tree_view<double>(c);
        for (int q = 0; q < kc; ++q) J.colT[q] = (const double*)c->cols[colu[q]];
        J.kc = kc;
        J.lam_stride = ns;
        J.porder = c->order;
        J.gm = g_m; J.gx = g_x; J.gy = g_y; J.gz = g_z;
        for (int q = 0; q < kc; ++q) J.gcol[q] = g_c[q];
        J.err = c->d_err;
        unsigned long long* dstats = (unsigned long long*)scratch(c, 13, 8 * sizeof(unsigned long long));
        if (!dstats) return fail(c, PSB_ENOMEM, "scratch allocation failed (stats)");
        PSB_CUDA_TRY(c, cudaMemsetAsync(dstats, 0, 8 * sizeof(unsigned long long), s), "memset stats");
        J.stats = dstats;
        const int kcl = kc <= 1 ? 1 : (kc <= 2 ? 2 : (kc <= 4 ? 4 : 8));
        PSB_CUDA_TRY(c, cudaEventRecord(c->ev[1], s), "event");
        if (!line) {
            // ---- LBVH over the samples, h = h_a ----
            if (!c->sctx) {
                psb_ctx* sc = nullptr;
                int r2 = psb_create(&sc, c->device);
                if (r2) return fail(c, r2, "could not create the sample-tree context");
                c->sctx = sc;
            }
            psb_set_stream(c->sctx, (void*)s);
            rc = psb_set_particles(c->sctx, ns, PSB_F64, xyz, xyz + ns, xyz + 2 * ns, ha, ha, ha, 0, nullptr,
                                   PSB_KERNEL_M4, PSB_FLAG_DEVICE_PTRS);
            if (!rc) rc = build_lbvh(c->sctx);
            if (rc) return fail(c, rc, std::string("sample tree: ") + c->sctx->err);
            double* lams = (double*)scratch(c, 26, sizeof(double) * (size_t)nq * ns);
            if (!lams) return fail(c, PSB_ENOMEM, "scratch allocation failed (cotangents)");
            k_gather_rows<<<(unsigned)((ns + 255) / 256), 256, 0, s>>>(lam, c->sctx->order, ns, nq, lams);
            PSB_CUDA_TRY(c, cudaGetLastError(), "cotangent gather");
            J.sv = tree_view<double>(c->sctx);
            J.lam = lams;
            const unsigned g = (unsigned)((n + 127) / 128);
            const int kf = (c->kern == PSB_KERNEL_M4) ? 0 : 1;
            if (c->adj_split) {
                // Two kernels and a combine: the walk writes each particle
                // tile's pair lists into blocks of a pool (k_adj_points in its
                // list form, at the walk's own register budget); one warp per
                // list block sums the block's pairs into partial sums
                // (k_adj_bodies), and the partial sums of each particle are
                // added in its chain's order (k_adj_combine).  If the pool runs
                // out, it grows to what the walk asked for and the walk runs
                // again; after three rounds (or at the pool's 32 GiB cap) the
                // tiles still left run in k_adj_points.  A call grows the pool
                // for the next; it starts at two blocks per tile.
                const int64_t ntiles = (n + 31) / 32;
                const int nf = 8 + kcl;  // AdjAcc<kcl>::NF
                const int64_t per_block = (int64_t)ADJ_CH * 32 * 8 + 32 + 8 + (int64_t)nf * 32 * 8;
                const int64_t cap = (int64_t)(32ll << 30) / per_block;
                if (c->adj_blocks <= 0) c->adj_blocks = std::min<int64_t>(cap, 2 * ntiles + 64);
                const int nqc = scal ? 1 + kcl : 8 + 4 * kcl;
                const int nrec = 6 + ((nqc + 1) & ~1);  // AdjRec<kcl, scal>::N
                double* recs = (double*)scratch(c, 88, sizeof(double) * (size_t)nrec * ns);
                if (!recs) return fail(c, PSB_ENOMEM, "scratch allocation failed (adjoint records)");
                J.lamT = recs;
                launch_adj_rows(kcl, scal, lams, ns, kc, J.sv, recs, s);
                AdjLists& al = J.al;
                unsigned ptop = 0, povf = 0;
                // The walk takes its tiles heaviest first (and with them the pool's
                // blocks, which k_adj_bodies then runs in that order) when there
                // are few tiles per SM: then the heavy tiles set the end (C2:
                // 65,536 tiles, 8-field backward 22.1 -> 21.5 ms).  With many (the
                // 2M tiles of 64M particles) the tail is a small part, and the
                // Morton order's locality in the sample tree counts for more
                // (there the cost-ordered walk took 101.5 against 99.8 ms).
                AdjArgs W = J;
                if (ntiles < (1ll << 18)) {
                    uint64_t* tk = (uint64_t*)scratch(c, 94, sizeof(uint64_t) * (size_t)ntiles);
                    char* tv = (char*)scratch(c, 95, sizeof(uint32_t) * (size_t)ntiles + 16);
                    if (!tk || !tv) return fail(c, PSB_ENOMEM, "scratch allocation failed (tile order)");
                    const double* bb = c->sctx->bbox;  // the samples' box
                    k_adj_tile_keys<<<(unsigned)((ntiles + 255) / 256), 256, 0, s>>>(
                        (const double*)c->x, (const double*)c->y, (const double*)c->z, (const double*)c->h, n, ntiles,
                        (double)J.pt.Kd, bb[0], bb[1], bb[2], bb[3], bb[4], bb[5], tk, (uint32_t*)(tv + 16));
                    unsigned cnt = (unsigned)ntiles;
                    PSB_CUDA_TRY(c, cudaMemcpyAsync(tv, &cnt, sizeof(unsigned), cudaMemcpyHostToDevice, s), "tile count");
                    PSB_CUDA_TRY(c, radix_sort_pairs(tk, (uint32_t*)(tv + 16), ntiles, c, 6, &launches, false, 16),
                                 "tile order sort");
                    W.tile_list = (const int32_t*)(tv + 16);
                    W.tile_count = (const unsigned*)tv;
                    launches += 1;
                }
                for (int round = 0;; ++round) {
                    const int64_t nb = c->adj_blocks;
                    const size_t b_ent = sizeof(uint2) * (size_t)nb * ADJ_CH * 32, b_cnt = (size_t)nb * 32,
                                 b_next = sizeof(int32_t) * (size_t)nb, b_part = sizeof(double) * (size_t)nb * nf * 32,
                                 b_tile = sizeof(int32_t) * (size_t)ntiles;
                    char* pool = (char*)scratch(c, 87, b_part + b_ent + b_cnt + 2 * b_next + 2 * b_tile + 256);
                    if (!pool) return fail(c, PSB_ENOMEM, "scratch allocation failed (adjoint pair lists)");
                    al.part = (double*)pool;
                    al.ent = (uint2*)(pool + b_part);
                    al.bcnt = (uint8_t*)(pool + b_part + b_ent);
                    al.bnext = (int32_t*)(pool + b_part + b_ent + b_cnt);
                    al.btile = (int32_t*)(pool + b_part + b_ent + b_cnt + b_next);
                    al.head = (int32_t*)(pool + b_part + b_ent + b_cnt + 2 * b_next);
                    al.ovf_tiles = (int32_t*)(pool + b_part + b_ent + b_cnt + 2 * b_next + b_tile);
                    al.top = (unsigned*)(pool + b_part + b_ent + b_cnt + 2 * b_next + 2 * b_tile);
                    al.ovf_count = al.top + 1;
                    al.nblocks = nb;
                    PSB_CUDA_TRY(c, cudaMemsetAsync(al.top, 0, 2 * sizeof(unsigned), s), "memset pool counters");
                    W.al = al;
                    launch_adj_points(W, kcl, st, scal, kf, 1, g, s);
                    PSB_CUDA_TRY(c, cudaGetLastError(), "adjoint walk launch");
                    unsigned hc[2] = {0, 0};
                    PSB_CUDA_TRY(c, cudaMemcpyAsync(hc, al.top, sizeof(hc), cudaMemcpyDeviceToHost, s), "pool D2H");
                    PSB_CUDA_TRY(c, cudaStreamSynchronize(s), "synchronize");
                    ptop = hc[0];
                    povf = hc[1];
                    launches += 1;
                    if (povf == 0 || c->adj_split == 2 || round == 2 || nb >= cap) break;
                    // the tiles that ran out stopped asking: at least double the pool
                    c->adj_blocks = std::min<int64_t>(cap, std::max<int64_t>(2 * nb, (int64_t)ptop + ptop / 4 + 64));
                }
                const int64_t used = std::min<int64_t>((int64_t)ptop, c->adj_blocks);
                if (used > 0) launch_adj_points(J, kcl, st, scal, kf, 2, (unsigned)((used + 3) / 4), s);
                launch_adj_points(J, kcl, st, scal, kf, 3, g, s);
                if (povf) {  // tiles the largest pool could not hold
                    AdjArgs F = J;
                    F.tile_list = al.ovf_tiles;
                    F.tile_count = al.ovf_count;
                    launch_adj_points(F, kcl, st, scal, kf, 0, g, s);
                    ++launches;
                }
                PSB_CUDA_TRY(c, cudaGetLastError(), "adjoint kernel launch");
                if ((int64_t)ptop > c->adj_blocks && c->adj_split != 2)
                    c->adj_blocks = std::min<int64_t>(cap, (int64_t)ptop + ptop / 4 + 64);
                launches += 3;
            } else {
                launch_adj_points(J, kcl, st, scal, kf, 0, g, s);
                PSB_CUDA_TRY(c, cudaGetLastError(), "adjoint kernel launch");
                launches += 2;
            }
        } else {
            J.lam = lam;
            SampleSrc<double>& B = J.beam;
            B.kind = SRC_BEAM;
            B.ns = ns;
            memcpy(B.frame, rq0.frame, sizeof(double) * 12);
            memcpy(B.params, rq0.params, sizeof(double) * 4);
            B.nx = rq0.nx; B.ny = rq0.ny; B.nz = 1;
            J.hmode = hmode;
            J.hs = hsd;
            double hmax = 0.0;
            for (double v : hs_host) hmax = std::max(hmax, v);
            J.ha_max = hmax;
            J.lut = c->lut_d;
            const unsigned g = (unsigned)((n + 127) / 128);
            if (kcl == 1) launch_adj_beam_k<1>(J, st, g, s);
            else if (kcl == 2) launch_adj_beam_k<2>(J, st, g, s);
            else if (kcl == 4) launch_adj_beam_k<4>(J, st, g, s);
            else launch_adj_beam_k<8>(J, st, g, s);
            PSB_CUDA_TRY(c, cudaGetLastError(), "adjoint kernel launch");
            launches += 1;
        }
        PSB_CUDA_TRY(c, cudaEventRecord(c->ev[2], s), "event");
        unsigned long long hst[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        PSB_CUDA_TRY(c, cudaMemcpyAsync(hst, dstats, sizeof(hst), cudaMemcpyDeviceToHost, s), "stats D2H");
        unsigned herr = 0;
        PSB_CUDA_TRY(c, cudaMemcpyAsync(&herr, c->d_err, sizeof(herr), cudaMemcpyDeviceToHost, s), "error D2H");
        PSB_CUDA_TRY(c, cudaStreamSynchronize(s), "synchronize");
        if (herr) {
            cudaMemsetAsync(c->d_err, 0, sizeof(unsigned), s);
            cudaStreamSynchronize(s);
            return device_error(c, herr);
        }
        if (stats) {
            memset(stats, 0, sizeof(*stats));
            float ms = 0.f;
            cudaEventElapsedTime(&ms, c->ev[1], c->ev[2]);
            stats->interp_ms = ms;
            stats->pairs = (int64_t)(hst[0] + hst[6]);  // k_adj_points, k_adj_bodies
            stats->warp_steps = (int64_t)hst[2];
            stats->spans = (int64_t)hst[3];       // spans visited (point samples)
            stats->span_tests = (int64_t)hst[4];  // particle-span tests
            stats->body_iters = (int64_t)hst[5];  // samples in the visited spans
        }
    }
    // ---- gradients to the caller ----
    if (!dev && n > 0) {
        PSB_CUDA_TRY(c, cudaMemcpyAsync(gm, g_m, sizeof(double) * n, cudaMemcpyDeviceToHost, s), "gradient D2H");
        PSB_CUDA_TRY(c, cudaMemcpyAsync(gx, g_x, sizeof(double) * n, cudaMemcpyDeviceToHost, s), "gradient D2H");
        PSB_CUDA_TRY(c, cudaMemcpyAsync(gy, g_y, sizeof(double) * n, cudaMemcpyDeviceToHost, s), "gradient D2H");
        PSB_CUDA_TRY(c, cudaMemcpyAsync(gz, g_z, sizeof(double) * n, cudaMemcpyDeviceToHost, s), "gradient D2H");
        for (int k = 0; gcols && k < c->ncol; ++k) {
            if (!gcols[k]) continue;
            int q = -1;
            for (int t = 0; t < kc; ++t)
                if (colu[t] == k) q = t;
            if (q >= 0)
                PSB_CUDA_TRY(c, cudaMemcpyAsync(gcols[k], g_c[q], sizeof(double) * n, cudaMemcpyDeviceToHost, s),
                             "gradient D2H");
            else
                memset(gcols[k], 0, sizeof(double) * n);
        }
    }
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[3], s), "event");
    PSB_CUDA_TRY(c, cudaStreamSynchronize(s), "synchronize");
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev[0], c->ev[3]);
        stats->total_ms = ms;
        stats->launches = launches;
    }
    return PSB_OK;
}

}  // namespace psb
