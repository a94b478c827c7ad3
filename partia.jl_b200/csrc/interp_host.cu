// interp_host.cu -- host drivers of the interpolation calls: argument checks,
// catalog -> output recipe, host<->device staging, sample ordering, launch,
// statistics and device error words.
#include "launch.hpp"
#include "psb_ctx.hpp"
#include "psb_host.hpp"

namespace psb {

template <class T> TreeView<T> tree_view(psb_ctx* c) {
    TreeView<T> v;
    v.n = c->n;
    v.root = c->root;
    v.left = c->left;
    v.escape = c->escape;
    v.range_lo = c->range_lo;
    v.range_hi = c->range_hi;
    v.links = c->links;
    v.codes = c->codes;
    for (int d = 0; d < 3; ++d) {
        v.qlo[d] = c->bbox[d];
        double ext = c->bbox[3 + d] - c->bbox[d];
        v.qscale[d] = ext > 0 ? 2097151.0 / ext : 0.0;
    }
    for (int d = 0; d < 3; ++d) { v.nmin[d] = (const T*)c->nmin[d]; v.nmax[d] = (const T*)c->nmax[d]; }
    v.nscale = (const T*)c->nscale;
    v.x = (const T*)c->x; v.y = (const T*)c->y; v.z = (const T*)c->z;
    v.h = (const T*)c->h; v.m = (const T*)c->m; v.rho = (const T*)c->rho;
    v.cols = (const T* const*)c->d_cols;
    v.ncol = c->ncol;
    v.node_lo = c->node_lo; v.node_hi = c->node_hi; v.leaf4 = c->leaf4;
    v.mrho = c->mrho; v.mf = c->mf; v.leafK = c->leafK; v.spanb = c->spanb;
    v.coord_err = c->coord_err;
    v.kern = (int)c->kern;
    v.Kd = kern_support(v.kern);
    v.Kf = (float)v.Kd;
    v.sig = kern_norm3(v.kern);
    v.qedge = kern_qedge(v.kern);
    return v;
}
template TreeView<double> tree_view<double>(psb_ctx*);
template TreeView<float> tree_view<float>(psb_ctx*);

// InterpolationCatalogConcise -> per-output recipe over the distinct columns.
// Output order: scalars, 3 per gradient, 1 per divergence, 3 per curl
// (grid_interpolation/kernels/PointSamples_kernel.jl:30-71).
int make_recipe(psb_ctx* c, const psb_catalog* cat, bool line, Recipe& rec, std::vector<int>& colu) {
    rec = Recipe();
    colu.clear();
    if (!cat) return fail(c, PSB_EINVAL, "catalog must not be NULL");
    if (cat->n_scalar < 0 || cat->n_grad < 0 || cat->n_div < 0 || cat->n_curl < 0)
        return fail(c, PSB_EINVAL, "catalog counts must be non-negative");
    if (line && (cat->n_grad || cat->n_div || cat->n_curl))
        return fail(c, PSB_EINVAL, "line-integrated interpolation supports scalar quantities only");
    const int L = cat->n_scalar + 3 * cat->n_grad + cat->n_div + 3 * cat->n_curl;
    if (L > MAX_OUT) return fail(c, PSB_EUNSUPPORTED, "catalog expands to more than 64 output fields");
    auto col_index = [&](int slot, int& ci) -> int {
        if (slot < 0 || slot >= c->ncol) return fail(c, PSB_EINVAL, "catalog column slot " + std::to_string(slot) +
                                                     " out of range (ncol=" + std::to_string(c->ncol) + ")");
        for (size_t q = 0; q < colu.size(); ++q)
            if (colu[q] == slot) { ci = (int)q; return PSB_OK; }
        if ((int)colu.size() >= MAX_KC) return fail(c, PSB_EUNSUPPORTED, "catalog references more than 8 distinct columns");
        colu.push_back(slot);
        ci = (int)colu.size() - 1;
        return PSB_OK;
    };
    int o = 0, ci, cj, ck, rc;
    for (int j = 0; j < cat->n_scalar; ++j) {
        if ((rc = col_index(cat->scalar_slots[j], ci))) return rc;
        rec.op[o] = OP_SCALAR; rec.a0[o] = (int8_t)ci; rec.a1[o] = (int8_t)(cat->scalar_shepard[j] ? 1 : 0); ++o;
    }
    for (int j = 0; j < cat->n_grad; ++j) {
        int slot = cat->grad_slots[j];
        if (slot == -1) {
            rec.need_dg = 1;
            for (int d = 0; d < 3; ++d) { rec.op[o] = OP_GRADD; rec.a1[o] = (int8_t)d; ++o; }
        } else {
            if ((rc = col_index(slot, ci))) return rc;
            for (int d = 0; d < 3; ++d) { rec.op[o] = OP_GRADC; rec.a0[o] = (int8_t)ci; rec.a1[o] = (int8_t)d; ++o; }
        }
    }
    for (int j = 0; j < cat->n_div; ++j) {
        if ((rc = col_index(cat->div_slots[3 * j], ci)) || (rc = col_index(cat->div_slots[3 * j + 1], cj)) ||
            (rc = col_index(cat->div_slots[3 * j + 2], ck)))
            return rc;
        rec.op[o] = OP_DIV; rec.a0[o] = (int8_t)ci; rec.a1[o] = (int8_t)cj; rec.a2[o] = (int8_t)ck; ++o;
    }
    for (int j = 0; j < cat->n_curl; ++j) {
        if ((rc = col_index(cat->curl_slots[3 * j], ci)) || (rc = col_index(cat->curl_slots[3 * j + 1], cj)) ||
            (rc = col_index(cat->curl_slots[3 * j + 2], ck)))
            return rc;
        for (int d = 0; d < 3; ++d) {
            rec.op[o] = OP_CURL; rec.a0[o] = (int8_t)ci; rec.a1[o] = (int8_t)cj; rec.a2[o] = (int8_t)ck;
            rec.a3[o] = (int8_t)d; ++o;
        }
    }
    rec.L = L;
    rec.kc = (int)colu.size();
    return PSB_OK;
}

static float ms_between(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

// Two-kernel point path over batches of tiles: k_collect writes the pair
// lists of a batch, k_bodies sums them, and k_points takes the tiles whose
// lists overflowed.  A batch holds at most SPLIT_BATCH tiles, which bounds the
// list memory at SPLIT_BATCH * RCAP * 32 * 20 bytes (640 MiB) per stream.
//
// A direct call (multi_stream) of at least two batches' worth of tiles
// spreads its batches over up to SPLIT_STREAMS streams (the context stream and
// the context's own), each with its own lists, so that the walks and pair sums
// of different batches run side by side: the walk is bound by compare and vote
// issue, the pair sums by load latency, and one kernel alone leaves SMs idle in
// its tail.  On the 2M-particle 128^3 grid this takes the FP32C step from 7.5
// to 5.9 ms and the FP64 step from 12.0 to 8.0 ms.
constexpr int64_t SPLIT_BATCH = 32768;
constexpr int SPLIT_STREAMS = 4;
template <class T>
static int run_split(psb_ctx* c, Args<T>& A, int prec, int st, int* launches, int slot_off = 0,
                     bool multi_stream = true) {
    cudaStream_t s = c->stream;
    const int64_t nt = A.src.ntiles;
    int nsets = 1;
    int64_t B = std::min<int64_t>(nt, SPLIT_BATCH);
    if (multi_stream && nt >= 2 * 4096) {
        nsets = (int)std::min<int64_t>(SPLIT_STREAMS, (nt + 4095) / 4096);
        B = std::min<int64_t>(SPLIT_BATCH, (nt + nsets - 1) / nsets);
    }
    cudaStream_t ss[SPLIT_STREAMS] = {s, s, s, s};
    if (nsets > 1) {
        for (auto& e : c->sev)
            if (!e) PSB_CUDA_TRY(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        PSB_CUDA_TRY(c, cudaEventRecord(c->sev[0], s), "event");
        for (int k = 1; k < nsets; ++k) {
            if (!c->sstream[k - 1])
                PSB_CUDA_TRY(c, cudaStreamCreateWithFlags(&c->sstream[k - 1], cudaStreamNonBlocking), "stream");
            ss[k] = c->sstream[k - 1];
            // the other streams start after everything the call staged on s
            PSB_CUDA_TRY(c, cudaStreamWaitEvent(ss[k], c->sev[0], 0), "stream wait");
        }
    }
    struct Lists {
        float4* ent4; uint32_t* emask; float* eshift; uint8_t* cnt; void* hab; unsigned* ovf_count; int32_t* ovf_tiles;
    };
    // FP32C sums of double inputs take per-entry column shifts for the kernels
    // other than M4 (span_shift; slots 80-86)
    const bool shifts = sizeof(T) == 8 && prec == PREC_FP32C && A.rec.kc > 0 && c->kern != PSB_KERNEL_M4;
    Lists ls[SPLIT_STREAMS];
    for (int k = 0; k < nsets; ++k) {
        // scratch slots 16-20 (+ slot_off), 48-52, 37-41 and 42-46 (clear of the
        // build, sort, sample-order and adjoint slots)
        static const int set_off[SPLIT_STREAMS] = {0, 32, 21, 26};
        const int so = slot_off + set_off[k];
        ls[k].ent4 = (float4*)scratch(c, 16 + so, sizeof(float4) * (size_t)RCAP * 32 * B);
        ls[k].emask = (uint32_t*)scratch(c, 20 + so, sizeof(uint32_t) * (size_t)RCAP * 32 * B);
        ls[k].eshift = nullptr;
        if (shifts) {
            const int es_slot = 80 + (slot_off == 0 ? k : (slot_off == 32 ? 4 : (slot_off == 14 ? 5 : 6)));
            ls[k].eshift = (float*)scratch(c, es_slot, sizeof(float) * (size_t)RCAP * 32 * B * A.rec.kc);
            if (!ls[k].eshift) return fail(c, PSB_ENOMEM, "scratch allocation failed (pair-list shifts)");
        }
        ls[k].cnt = (uint8_t*)scratch(c, 17 + so, (size_t)32 * B);
        ls[k].hab = scratch(c, 18 + so, sizeof(double) * 32 * (size_t)B);
        char* ovf = (char*)scratch(c, 19 + so, 256 + sizeof(int32_t) * (size_t)B);
        if (!ls[k].ent4 || !ls[k].emask || !ls[k].cnt || !ls[k].hab || !ovf)
            return fail(c, PSB_ENOMEM, "scratch allocation failed (pair lists)");
        ls[k].ovf_count = (unsigned*)ovf;
        ls[k].ovf_tiles = (int32_t*)(ovf + 256);
    }
    // The adjoint's cotangent pass (double particles) collects its pair lists
    // with the FP32C walk: float tests with the exact double test for every
    // undecided pair give the same pairs in the same order as the double
    // walk, at about half its cost; the sums stay in double.
    const int cprec = (sizeof(T) == 8 && A.lam) ? PREC_FP32C : prec;
    int64_t bi = 0;
    for (int64_t t0 = 0; t0 < nt; t0 += B, ++bi) {
        const int k = (int)(bi % nsets);
        const cudaStream_t sk = ss[k];
        const int64_t nb = std::min<int64_t>(B, nt - t0);
        PSB_CUDA_TRY(c, cudaMemsetAsync(ls[k].ovf_count, 0, sizeof(unsigned), sk), "memset overflow count");
        A.sp.ent4 = ls[k].ent4; A.sp.emask = ls[k].emask; A.sp.cnt = ls[k].cnt; A.sp.ha = ls[k].hab;
        A.sp.eshift = ls[k].eshift;
        A.sp.ovf_tiles = ls[k].ovf_tiles; A.sp.ovf_count = ls[k].ovf_count;
        A.sp.tile0 = t0; A.sp.ntiles = nb;
        PSB_CUDA_TRY(c, launch_split(A, cprec, st, A.rec.kc, false, sk), "pair-list kernel launch");
        PSB_CUDA_TRY(c, launch_split(A, prec, st, A.rec.kc, true, sk), "pair-sum kernel launch");
        Args<T> F = A;
        F.tile_list = ls[k].ovf_tiles;
        F.tile_count = ls[k].ovf_count;
        F.src.ntiles = nb;  // grid of the list pass: at most nb tiles
        PSB_CUDA_TRY(c, launch_points<T>(F, prec, st, A.rec.kc, WHAT_INTERP, sk), "overflow pass launch");
        *launches += 3;
    }
    for (int k = 1; k < nsets; ++k) {  // the call's later work on s follows every stream
        PSB_CUDA_TRY(c, cudaEventRecord(c->sev[k], ss[k]), "event");
        PSB_CUDA_TRY(c, cudaStreamWaitEvent(s, c->sev[k], 0), "stream wait");
    }
    return PSB_OK;
}

// Heavy tiles first for parallel beams.  A line's work is the particles
// whose support it crosses, and lines through dense clumps take many times
// the mean: in index order the heaviest tiles can start last and leave the
// SMs idle at the end (on the 8M-particle clump beam, a list-scheduling
// estimate from the per-tile pair counts puts the last CTA at 1.19x the
// ideal finish, 1.01x with the heaviest first).  The cost of a tile is
// estimated from the particles projected onto the frame plane: each adds
// the lines its support can cross, pi (K h / dx) (K h / dy) + 1, to the
// tile of its centre pixel.  Only the order of the tiles changes, never a
// result.
template <class T>
__global__ void k_beam_tile_cost(const TreeView<T> tv, const SampleSrc<T> s, int64_t nbx, float* cost) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= tv.n) return;
    const double v0 = (double)tv.x[i] - (double)s.frame[0], v1 = (double)tv.y[i] - (double)s.frame[1],
                 v2 = (double)tv.z[i] - (double)s.frame[2];
    const double xi = v0 * (double)s.frame[3] + v1 * (double)s.frame[4] + v2 * (double)s.frame[5];
    const double eta = v0 * (double)s.frame[6] + v1 * (double)s.frame[7] + v2 * (double)s.frame[8];
    const double dx = ((double)s.params[1] - (double)s.params[0]) / (double)(s.nx - 1);
    const double dy = ((double)s.params[3] - (double)s.params[2]) / (double)(s.ny - 1);
    const double u = (xi - (double)s.params[0]) / dx, w = (eta - (double)s.params[2]) / dy;
    const double r = tv.Kd * (double)tv.h[i];
    const double ru = fabs(r / dx), rw = fabs(r / dy);
    if (!(u > -ru - 1.0 && u < (double)s.nx + ru && w > -rw - 1.0 && w < (double)s.ny + rw)) return;
    const int64_t ic = (int64_t)fmin(fmax(rint(u), 0.0), (double)(s.nx - 1));
    const int64_t jc = (int64_t)fmin(fmax(rint(w), 0.0), (double)(s.ny - 1));
    atomicAdd(&cost[(jc >> 2) * nbx + (ic >> 3)], (float)(3.141592653589793 * ru * rw + 1.0));
}
// keys for an ascending sort that puts the largest cost first
__global__ void k_cost_keys(const float* cost, int64_t n, uint64_t* keys, uint32_t* vals) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    keys[t] = 0xFFFFFFFFull - (uint64_t)__float_as_uint(cost[t]);
    vals[t] = (uint32_t)t;
}

template <class T>
static int run_typed(psb_ctx* c, const SampleReq& rq, int hmode, const void* hs, int st, const psb_catalog* cat,
                     int prec, void* const* out, uint32_t flags, psb_stats* stats, int what, int64_t* dcount,
                     uint64_t* dhash, void* ha_out) {
    const bool dev = (flags & PSB_FLAG_DEVICE_PTRS) != 0;
    cudaStream_t s = c->stream;
    const size_t es = sizeof(T);
    const int64_t ns = rq.ns;
    int launches = 0;

    Args<T> A;
    memset((void*)&A, 0, sizeof(A));
    std::vector<int> colu;
    if (what == WHAT_INTERP) {
        int rc = make_recipe(c, cat, rq.line, A.rec, colu);
        if (rc) return rc;
        if (flags & PSB_FLAG_DENSITY_GRADIENT_PLAIN)
            for (int o = 0; o < A.rec.L; ++o)
                if (A.rec.op[o] == OP_GRADD) A.rec.a2[o] = 1;
    } else {
        A.rec.L = (what == WHAT_DENSITY) ? 1 : 0;
        A.unit_mass = (what == WHAT_DENSITY && (flags & PSB_FLAG_NUMBER_DENSITY)) ? 1 : 0;
    }
    const int L = A.rec.L;
    const bool adj = (what == WHAT_INTERP) && c->adj_lam;  // adjoint sum-cotangent pass: no fields written
    if (what == WHAT_INTERP && !adj && L > 0 && !out) return fail(c, PSB_EINVAL, "output pointer array must not be NULL");
    for (int k = 0; what == WHAT_INTERP && !adj && k < L && ns > 0; ++k)
        if (!out[k]) return fail(c, PSB_EINVAL, "output pointer " + std::to_string(k) + " is NULL");
    if (what == WHAT_DENSITY && ns > 0 && (!out || !out[0])) return fail(c, PSB_EINVAL, "density output is NULL");
    if (what == WHAT_DIGEST && ns > 0 && (!dcount || !dhash)) return fail(c, PSB_EINVAL, "digest outputs are NULL");
    const bool need_h = (st != ST_SCATTER) && !(hmode == PSB_H_NEAREST && !rq.line);
    if (need_h && !hs) return fail(c, PSB_EINVAL, "hs must not be NULL for this strategy and hmode");
    if (dev && ns > 0) {  // pointers the kernels dereference directly
        int rc = PSB_OK;
        for (int q = 0; !rc && rq.kind == SRC_ARRAYS && q < (rq.line ? 6 : 3); ++q)
            rc = check_device_ptr(c, rq.a[q], "a sample coordinate array");
        if (!rc && need_h) rc = check_device_ptr(c, hs, "hs");
        for (int k = 0; !rc && what == WHAT_INTERP && !adj && k < L; ++k) rc = check_device_ptr(c, out[k], "an output array");
        if (!rc && what == WHAT_DENSITY) rc = check_device_ptr(c, out[0], "the density output");
        if (!rc && what == WHAT_DIGEST) rc = check_device_ptr(c, dcount, "the digest counts");
        if (!rc && what == WHAT_DIGEST) rc = check_device_ptr(c, dhash, "the digest hashes");
        if (!rc && what == WHAT_DIGEST) rc = check_device_ptr(c, ha_out, "the digest smoothing lengths");
        if (rc) return rc;
    }

    A.tv = tree_view<T>(c);
    A.hmode = hmode;
    A.err = c->d_err;
    A.lut_d = c->lut_d;
    A.lut_f = c->lut_f;
    A.lut_fs = c->lut_fs;
    A.lut_n = (flags & PSB_FLAG_LUT1000_F32) ? LUT_SHORT_N : LUT_N;
    if (adj) {
        A.gout = c->adj_gout;
        A.lam = c->adj_lam;
        A.lam_stride = c->adj_lam_stride;
        A.ha_out = (T*)c->adj_ha;
    }
    for (size_t q = 0; q < colu.size(); ++q) {
        A.colT[q] = (const T*)c->cols[colu[q]];
        A.colF[q] = (sizeof(T) == 8) ? c->colsf + (size_t)colu[q] * c->n : (const float*)c->cols[colu[q]];
        A.colR[q] = (sizeof(T) == 8) ? c->colsr + (size_t)colu[q] * c->n : nullptr;
    }
    SampleSrc<T>& S = A.src;
    S.kind = rq.kind;
    S.ns = ns;

    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[0], s), "event");
    // ---- stage samples ----
    const int narr = rq.line ? 6 : 3;
    if (rq.kind == SRC_ARRAYS) {
        if (dev) {
            for (int q = 0; q < narr; ++q) S.a[q] = (const T*)rq.a[q];
        } else if (ns > 0) {
            char* buf = (char*)scratch(c, 0, es * ns * narr);
            if (!buf) return fail(c, PSB_ENOMEM, "scratch allocation failed (samples)");
            for (int q = 0; q < narr; ++q) {
                PSB_CUDA_TRY(c, cudaMemcpyAsync(buf + es * ns * q, rq.a[q], es * ns, cudaMemcpyHostToDevice, s), "sample H2D");
                S.a[q] = (const T*)(buf + es * ns * q);
            }
        }
        S.ntiles = (ns + 31) / 32;
    } else if (rq.kind == SRC_GRID) {
        char* buf = (char*)scratch(c, 14, es * (rq.nx + rq.ny + rq.nz));
        if (!buf) return fail(c, PSB_ENOMEM, "scratch allocation failed (axes)");
        PSB_CUDA_TRY(c, cudaMemcpyAsync(buf, rq.ax, es * rq.nx, cudaMemcpyHostToDevice, s), "axis H2D");
        PSB_CUDA_TRY(c, cudaMemcpyAsync(buf + es * rq.nx, rq.ay, es * rq.ny, cudaMemcpyHostToDevice, s), "axis H2D");
        PSB_CUDA_TRY(c, cudaMemcpyAsync(buf + es * (rq.nx + rq.ny), rq.az, es * rq.nz, cudaMemcpyHostToDevice, s), "axis H2D");
        S.ax = (const T*)buf; S.ay = (const T*)(buf + es * rq.nx); S.az = (const T*)(buf + es * (rq.nx + rq.ny));
        S.nx = rq.nx; S.ny = rq.ny; S.nz = rq.nz;
        S.ntiles = ((rq.nx + 3) / 4) * ((rq.ny + 3) / 4) * ((rq.nz + 1) / 2);
    } else {
        memcpy(S.frame, rq.frame, es * 12);
        memcpy(S.params, rq.params, es * (rq.kind == SRC_BOX ? 6 : 4));
        S.nx = rq.nx; S.ny = rq.ny; S.nz = rq.nz;
        S.ntiles = (rq.kind == SRC_BOX) ? ((rq.nx + 3) / 4) * ((rq.ny + 3) / 4) * ((rq.nz + 1) / 2)
                                        : ((rq.nx + 7) / 8) * ((rq.ny + 3) / 4);
    }
    if (need_h) {
        if (dev) A.hs = (const T*)hs;
        else {
            const int64_t nh = (hmode == PSB_H_PER_SAMPLE) ? ns : 1;
            T* hb = (T*)scratch(c, 1, es * std::max<int64_t>(nh, 1));
            if (!hb) return fail(c, PSB_ENOMEM, "scratch allocation failed (hs)");
            if (nh > 0) PSB_CUDA_TRY(c, cudaMemcpyAsync(hb, hs, es * nh, cudaMemcpyHostToDevice, s), "hs H2D");
            A.hs = hb;
        }
    }
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[1], s), "event");

    // ---- Morton order of explicit samples ----
    if (rq.kind == SRC_ARRAYS && ns > 64) {
        uint64_t* codes = (uint64_t*)scratch(c, 3, sizeof(uint64_t) * ns);
        uint32_t* idx = (uint32_t*)scratch(c, 4, sizeof(uint32_t) * ns);
        if (!codes || !idx) return fail(c, PSB_ENOMEM, "scratch allocation failed (sample order)");
        double3 lo = make_double3(c->bbox[0], c->bbox[1], c->bbox[2]);
        double sc[3];
        for (int d = 0; d < 3; ++d) {
            double ext = c->bbox[3 + d] - c->bbox[d];
            sc[d] = ext > 0 ? 2097151.0 / ext : 0.0;
        }
        k_sample_codes<T><<<(unsigned)((ns + 255) / 256), 256, 0, s>>>(S.a[0], S.a[1], S.a[2], ns, lo,
                                                                    make_double3(sc[0], sc[1], sc[2]), codes, idx);
        PSB_CUDA_TRY(c, cudaGetLastError(), "sample code kernel");
        ++launches;
        PSB_CUDA_TRY(c, radix_sort_pairs(codes, idx, ns, c, 6, &launches, false, SAMPLE_KEY_BITS), "sample sort");
        S.order = idx;
    }
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[2], s), "event");

    // ---- outputs ----
    char* obuf = nullptr;
    if (what == WHAT_DIGEST) {
        if (dev) {
            A.dig_count = dcount; A.dig_hash = dhash; A.ha_out = (T*)ha_out;
        } else if (ns > 0) {
            obuf = (char*)scratch(c, 2, (16 + es) * ns);
            if (!obuf) return fail(c, PSB_ENOMEM, "scratch allocation failed (digest)");
            A.dig_count = (int64_t*)obuf;
            A.dig_hash = (uint64_t*)(obuf + 8 * ns);
            A.ha_out = (T*)(obuf + 16 * ns);
        }
    } else if (!adj) {
        if (dev) {
            for (int q = 0; ns > 0 && q < L; ++q) A.out[q] = (T*)out[q];
        } else if (ns > 0 && L > 0) {
            obuf = (char*)scratch(c, 2, es * ns * L);
            if (!obuf) return fail(c, PSB_ENOMEM, "scratch allocation failed (outputs)");
            for (int q = 0; q < L; ++q) A.out[q] = (T*)(obuf + es * ns * q);
        }
    }
    unsigned long long* dstats = (unsigned long long*)scratch(c, 13, 8 * sizeof(unsigned long long));
    if (!dstats) return fail(c, PSB_ENOMEM, "scratch allocation failed (stats)");
    PSB_CUDA_TRY(c, cudaMemsetAsync(dstats, 0, 8 * sizeof(unsigned long long), s), "memset stats");
    A.stats = dstats;

    // ---- launch ----
    if (ns > 0) {
        const bool split = what == WHAT_INTERP && !rq.line && !(flags & PSB_FLAG_SINGLE_KERNEL);
        if (split) {
            int rc = run_split(c, A, prec, st, &launches);
            if (rc) return rc;
        } else {
            if (rq.line && A.src.kind == SRC_BEAM && A.src.ntiles >= 4096) {  // heavy tiles first
                const int64_t nt = A.src.ntiles, nbx = (A.src.nx + 7) >> 3;
                float* cost = (float*)scratch(c, 93, sizeof(float) * nt);
                uint64_t* keys = (uint64_t*)scratch(c, 94, sizeof(uint64_t) * nt);
                uint32_t* vals = (uint32_t*)scratch(c, 95, sizeof(uint32_t) * nt);
                if (!cost || !keys || !vals) return fail(c, PSB_ENOMEM, "scratch allocation failed (tile order)");
                PSB_CUDA_TRY(c, cudaMemsetAsync(cost, 0, sizeof(float) * nt, s), "memset tile costs");
                if (c->n > 0)
                    k_beam_tile_cost<T><<<(unsigned)((c->n + 255) / 256), 256, 0, s>>>(A.tv, A.src, nbx, cost);
                k_cost_keys<<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(cost, nt, keys, vals);
                PSB_CUDA_TRY(c, cudaGetLastError(), "tile cost kernels");
                PSB_CUDA_TRY(c, radix_sort_pairs(keys, vals, nt, c, 6, &launches, false, 32), "tile order sort");
                A.tile_list = (const int32_t*)vals;
                launches += 2;
            }
            cudaError_t e = rq.line ? launch_lines<T>(A, prec, st, A.rec.kc, what, s)
                                    : launch_points<T>(A, prec, st, A.rec.kc, what, s);
            PSB_CUDA_TRY(c, e, "interpolation kernel launch");
            ++launches;
        }
    }
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[3], s), "event");

    // ---- copy back ----
    if (!dev && !adj && ns > 0) {
        if (what == WHAT_DIGEST) {
            PSB_CUDA_TRY(c, cudaMemcpyAsync(dcount, A.dig_count, 8 * ns, cudaMemcpyDeviceToHost, s), "digest D2H");
            PSB_CUDA_TRY(c, cudaMemcpyAsync(dhash, A.dig_hash, 8 * ns, cudaMemcpyDeviceToHost, s), "digest D2H");
            if (ha_out) PSB_CUDA_TRY(c, cudaMemcpyAsync(ha_out, A.ha_out, es * ns, cudaMemcpyDeviceToHost, s), "digest D2H");
        } else {
            for (int q = 0; q < L; ++q)
                PSB_CUDA_TRY(c, cudaMemcpyAsync(out[q], A.out[q], es * ns, cudaMemcpyDeviceToHost, s), "output D2H");
        }
    }
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[4], s), "event");
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
        stats->h2d_ms = ms_between(c->ev[0], c->ev[1]);
        stats->order_ms = ms_between(c->ev[1], c->ev[2]);
        stats->nearest_ms = 0.0;
        stats->interp_ms = ms_between(c->ev[2], c->ev[3]);
        stats->d2h_ms = ms_between(c->ev[3], c->ev[4]);
        stats->total_ms = ms_between(c->ev[0], c->ev[4]);
        stats->pairs = (int64_t)hst[0];
        stats->exact_retests = (int64_t)hst[1];
        stats->warp_steps = (int64_t)hst[2];
        stats->spans = (int64_t)hst[3];
        stats->span_tests = (int64_t)hst[4];
        stats->body_iters = (int64_t)hst[5];
        stats->launches = launches;
    }
    return PSB_OK;
}

// Point samples in host memory, in chunks of PIPE_CHUNK: chunk k+1 is copied
// in on one copy stream and chunk k-1 copied out on another while chunk k
// computes, so a large call costs about max(compute, copies) instead of their
// sum.  Consecutive chunks compute on PIPE_SETS streams, each with its own
// input, output and list buffers, so the kernels of several chunks share the
// GPU and a chunk waits only for the copy-out of the chunk PIPE_SETS before it.
// Each chunk is Morton-ordered on its own.  Buffers are guarded by events.
// (Copies from pageable memory still work, with less overlap.)
constexpr int64_t PIPE_CHUNK = int64_t(1) << 19;
constexpr int PIPE_SETS = 4;

template <class T>
static int run_points_pipelined(psb_ctx* c, const SampleReq& rq, int hmode, const void* hs, int st,
                                const psb_catalog* cat, int prec, void* const* out, uint32_t flags,
                                psb_stats* stats) {
    cudaStream_t s = c->stream;
    const size_t es = sizeof(T);
    const int64_t ns = rq.ns;
    const int64_t CH = PIPE_CHUNK;
    // Chunk k covers samples [cb[k], cb[k+1]).  The first chunk's copy-in and
    // the last one's copy-out overlap no kernel, so the two chunks at each end
    // take a quarter and a half of CH; those between share the rest evenly
    // (at most CH each).  The caller guarantees ns >= 2 CH.
    std::vector<int64_t> cb;
    {
        const int64_t q = CH / 4, h = CH / 2, mid = ns - 2 * (q + h);
        const int64_t nm = (mid + CH - 1) / CH;
        cb.push_back(0);
        cb.push_back(q);
        cb.push_back(q + h);
        for (int64_t i = 1; i <= nm; ++i) cb.push_back(q + h + mid * i / nm);
        cb.push_back(ns - q);
        cb.push_back(ns);
    }
    const int64_t nch = (int64_t)cb.size() - 1;
    int launches = 0;

    Args<T> A;
    memset((void*)&A, 0, sizeof(A));
    std::vector<int> colu;
    int rc = make_recipe(c, cat, false, A.rec, colu);
    if (rc) return rc;
    const int L = A.rec.L;
    if (L > 0 && !out) return fail(c, PSB_EINVAL, "output pointer array must not be NULL");
    for (int k = 0; k < L; ++k)
        if (!out[k]) return fail(c, PSB_EINVAL, "output pointer " + std::to_string(k) + " is NULL");
    const bool need_h = (st != ST_SCATTER) && hmode != PSB_H_NEAREST;
    if (need_h && !hs) return fail(c, PSB_EINVAL, "hs must not be NULL for this strategy and hmode");
    const bool ph = need_h && hmode == PSB_H_PER_SAMPLE;

    for (auto& q : c->cstream)
        if (!q) PSB_CUDA_TRY(c, cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking), "stream");
    for (auto& q : c->pev)
        if (!q) PSB_CUDA_TRY(c, cudaEventCreateWithFlags(&q, cudaEventDisableTiming), "event");
    cudaStream_t sin = c->cstream[0], sout = c->cstream[1];
    const cudaStream_t cs[PIPE_SETS] = {s, c->cstream[2], c->cstream[3], c->cstream[4]};
    // the launch helpers use c->stream: point it at the chunk's compute stream, restore on exit
    struct StreamRestore {
        psb_ctx* c;
        cudaStream_t s;
        ~StreamRestore() { c->stream = s; }
    } restore{c, s};
    cudaEvent_t* in_ready = c->pev;  // [PIPE_SETS] each
    cudaEvent_t* in_free = c->pev + PIPE_SETS;
    cudaEvent_t* done = c->pev + 2 * PIPE_SETS;
    cudaEvent_t* out_free = c->pev + 3 * PIPE_SETS;

    A.tv = tree_view<T>(c);
    A.hmode = hmode;
    A.err = c->d_err;
    A.lut_d = c->lut_d;
    A.lut_f = c->lut_f;
    A.lut_fs = c->lut_fs;
    A.lut_n = (flags & PSB_FLAG_LUT1000_F32) ? LUT_SHORT_N : LUT_N;
    for (size_t q = 0; q < colu.size(); ++q) {
        A.colT[q] = (const T*)c->cols[colu[q]];
        A.colF[q] = (sizeof(T) == 8) ? c->colsf + (size_t)colu[q] * c->n : (const float*)c->cols[colu[q]];
        A.colR[q] = (sizeof(T) == 8) ? c->colsr + (size_t)colu[q] * c->n : nullptr;
    }
    const int nin = 3 + (ph ? 1 : 0);
    char* inb = (char*)scratch(c, 0, es * CH * nin * PIPE_SETS);
    char* outb = (char*)scratch(c, 2, es * CH * (L > 0 ? L : 1) * PIPE_SETS);
    // per set: sample codes and order (slots), the sample sort's scratch
    // (slot base, 7 slots) and the pair lists (slot offset: slots 16-20 + off)
    static const int code_slot[PIPE_SETS] = {3, 35, 53, 55};
    static const int sort_slot[PIPE_SETS] = {6, 38, 64, 72};
    static const int list_off[PIPE_SETS] = {0, 32, 14, 41};
    uint64_t* codes[PIPE_SETS];
    uint32_t* idx[PIPE_SETS];
    for (int b = 0; b < PIPE_SETS; ++b) {
        codes[b] = (uint64_t*)scratch(c, code_slot[b], sizeof(uint64_t) * CH);
        idx[b] = (uint32_t*)scratch(c, code_slot[b] + 1, sizeof(uint32_t) * CH);
        if (!codes[b] || !idx[b]) return fail(c, PSB_ENOMEM, "scratch allocation failed (chunked samples)");
    }
    unsigned long long* dstats = (unsigned long long*)scratch(c, 13, 8 * sizeof(unsigned long long));
    T* hconst = (need_h && !ph) ? (T*)scratch(c, 1, es) : nullptr;
    if (!inb || !outb || !dstats || (need_h && !ph && !hconst))
        return fail(c, PSB_ENOMEM, "scratch allocation failed (chunked samples)");
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[0], s), "event");
    PSB_CUDA_TRY(c, cudaMemsetAsync(dstats, 0, 8 * sizeof(unsigned long long), s), "memset stats");
    if (hconst) PSB_CUDA_TRY(c, cudaMemcpyAsync(hconst, hs, es, cudaMemcpyHostToDevice, s), "hs H2D");
    A.stats = dstats;
    // the copy streams start after everything queued on the compute stream so far
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[1], s), "event");
    PSB_CUDA_TRY(c, cudaStreamWaitEvent(sin, c->ev[1], 0), "stream wait");
    PSB_CUDA_TRY(c, cudaStreamWaitEvent(sout, c->ev[1], 0), "stream wait");
    for (int b = 1; b < PIPE_SETS; ++b) PSB_CUDA_TRY(c, cudaStreamWaitEvent(cs[b], c->ev[1], 0), "stream wait");
    double sc[3];
    for (int d = 0; d < 3; ++d) {
        double ext = c->bbox[3 + d] - c->bbox[d];
        sc[d] = ext > 0 ? 2097151.0 / ext : 0.0;
    }
    const double3 lo3 = make_double3(c->bbox[0], c->bbox[1], c->bbox[2]);
    const double3 sc3 = make_double3(sc[0], sc[1], sc[2]);

    for (int64_t k = 0; k < nch; ++k) {
        const int b = (int)(k % PIPE_SETS);
        const int64_t off = cb[k], cn = cb[k + 1] - cb[k];
        char* ib = inb + es * CH * nin * b;
        // in
        if (k >= PIPE_SETS) PSB_CUDA_TRY(c, cudaStreamWaitEvent(sin, in_free[b], 0), "stream wait");
        for (int q = 0; q < 3; ++q)
            PSB_CUDA_TRY(c, cudaMemcpyAsync(ib + es * CH * q, (const char*)rq.a[q] + es * off, es * cn,
                                            cudaMemcpyHostToDevice, sin), "sample H2D");
        if (ph)
            PSB_CUDA_TRY(c, cudaMemcpyAsync(ib + es * CH * 3, (const char*)hs + es * off, es * cn,
                                            cudaMemcpyHostToDevice, sin), "hs H2D");
        PSB_CUDA_TRY(c, cudaEventRecord(in_ready[b], sin), "event");
        // compute
        const cudaStream_t sc_ = cs[b];
        c->stream = sc_;
        PSB_CUDA_TRY(c, cudaStreamWaitEvent(sc_, in_ready[b], 0), "stream wait");
        if (k >= PIPE_SETS) PSB_CUDA_TRY(c, cudaStreamWaitEvent(sc_, out_free[b], 0), "stream wait");
        SampleSrc<T>& S = A.src;
        S.kind = SRC_ARRAYS;
        S.ns = cn;
        for (int q = 0; q < 3; ++q) S.a[q] = (const T*)(ib + es * CH * q);
        S.ntiles = (cn + 31) / 32;
        S.order = nullptr;
        A.hs = ph ? (const T*)(ib + es * CH * 3) : hconst;
        for (int q = 0; q < L; ++q) A.out[q] = (T*)(outb + es * CH * ((size_t)L * b + q));
        if (cn > 64) {
            k_sample_codes<T><<<(unsigned)((cn + 255) / 256), 256, 0, sc_>>>(S.a[0], S.a[1], S.a[2], cn, lo3, sc3,
                                                                          codes[b], idx[b]);
            PSB_CUDA_TRY(c, cudaGetLastError(), "sample code kernel");
            ++launches;
            PSB_CUDA_TRY(c, radix_sort_pairs(codes[b], idx[b], cn, c, sort_slot[b], &launches, false, SAMPLE_KEY_BITS), "sample sort");
            S.order = idx[b];
        }
        const bool split = !(flags & PSB_FLAG_SINGLE_KERNEL);
        if (split) {
            rc = run_split(c, A, prec, st, &launches, list_off[b], false);  // chunks already overlap
            if (rc) return rc;
        } else {
            PSB_CUDA_TRY(c, launch_points<T>(A, prec, st, A.rec.kc, WHAT_INTERP, sc_), "interpolation kernel launch");
            ++launches;
        }
        PSB_CUDA_TRY(c, cudaEventRecord(in_free[b], sc_), "event");
        PSB_CUDA_TRY(c, cudaEventRecord(done[b], sc_), "event");
        // out
        PSB_CUDA_TRY(c, cudaStreamWaitEvent(sout, done[b], 0), "stream wait");
        for (int q = 0; q < L; ++q)
            PSB_CUDA_TRY(c, cudaMemcpyAsync((char*)out[q] + es * off, A.out[q], es * cn, cudaMemcpyDeviceToHost, sout),
                         "output D2H");
        PSB_CUDA_TRY(c, cudaEventRecord(out_free[b], sout), "event");
    }
    // join the copy streams and the second compute stream back into the compute stream
    c->stream = s;
    PSB_CUDA_TRY(c, cudaStreamWaitEvent(s, out_free[(nch - 1) % PIPE_SETS], 0), "stream wait");
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[4], s), "event");
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
        memset(stats, 0, sizeof(*stats));
        stats->total_ms = ms_between(c->ev[0], c->ev[4]);
        stats->interp_ms = stats->total_ms;
        stats->pairs = (int64_t)hst[0];
        stats->exact_retests = (int64_t)hst[1];
        stats->warp_steps = (int64_t)hst[2];
        stats->spans = (int64_t)hst[3];
        stats->span_tests = (int64_t)hst[4];
        stats->body_iters = (int64_t)hst[5];
        stats->launches = launches;
    }
    return PSB_OK;
}

int run(psb_ctx* c, const SampleReq& rq, int hmode, const void* hs, int st, const psb_catalog* cat, int prec,
        void* const* out, uint32_t flags, psb_stats* stats, int what, int64_t* dcount, uint64_t* dhash, void* ha_out) {
    if (!c->built) return fail(c, PSB_ESTATE, "psb_build_lbvh must run before interpolation");
    if (rq.ns < 0) return fail(c, PSB_EINVAL, "sample count must be non-negative");
    if (st < 0 || st > 2) return fail(c, PSB_EINVAL, "unknown interpolation strategy");
    if (prec < 0 || prec > 1) return fail(c, PSB_EINVAL, "unknown precision mode");
    if (hmode < 0 || hmode > 2) return fail(c, PSB_EINVAL, "unknown smoothing-length mode");
    if (rq.line && st != ST_SCATTER && hmode == PSB_H_NEAREST)
        return fail(c, PSB_EINVAL,
                    "LineSamples_interpolation only supports itpScatter. Line-integrated samples do not have a "
                    "well-defined query smoothing length ha, so itpGather and itpSymmetric are not supported.");
    const bool pipelined = what == WHAT_INTERP && !(flags & PSB_FLAG_DEVICE_PTRS) && rq.kind == SRC_ARRAYS &&
                           !rq.line && !c->adj_lam && rq.ns >= 2 * PIPE_CHUNK;
    if (pipelined)
        return c->dt == PSB_F64 ? run_points_pipelined<double>(c, rq, hmode, hs, st, cat, prec, out, flags, stats)
                                : run_points_pipelined<float>(c, rq, hmode, hs, st, cat, prec, out, flags, stats);
    return c->dt == PSB_F64
               ? run_typed<double>(c, rq, hmode, hs, st, cat, prec, out, flags, stats, what, dcount, dhash, ha_out)
               : run_typed<float>(c, rq, hmode, hs, st, cat, prec, out, flags, stats, what, dcount, dhash, ha_out);
}

}  // namespace psb
