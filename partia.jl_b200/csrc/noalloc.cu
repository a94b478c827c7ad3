// noalloc.cu -- point interpolation that allocates no device memory.
//
// Some callers cannot allocate device memory at the time they interpolate:
// a host whose device memory is already held by another framework's caching
// pool (Julia's CUDA.jl, PyTorch), where a cudaMalloc in the middle of its
// step can fail even though the pool has room; a real-time pipeline that
// fixes its memory budget at start-up; and any caller that cannot afford the
// device-wide synchronisation a cudaFree implies when a scratch buffer grows.
// psb_interp_points_noalloc serves them.  It is the
// device-pointer point interpolation of psb_interp_points with one
// difference: the per-call scratch it needs (the Morton ordering of the
// samples and the call's counters) lives in the file-scope device array below
// instead of context-owned buffers that grow with cudaMalloc.
//
// Limits and sharing:
//  * at most PSB_NOALLOC_MAX_SAMPLES samples per call; larger calls are
//    rejected with PSB_EINVAL (split them);
//  * the array (PSB_NOALLOC_SCRATCH_BYTES) is part of the library's device
//    image: every GPU that loads the library holds it until the process exits;
//  * every call on a device uses the same array and leaves its contents
//    behind; the call clears what must start at zero.  Calls whose GPU work
//    overlaps (different streams, different contexts on one device) race on
//    the array and must be serialised by the caller;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) once, with that device current; make that first
//    call before any stream capture begins.  The address is kept with the
//    CUDA context it belongs to: after a cudaDeviceReset the device gets a new
//    context (and a new copy of the array), and the next call looks the
//    address up again instead of handing the kernels a stale one.
// The particles and the LBVH must already be on the device (psb_set_particles
// and psb_build_lbvh allocate; this call does not).
#include <cstring>
#include <mutex>

#include "launch.hpp"
#include "psb_host.hpp"

// The shared scratch of every psb_interp_points_noalloc call on a device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[PSB_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_addr[kMaxDevices] = {};
void* g_noalloc_owner[kMaxDevices] = {};  // the CUDA context each address belongs to

// cuCtxGetCurrent, reached through the runtime so that the library does not
// link the driver library (it must load on machines without a GPU).
typedef int (*ctx_get_current_fn)(void** pctx);
ctx_get_current_fn g_ctx_get_current = nullptr;

// Handle of the CUDA context current on this thread (nullptr if unknown).
void* current_cuda_context() {
    if (!g_ctx_get_current) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            cudaGetLastError();
            return nullptr;
        }
        g_ctx_get_current = (ctx_get_current_fn)fn;
    }
    void* cur = nullptr;
    if (g_ctx_get_current(&cur) != 0) return nullptr;
    return cur;
}

// Device address of g_noalloc_scratch on the current device.  In host code
// the symbol name is only a host-side handle; the address the kernels use is
// looked up once per device with that device current, and again only if the
// device's CUDA context has changed since (cudaDeviceReset).
cudaError_t noalloc_scratch_address(int device, void** out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    void* owner = current_cuda_context();
    if (!g_noalloc_addr[device] || !owner || owner != g_noalloc_owner[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_addr[device] = p;
        // the runtime has made the device's context current by now
        g_noalloc_owner[device] = owner ? owner : current_cuda_context();
    }
    *out = g_noalloc_addr[device];
    return cudaSuccess;
}

inline size_t al256(size_t b) { return (b + 255) & ~size_t(255); }

// Catalog -> output recipe with fixed-size storage (the same mapping as the
// allocating drivers, without a growing column list).
int recipe_fixed(psb_ctx* c, const psb_catalog* cat, psb::Recipe& rec, int colu[psb::MAX_KC]) {
    using namespace psb;
    rec = Recipe();
    if (!cat) return fail(c, PSB_EINVAL, "catalog must not be NULL");
    if (cat->n_scalar < 0 || cat->n_grad < 0 || cat->n_div < 0 || cat->n_curl < 0)
        return fail(c, PSB_EINVAL, "catalog counts must be non-negative");
    const int L = cat->n_scalar + 3 * cat->n_grad + cat->n_div + 3 * cat->n_curl;
    if (L > MAX_OUT) return fail(c, PSB_EUNSUPPORTED, "catalog expands to more than 64 output fields");
    int kc = 0;
    auto col = [&](int slot, int& ci) -> int {
        if (slot < 0 || slot >= c->ncol) return fail(c, PSB_EINVAL, "catalog column slot out of range");
        for (int q = 0; q < kc; ++q)
            if (colu[q] == slot) { ci = q; return PSB_OK; }
        if (kc >= MAX_KC) return fail(c, PSB_EUNSUPPORTED, "catalog references more than 8 distinct columns");
        colu[kc] = slot;
        ci = kc++;
        return PSB_OK;
    };
    int o = 0, ci, cj, ck, rc;
    for (int j = 0; j < cat->n_scalar; ++j) {
        if ((rc = col(cat->scalar_slots[j], ci))) return rc;
        rec.op[o] = OP_SCALAR; rec.a0[o] = (int8_t)ci; rec.a1[o] = (int8_t)(cat->scalar_shepard[j] ? 1 : 0); ++o;
    }
    for (int j = 0; j < cat->n_grad; ++j) {
        if (cat->grad_slots[j] == -1) {
            rec.need_dg = 1;
            for (int d = 0; d < 3; ++d) { rec.op[o] = OP_GRADD; rec.a1[o] = (int8_t)d; ++o; }
        } else {
            if ((rc = col(cat->grad_slots[j], ci))) return rc;
            for (int d = 0; d < 3; ++d) { rec.op[o] = OP_GRADC; rec.a0[o] = (int8_t)ci; rec.a1[o] = (int8_t)d; ++o; }
        }
    }
    for (int j = 0; j < cat->n_div; ++j) {
        if ((rc = col(cat->div_slots[3 * j], ci)) || (rc = col(cat->div_slots[3 * j + 1], cj)) ||
            (rc = col(cat->div_slots[3 * j + 2], ck)))
            return rc;
        rec.op[o] = OP_DIV; rec.a0[o] = (int8_t)ci; rec.a1[o] = (int8_t)cj; rec.a2[o] = (int8_t)ck; ++o;
    }
    for (int j = 0; j < cat->n_curl; ++j) {
        if ((rc = col(cat->curl_slots[3 * j], ci)) || (rc = col(cat->curl_slots[3 * j + 1], cj)) ||
            (rc = col(cat->curl_slots[3 * j + 2], ck)))
            return rc;
        for (int d = 0; d < 3; ++d) {
            rec.op[o] = OP_CURL; rec.a0[o] = (int8_t)ci; rec.a1[o] = (int8_t)cj; rec.a2[o] = (int8_t)ck;
            rec.a3[o] = (int8_t)d; ++o;
        }
    }
    rec.L = L;
    rec.kc = kc;
    return PSB_OK;
}

template <class T>
int noalloc_typed(psb_ctx* c, int64_t ns, const void* sx, const void* sy, const void* sz, int hmode, const void* hs,
                  int st, const psb_catalog* cat, int prec, void* const* out, psb_stats* stats) {
    using namespace psb;
    cudaStream_t s = c->stream;
    Args<T> A;
    memset((void*)&A, 0, sizeof(A));
    int colu[MAX_KC] = {0};
    int rc = recipe_fixed(c, cat, A.rec, colu);
    if (rc) return rc;
    const int L = A.rec.L;
    if (ns > 0) {
        if (!sx || !sy || !sz) return fail(c, PSB_EINVAL, "sample arrays must not be NULL");
        if (L > 0 && !out) return fail(c, PSB_EINVAL, "output pointer array must not be NULL");
        for (int k = 0; k < L; ++k)
            if (!out[k]) return fail(c, PSB_EINVAL, "an output pointer is NULL");
    }
    const bool need_h = (st != ST_SCATTER) && hmode != PSB_H_NEAREST;
    if (need_h && !hs) return fail(c, PSB_EINVAL, "hs must not be NULL for this strategy and hmode");
    if (ns > 0) {  // the kernels dereference these directly
        for (const void* p : {sx, sy, sz})
            if (!rc) rc = check_device_ptr(c, p, "a sample coordinate array");
        if (!rc && need_h) rc = check_device_ptr(c, hs, "hs");
        for (int k = 0; !rc && k < L; ++k) rc = check_device_ptr(c, out[k], "an output array");
        if (rc) return rc;
    }

    // carve the static scratch: counters | sample codes | sample order | sort scratch
    void* base = nullptr;
    cudaError_t e = noalloc_scratch_address(c->device, &base);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaGetSymbolAddress of the no-allocation scratch");
    char* sp = (char*)base;
    unsigned long long* dstats = (unsigned long long*)sp;
    sp += 256;
    uint64_t* codes = (uint64_t*)sp;
    sp += al256(sizeof(uint64_t) * ns);
    uint32_t* idx = (uint32_t*)sp;
    sp += al256(sizeof(uint32_t) * ns);
    const size_t used = (size_t)(sp - (char*)base);
    const size_t sort_bytes = radix_sort_pairs_scratch_bytes(ns);
    if (used + sort_bytes > PSB_NOALLOC_SCRATCH_BYTES)
        return fail(c, PSB_EINVAL, "sample count exceeds the no-allocation scratch; split the call");

    A.tv = tree_view<T>(c);
    A.hmode = hmode;
    A.err = c->d_err;
    A.lut_d = c->lut_d;
    A.lut_f = c->lut_f;
    A.lut_fs = c->lut_fs;
    A.lut_n = LUT_N;
    for (int q = 0; q < A.rec.kc; ++q) {
        A.colT[q] = (const T*)c->cols[colu[q]];
        A.colF[q] = (sizeof(T) == 8) ? c->colsf + (size_t)colu[q] * c->n : (const float*)c->cols[colu[q]];
        A.colR[q] = (sizeof(T) == 8) ? c->colsr + (size_t)colu[q] * c->n : nullptr;
    }
    A.src.kind = SRC_ARRAYS;
    A.src.ns = ns;
    A.src.a[0] = (const T*)sx; A.src.a[1] = (const T*)sy; A.src.a[2] = (const T*)sz;
    A.src.ntiles = (ns + 31) / 32;
    if (need_h) A.hs = (const T*)hs;
    for (int q = 0; ns > 0 && q < L; ++q) A.out[q] = (T*)out[q];
    A.stats = dstats;

    int launches = 0;
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[0], s), "event");
    PSB_CUDA_TRY(c, cudaMemsetAsync(dstats, 0, 8 * sizeof(unsigned long long), s), "clear counters");
    if (ns > 64) {
        double3 lo = make_double3(c->bbox[0], c->bbox[1], c->bbox[2]);
        double scl[3];
        for (int d = 0; d < 3; ++d) {
            double ext = c->bbox[3 + d] - c->bbox[d];
            scl[d] = ext > 0 ? 2097151.0 / ext : 0.0;
        }
        k_sample_codes<T><<<(unsigned)((ns + 255) / 256), 256, 0, s>>>(A.src.a[0], A.src.a[1], A.src.a[2], ns, lo,
                                                                    make_double3(scl[0], scl[1], scl[2]), codes, idx);
        PSB_CUDA_TRY(c, cudaGetLastError(), "sample code kernel");
        ++launches;
        PSB_CUDA_TRY(c, radix_sort_pairs_in(codes, idx, ns, sp, sort_bytes, s, c->d_err, &launches), "sample sort");
        A.src.order = idx;
    }
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[2], s), "event");
    if (ns > 0) {
        PSB_CUDA_TRY(c, launch_points<T>(A, prec, st, A.rec.kc, WHAT_INTERP, s), "interpolation kernel launch");
        ++launches;
    }
    PSB_CUDA_TRY(c, cudaEventRecord(c->ev[3], s), "event");
    unsigned long long hst[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    unsigned herr = 0;
    PSB_CUDA_TRY(c, cudaMemcpyAsync(hst, dstats, sizeof(hst), cudaMemcpyDeviceToHost, s), "counters D2H");
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
        cudaEventElapsedTime(&ms, c->ev[0], c->ev[2]);
        stats->order_ms = ms;
        cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]);
        stats->interp_ms = ms;
        cudaEventElapsedTime(&ms, c->ev[0], c->ev[3]);
        stats->total_ms = ms;
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

}  // namespace

extern "C" __attribute__((visibility("default"))) int psb_interp_points_noalloc(
    psb_ctx* c, int64_t ns, const void* sx, const void* sy, const void* sz, psb_hmode hmode, const void* hs,
    psb_strategy strategy, const psb_catalog* cat, psb_precision prec, void* const* out, psb_stats* stats) {
    using namespace psb;
    if (!c) return PSB_EINVAL;
    c->err.clear();
    if (!c->built) return fail(c, PSB_ESTATE, "psb_build_lbvh must run before interpolation");
    if (ns < 0) return fail(c, PSB_EINVAL, "sample count must be non-negative");
    if (ns > PSB_NOALLOC_MAX_SAMPLES)
        return fail(c, PSB_EINVAL, "psb_interp_points_noalloc takes at most 262144 samples per call; split the call");
    if (strategy < 0 || strategy > 2) return fail(c, PSB_EINVAL, "unknown interpolation strategy");
    if (prec < 0 || prec > 1) return fail(c, PSB_EINVAL, "unknown precision mode");
    if (hmode < 0 || hmode > 2) return fail(c, PSB_EINVAL, "unknown smoothing-length mode");
    DeviceGuard dg(c->device);
    if (dg.err != cudaSuccess) return cuda_fail(c, dg.err, "cudaSetDevice");
    return c->dt == PSB_F64 ? noalloc_typed<double>(c, ns, sx, sy, sz, hmode, hs, strategy, cat, prec, out, stats)
                            : noalloc_typed<float>(c, ns, sx, sy, sz, hmode, hs, strategy, cat, prec, out, stats);
}
