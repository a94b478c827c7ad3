// capi.cu -- the extern "C" entry points of libpartia_b200 (include/partia_b200.h).
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "psb_host.hpp"

namespace psb {

int fail(psb_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(psb_ctx* c, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    cudaGetLastError();  // clear a sticky launch error where possible
    return fail(c, e == cudaErrorMemoryAllocation ? PSB_ENOMEM : PSB_ECUDA, m);
}

int device_error(psb_ctx* c, unsigned herr) {
    if (herr & PSB_DERR_SORT)
        return fail(c, PSB_ETRAVERSAL, "a radix-sort look-back wait ran out of iterations");
    return fail(c, PSB_ETRAVERSAL, "a traversal exceeded its step bound (corrupt escape links)");
}

void* scratch(psb_ctx* c, int k, size_t bytes) {
    if (k < 0 || k >= (int)(sizeof(c->scratch) / sizeof(c->scratch[0]))) return nullptr;
    auto& sl = c->scratch[k];
    if (sl.bytes >= bytes && sl.p) return sl.p;
    if (sl.p) {
        cudaStreamSynchronize(c->stream);  // the old buffer may still be in use
        cudaFree(sl.p);
        sl.p = nullptr;
        sl.bytes = 0;
    }
    size_t want = bytes < 256 ? 256 : bytes;
    if (cudaMalloc(&sl.p, want) != cudaSuccess) {
        cudaGetLastError();
        sl.p = nullptr;
        return nullptr;
    }
    sl.bytes = want;
    return sl.p;
}

int check_device_ptr(psb_ctx* c, const void* p, const char* what) {
    if (!p) return PSB_OK;
    cudaPointerAttributes at;
    memset(&at, 0, sizeof(at));
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, PSB_EINVAL, std::string(what) + " is not a device pointer (PSB_FLAG_DEVICE_PTRS is set)");
    }
    switch (at.type) {
        case cudaMemoryTypeManaged:
            return PSB_OK;
        case cudaMemoryTypeHost:
            if (at.devicePointer == p) return PSB_OK;
            return fail(c, PSB_EINVAL, std::string(what) + " is page-locked host memory not mapped at the same "
                                                           "device address (PSB_FLAG_DEVICE_PTRS is set)");
        case cudaMemoryTypeDevice:
            if (at.device == c->device) return PSB_OK;
            return fail(c, PSB_EINVAL, std::string(what) + " is memory of device " + std::to_string(at.device) +
                                           ", the context is on device " + std::to_string(c->device));
        default:
            return fail(c, PSB_EINVAL, std::string(what) + " is a pageable host pointer, but PSB_FLAG_DEVICE_PTRS is set");
    }
}

static cudaError_t grow_buf(psb_ctx* c, void*& p, size_t& cap, size_t bytes) {
    if (bytes < 256) bytes = 256;
    if (p && cap >= bytes) return cudaSuccess;
    if (p) {
        cudaStreamSynchronize(c->stream);  // the old buffer may still be in use
        cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    const cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        p = nullptr;
        return e;
    }
    cap = bytes;
    return cudaSuccess;
}

cudaError_t dgrow(psb_ctx* c, void** p, size_t bytes) { return grow_buf(c, *p, c->caps[(const void*)p], bytes); }

void reset_tree(psb_ctx* c) {
    c->built = false;
    c->root = 0;
}

void release_buffers(psb_ctx* c) {
    reset_tree(c);
    for (auto& kv : c->caps) {
        void** p = (void**)kv.first;
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    c->caps.clear();
    for (void*& p : c->colpool)
        if (p) cudaFree(p);
    c->colpool.clear();
    c->colcap.clear();
    c->cols.clear();
    c->n = 0;
}


// Line-integrated kernel tables: I(q) = sigma * 2 * integral over s in
// [0, sqrt(K^2 - q^2)] of f(sqrt(q^2 + s^2)), for the kernel family's shape
// f (kernel_function/kernels/*.jl) and 3D norm sigma, on q_k = K k/(n-1), by
// 64-point Gauss-Legendre quadrature on each smooth piece (split where
// sqrt(q^2+s^2) crosses a break point of f), in long double.  The reference
// tabulates the same integrals at 4096 points over [0, K]
// (table/line_integrated_kernel_tables.jl).
static long double shape_ld(int kid, long double q) {
    switch (kid) {
    case KERN_M5: {
        long double a = 2.5L - q, b = 1.5L - q, c = 0.5L - q;
        if (q < 0.5L) return a * a * a * a - 5 * b * b * b * b + 10 * c * c * c * c;
        if (q < 1.5L) return a * a * a * a - 5 * b * b * b * b;
        return q < 2.5L ? a * a * a * a : 0;
    }
    case KERN_M6: {
        long double a = 3 - q, b = 2 - q, c = 1 - q;
        if (q < 1) return a * a * a * a * a - 6 * b * b * b * b * b + 15 * c * c * c * c * c;
        if (q < 2) return a * a * a * a * a - 6 * b * b * b * b * b;
        return q < 3 ? a * a * a * a * a : 0;
    }
    case KERN_C2: case KERN_C4: case KERN_C6: {
        if (q >= 2) return 0;
        long double a = 1 - 0.5L * q, a2 = a * a;
        if (kid == KERN_C2) return a2 * a2 * (2 * q + 1);
        if (kid == KERN_C4) return a2 * a2 * a2 * (35.0L / 12 * q * q + 3 * q + 1);
        return a2 * a2 * a2 * a2 * (4 * q * q * q + 6.25L * q * q + 4 * q + 1);
    }
    default:
        if (q < 1) { long double a = 2 - q, b = 1 - q; return 0.25L * a * a * a - b * b * b; }
        if (q < 2) { long double a = 2 - q; return 0.25L * a * a * a; }
        return 0;
    }
}

static long double norm3_ld(int kid) {
    const long double pi = 3.141592653589793238462643383279502884L;
    switch (kid) {
    case KERN_M5: return 0.05L / pi;
    case KERN_M6: return 1 / (120 * pi);
    case KERN_C2: return 21 / (16 * pi);
    case KERN_C4: return 495 / (256 * pi);
    case KERN_C6: return 1365 / (512 * pi);
    default: return 1 / pi;
    }
}

void line_table(int kid, double* I, int n) {
    const int G = 64;
    long double gx[G], gw[G];
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int i = 0; i < G; ++i) {
        long double z = std::cos(pi * (i + 0.75L) / (G + 0.5L)), pp = 0;
        for (int it = 0; it < 100; ++it) {
            long double p1 = 1, p2 = 0;
            for (int j = 1; j <= G; ++j) {
                long double p3 = p2;
                p2 = p1;
                p1 = ((2 * j - 1) * z * p2 - (j - 1) * p3) / j;
            }
            pp = G * (z * p1 - p2) / (z * z - 1);
            long double dz = p1 / pp;
            z -= dz;
            if (std::fabs(dz) < 1e-19L) break;
        }
        gx[i] = z;
        gw[i] = 2 / ((1 - z * z) * pp * pp);
    }
    long double brk[3];
    int nb = 0;
    switch (kid) {
    case KERN_M5: brk[0] = 0.5L; brk[1] = 1.5L; brk[2] = 2.5L; nb = 3; break;
    case KERN_M6: brk[0] = 1; brk[1] = 2; brk[2] = 3; nb = 3; break;
    case KERN_C2: case KERN_C4: case KERN_C6: brk[0] = 2; nb = 1; break;
    default: brk[0] = 1; brk[1] = 2; nb = 2; break;
    }
    const long double K = brk[nb - 1], sig = norm3_ld(kid);
    for (int k = 0; k < n; ++k) {
        long double b = K / (n - 1) * k, tot = 0;
        if (b < K) {
            long double edges[4] = {0, 0, 0, 0};
            int ne = 0;
            for (int t = 0; t < nb; ++t)
                if (brk[t] > b) edges[++ne] = std::sqrt(brk[t] * brk[t] - b * b);
            for (int g = 0; g < ne; ++g) {
                long double a = edges[g], e = edges[g + 1];
                for (int i = 0; i < G; ++i) {
                    long double s = 0.5L * (e - a) * gx[i] + 0.5L * (e + a);
                    tot += 0.5L * (e - a) * gw[i] * shape_ld(kid, std::sqrt(b * b + s * s));
                }
            }
            tot *= 2;
        }
        I[k] = (double)(tot * sig);
    }
}

// the kernel family's tables (4096 double, 1000 double), built once per family
struct HostTables {
    double full[LUT_N];
    double shrt[LUT_SHORT_N];
};
static const HostTables& host_line_tables(int kid) {
    static HostTables t[KERN_COUNT];
    static bool ready[KERN_COUNT] = {};
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (!ready[kid]) {
        line_table(kid, t[kid].full, LUT_N);
        line_table(kid, t[kid].shrt, LUT_SHORT_N);
        ready[kid] = true;
    }
    return t[kid];
}

// Upload kernel family kid's line tables (double, float and the short float
// table) to the context, unless they are the ones it holds.
static cudaError_t load_line_tables(psb_ctx* c, int kid) {
    if (c->lut_kern == kid) return cudaSuccess;
    const HostTables& t = host_line_tables(kid);
    std::vector<float> tf(LUT_N), ts(LUT_SHORT_N);
    for (int k = 0; k < LUT_N; ++k) tf[k] = (float)t.full[k];
    for (int k = 0; k < LUT_SHORT_N; ++k) ts[k] = (float)t.shrt[k];
    cudaStreamSynchronize(c->stream);  // a running line kernel may still read the old tables
    cudaError_t e = cudaMemcpy(c->lut_d, t.full, sizeof(double) * LUT_N, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->lut_f, tf.data(), sizeof(float) * LUT_N, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->lut_fs, ts.data(), sizeof(float) * LUT_SHORT_N, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) c->lut_kern = kid;
    return e;
}

}  // namespace psb

using namespace psb;

#define PSB_API extern "C" __attribute__((visibility("default")))

PSB_API int32_t psb_abi_version(void) { return PSB_ABI_VERSION; }

PSB_API int psb_create(psb_ctx** out, int device) {
    if (!out) return PSB_EINVAL;
    *out = nullptr;
    psb_ctx* c = new (std::nothrow) psb_ctx();
    if (!c) return PSB_ENOMEM;
    c->device = device;
    DeviceGuard dg(device);
    cudaError_t e = dg.err;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    for (int k = 0; k < 8 && e == cudaSuccess; ++k) e = cudaEventCreate(&c->ev[k]);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_err, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&c->lut_d, sizeof(double) * LUT_N);
    if (e == cudaSuccess) e = cudaMalloc(&c->lut_f, sizeof(float) * LUT_N);
    if (e == cudaSuccess) e = cudaMalloc(&c->lut_fs, sizeof(float) * LUT_SHORT_N);
    if (e == cudaSuccess) e = load_line_tables(c, KERN_M4);
    if (e != cudaSuccess) {
        cudaGetLastError();
        int code = (e == cudaErrorMemoryAllocation) ? PSB_ENOMEM : PSB_ECUDA;
        psb_destroy(c);
        return code;
    }
    c->stream = c->own_stream;
    *out = c;
    return PSB_OK;
}

PSB_API int psb_destroy(psb_ctx* c) {
    if (!c) return PSB_OK;
    DeviceGuard dg(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    release_buffers(c);
    if (c->sctx) psb_destroy(c->sctx);
    c->sctx = nullptr;
    for (auto& sl : c->scratch) {
        if (sl.p) cudaFree(sl.p);
        sl.p = nullptr;
    }
    if (c->d_err) cudaFree(c->d_err);
    if (c->lut_d) cudaFree(c->lut_d);
    if (c->lut_f) cudaFree(c->lut_f);
    if (c->lut_fs) cudaFree(c->lut_fs);
    for (auto& ev : c->ev)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : c->pev)
        if (ev) cudaEventDestroy(ev);
    for (auto& cs : c->cstream)
        if (cs) cudaStreamDestroy(cs);
    for (auto& ev : c->sev)
        if (ev) cudaEventDestroy(ev);
    for (auto& ss : c->sstream)
        if (ss) cudaStreamDestroy(ss);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return PSB_OK;
}

PSB_API const char* psb_last_error(const psb_ctx* c) {
    if (!c) return "null context";
    return c->err.c_str();
}

PSB_API int psb_set_stream(psb_ctx* c, void* stream) {
    if (!c) return PSB_EINVAL;
    cudaStreamSynchronize(c->stream);
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return PSB_OK;
}

PSB_API int psb_set_particles(psb_ctx* c, int64_t n, psb_dtype dt, const void* x, const void* y, const void* z,
                              const void* m, const void* h, const void* rho, int32_t ncol, const void* const* cols,
                              psb_kernel kernel, uint32_t flags) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    if (n < 0) return fail(c, PSB_EINVAL, "particle count must be non-negative");
    if (dt != PSB_F64 && dt != PSB_F32) return fail(c, PSB_EINVAL, "unknown dtype");
    if (ncol < 0) return fail(c, PSB_EINVAL, "ncol must be non-negative");
    if ((int)kernel < 0 || (int)kernel >= KERN_COUNT) return fail(c, PSB_EINVAL, "unknown kernel");
    if (n > 0 && (!x || !y || !z || !m || !h || !rho)) return fail(c, PSB_EINVAL, "particle arrays must not be NULL");
    if (n > 0 && ncol > 0 && !cols) return fail(c, PSB_EINVAL, "column pointer array must not be NULL");
    for (int k = 0; n > 0 && k < ncol; ++k)
        if (!cols[k]) return fail(c, PSB_EINVAL, "column " + std::to_string(k) + " is NULL");
    DeviceGuard dg(c->device);
    if ((flags & PSB_FLAG_DEVICE_PTRS) && n > 0) {
        int rc = PSB_OK;
        for (const void* p : {x, y, z, m, h, rho})
            if (!rc) rc = check_device_ptr(c, p, "a particle array");
        for (int k = 0; !rc && k < ncol; ++k) rc = check_device_ptr(c, cols[k], "a particle column");
        if (rc) return rc;
    }
    reset_tree(c);
    c->order_fresh = true;
    PSB_CUDA_TRY(c, load_line_tables(c, (int)kernel), "line table upload");
    c->dt = dt;
    c->es = (dt == PSB_F64) ? 8 : 4;
    c->kern = kernel;
    c->n = n;
    c->ncol = ncol;
    const size_t bytes = c->es * (size_t)(n > 0 ? n : 1);
    const cudaMemcpyKind kind = (flags & PSB_FLAG_DEVICE_PTRS) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    void** dst[6] = {&c->x, &c->y, &c->z, &c->m, &c->h, &c->rho};
    const void* src[6] = {x, y, z, m, h, rho};
    for (int k = 0; k < 6; ++k) {
        PSB_CUDA_TRY(c, dgrow(c, dst[k], bytes), "cudaMalloc particles");
        if (n > 0) PSB_CUDA_TRY(c, cudaMemcpyAsync(*dst[k], src[k], c->es * n, kind, c->stream), "particle copy");
    }
    if ((int32_t)c->colpool.size() < ncol) {
        c->colpool.resize(ncol, nullptr);
        c->colcap.resize(ncol, 0);
    }
    c->cols.assign(ncol, nullptr);
    for (int k = 0; k < ncol; ++k) {
        PSB_CUDA_TRY(c, grow_buf(c, c->colpool[k], c->colcap[k], bytes), "cudaMalloc columns");
        c->cols[k] = c->colpool[k];
        if (n > 0) PSB_CUDA_TRY(c, cudaMemcpyAsync(c->cols[k], cols[k], c->es * n, kind, c->stream), "column copy");
    }
    PSB_CUDA_TRY(c, dgrow_t(c, &c->d_cols, sizeof(void*) * (ncol > 0 ? ncol : 1)), "cudaMalloc column table");
    if (ncol > 0)
        PSB_CUDA_TRY(c, cudaMemcpyAsync(c->d_cols, c->cols.data(), sizeof(void*) * ncol, cudaMemcpyHostToDevice, c->stream),
                     "column table copy");
    PSB_CUDA_TRY(c, cudaStreamSynchronize(c->stream), "synchronize");
    return PSB_OK;
}

PSB_API int psb_build_lbvh(psb_ctx* c, int64_t* perm_out, uint64_t* codes_out) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    DeviceGuard dg(c->device);
    int rc = build_lbvh(c);
    if (rc) return rc;
    if (perm_out) PSB_CUDA_TRY(c, cudaMemcpyAsync(perm_out, c->order, sizeof(int64_t) * c->n, cudaMemcpyDeviceToHost, c->stream), "perm D2H");
    if (codes_out) PSB_CUDA_TRY(c, cudaMemcpyAsync(codes_out, c->codes, sizeof(uint64_t) * c->n, cudaMemcpyDeviceToHost, c->stream), "codes D2H");
    PSB_CUDA_TRY(c, cudaStreamSynchronize(c->stream), "synchronize");
    return PSB_OK;
}

PSB_API int psb_set_values(psb_ctx* c, const void* m, const void* rho, int32_t ncol, const void* const* cols,
                           uint32_t flags) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    if (!c->built) return fail(c, PSB_ESTATE, "psb_build_lbvh must run before psb_set_values");
    if (ncol < 0) return fail(c, PSB_EINVAL, "ncol must be non-negative");
    if (!m || !rho) return fail(c, PSB_EINVAL, "mass and density arrays must not be NULL");
    if (ncol > 0 && !cols) return fail(c, PSB_EINVAL, "column pointer array must not be NULL");
    for (int k = 0; k < ncol; ++k)
        if (!cols[k]) return fail(c, PSB_EINVAL, "column " + std::to_string(k) + " is NULL");
    DeviceGuard dg(c->device);
    if (flags & PSB_FLAG_DEVICE_PTRS) {
        int rc = check_device_ptr(c, m, "the mass array");
        if (!rc) rc = check_device_ptr(c, rho, "the density array");
        for (int k = 0; !rc && k < ncol; ++k) rc = check_device_ptr(c, cols[k], "a particle column");
        if (rc) return rc;
    }
    const int64_t n = c->n;
    const size_t bytes = c->es * (size_t)n;
    const cudaMemcpyKind kind = (flags & PSB_FLAG_DEVICE_PTRS) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    PSB_CUDA_TRY(c, cudaMemcpyAsync(c->m, m, bytes, kind, c->stream), "mass copy");
    PSB_CUDA_TRY(c, cudaMemcpyAsync(c->rho, rho, bytes, kind, c->stream), "density copy");
    if ((int32_t)c->colpool.size() < ncol) {
        c->colpool.resize(ncol, nullptr);
        c->colcap.resize(ncol, 0);
    }
    c->cols.assign(ncol, nullptr);
    for (int k = 0; k < ncol; ++k) {
        PSB_CUDA_TRY(c, grow_buf(c, c->colpool[k], c->colcap[k], bytes), "cudaMalloc columns");
        c->cols[k] = c->colpool[k];
        PSB_CUDA_TRY(c, cudaMemcpyAsync(c->cols[k], cols[k], bytes, kind, c->stream), "column copy");
    }
    PSB_CUDA_TRY(c, dgrow_t(c, &c->d_cols, sizeof(void*) * (ncol > 0 ? ncol : 1)), "cudaMalloc column table");
    if (ncol > 0)
        PSB_CUDA_TRY(c, cudaMemcpyAsync(c->d_cols, c->cols.data(), sizeof(void*) * ncol, cudaMemcpyHostToDevice, c->stream),
                     "column table copy");
    c->ncol = ncol;
    int rc = repack_values(c);
    if (rc) return rc;
    PSB_CUDA_TRY(c, cudaStreamSynchronize(c->stream), "synchronize");
    return PSB_OK;
}

PSB_API int psb_test_loop_escapes(psb_ctx* c) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    DeviceGuard dg(c->device);
    return loop_escapes(c);
}

PSB_API int psb_test_adjoint_pool(psb_ctx* c, int64_t blocks, int32_t split) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    if (blocks < 0) return fail(c, PSB_EINVAL, "blocks must be non-negative");
    if (blocks > 0) c->adj_blocks = blocks;
    if (split < 0 || split > 2) return fail(c, PSB_EINVAL, "split must be 0, 1 or 2");
    c->adj_split = split;
    return PSB_OK;
}

PSB_API int psb_get_tree(psb_ctx* c, int32_t* root, int32_t* left, int32_t* right, int32_t* escape, int32_t* parent,
                         double* node_min, double* node_max, double* node_scale) {
    if (!c) return PSB_EINVAL;
    if (!c->built) return fail(c, PSB_ESTATE, "psb_build_lbvh must run first");
    DeviceGuard dg(c->device);
    const int64_t tot = 2 * c->n - 1, nint = c->n - 1;
    if (root) *root = c->root;
    int32_t* src[4] = {c->left, c->right, c->escape, c->parent};
    int32_t* dst[4] = {left, right, escape, parent};
    for (int k = 0; k < 4; ++k)
        if (dst[k]) PSB_CUDA_TRY(c, cudaMemcpyAsync(dst[k], src[k], sizeof(int32_t) * tot, cudaMemcpyDeviceToHost, c->stream), "tree D2H");
    std::vector<char> tmp(c->es * (size_t)(nint > 0 ? nint : 1));
    auto fetch = [&](const void* d, double* h) -> int {
        if (!h || nint <= 0) return PSB_OK;
        PSB_CUDA_TRY(c, cudaMemcpyAsync(tmp.data(), d, c->es * nint, cudaMemcpyDeviceToHost, c->stream), "node D2H");
        PSB_CUDA_TRY(c, cudaStreamSynchronize(c->stream), "synchronize");
        for (int64_t i = 0; i < nint; ++i)
            h[i] = (c->dt == PSB_F64) ? ((const double*)tmp.data())[i] : (double)((const float*)tmp.data())[i];
        return PSB_OK;
    };
    int rc;
    for (int d = 0; d < 3; ++d) {
        if ((rc = fetch(c->nmin[d], node_min ? node_min + d * nint : nullptr))) return rc;
        if ((rc = fetch(c->nmax[d], node_max ? node_max + d * nint : nullptr))) return rc;
    }
    if ((rc = fetch(c->nscale, node_scale))) return rc;
    PSB_CUDA_TRY(c, cudaStreamSynchronize(c->stream), "synchronize");
    return PSB_OK;
}

static SampleReq points_req(int64_t ns, const void* sx, const void* sy, const void* sz) {
    SampleReq r;
    r.kind = SRC_ARRAYS;
    r.ns = ns;
    r.a[0] = sx; r.a[1] = sy; r.a[2] = sz;
    return r;
}

static int check_samples(psb_ctx* c, int64_t ns, const void* a, const void* b, const void* d) {
    if (ns > 0 && (!a || !b || !d)) return fail(c, PSB_EINVAL, "sample arrays must not be NULL");
    return PSB_OK;
}

PSB_API int psb_interp_points(psb_ctx* c, int64_t ns, const void* sx, const void* sy, const void* sz, psb_hmode hmode,
                              const void* hs, psb_strategy strategy, const psb_catalog* cat, psb_precision prec,
                              void* const* out, uint32_t flags, psb_stats* stats) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    DeviceGuard dg(c->device);
    int rc = check_samples(c, ns, sx, sy, sz);
    if (rc) return rc;
    return run(c, points_req(ns, sx, sy, sz), hmode, hs, strategy, cat, prec, out, flags, stats, WHAT_INTERP, nullptr,
               nullptr, nullptr);
}

PSB_API int psb_interp_grid(psb_ctx* c, const void* ax, int64_t nx, const void* ay, int64_t ny, const void* az,
                            int64_t nz, psb_hmode hmode, const void* hs, psb_strategy strategy,
                            const psb_catalog* cat, psb_precision prec, void* const* out, uint32_t flags,
                            psb_stats* stats) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    DeviceGuard dg(c->device);
    if (nx < 0 || ny < 0 || nz < 0) return fail(c, PSB_EINVAL, "grid sizes must be non-negative");
    if ((nx > 0 && !ax) || (ny > 0 && !ay) || (nz > 0 && !az)) return fail(c, PSB_EINVAL, "axis arrays must not be NULL");
    SampleReq r;
    r.kind = SRC_GRID;
    r.ns = nx * ny * nz;
    r.ax = ax; r.ay = ay; r.az = az;
    r.nx = nx; r.ny = ny; r.nz = nz;
    return run(c, r, hmode, hs, strategy, cat, prec, out, flags, stats, WHAT_INTERP, nullptr, nullptr, nullptr);
}

static int check_frame(psb_ctx* c, const void* frame, const void* params, int64_t nx, int64_t ny, int64_t nz, bool box) {
    if (!frame || !params) return fail(c, PSB_EINVAL, "frame and params must not be NULL");
    // _cartesian_plane_coordinates / _cartesian_box_coordinates argument checks
    // (src/julia/Grids/grids/coordinate.jl:37-54,93-110)
    const int na = box ? 3 : 2;
    double p[6];
    for (int k = 0; k < 2 * na; ++k)
        p[k] = (c->dt == PSB_F64) ? ((const double*)params)[k] : (double)((const float*)params)[k];
    const char* nm[3] = {"x", "y", "z"};
    const int64_t nn[3] = {nx, ny, nz};
    for (int k = 0; k < na; ++k) {
        if (!(p[2 * k + 1] > p[2 * k])) return fail(c, PSB_EINVAL, std::string(nm[k]) + "max must be greater than " + nm[k] + "min.");
        if (nn[k] < 2) return fail(c, PSB_EINVAL, std::string("n") + nm[k] + " must be at least 2.");
    }
    return PSB_OK;
}

PSB_API int psb_interp_box(psb_ctx* c, const void* frame, const void* params, int64_t nx, int64_t ny, int64_t nz,
                           psb_hmode hmode, const void* hs, psb_strategy strategy, const psb_catalog* cat,
                           psb_precision prec, void* const* out, uint32_t flags, psb_stats* stats) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    DeviceGuard dg(c->device);
    int rc = check_frame(c, frame, params, nx, ny, nz, true);
    if (rc) return rc;
    SampleReq r;
    r.kind = SRC_BOX;
    r.ns = nx * ny * nz;
    r.frame = frame; r.params = params;
    r.nx = nx; r.ny = ny; r.nz = nz;
    return run(c, r, hmode, hs, strategy, cat, prec, out, flags, stats, WHAT_INTERP, nullptr, nullptr, nullptr);
}

PSB_API int psb_interp_lines(psb_ctx* c, int64_t nl, const void* ox, const void* oy, const void* oz, const void* dx,
                             const void* dy, const void* dz, psb_hmode hmode, const void* hs,
                             psb_strategy strategy, const psb_catalog* cat, psb_precision prec, void* const* out,
                             uint32_t flags, psb_stats* stats) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    DeviceGuard dg(c->device);
    int rc = check_samples(c, nl, ox, oy, oz);
    if (!rc) rc = check_samples(c, nl, dx, dy, dz);
    if (rc) return rc;
    SampleReq r = points_req(nl, ox, oy, oz);
    r.line = true;
    r.a[3] = dx; r.a[4] = dy; r.a[5] = dz;
    return run(c, r, hmode, hs, strategy, cat, prec, out, flags, stats, WHAT_INTERP, nullptr, nullptr, nullptr);
}

PSB_API int psb_interp_beam(psb_ctx* c, const void* frame, const void* params, int64_t nx, int64_t ny,
                            psb_hmode hmode, const void* hs, psb_strategy strategy, const psb_catalog* cat,
                            psb_precision prec, void* const* out, uint32_t flags, psb_stats* stats) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    DeviceGuard dg(c->device);
    int rc = check_frame(c, frame, params, nx, ny, 1, false);
    if (rc) return rc;
    SampleReq r;
    r.kind = SRC_BEAM;
    r.line = true;
    r.ns = nx * ny;
    r.frame = frame; r.params = params;
    r.nx = nx; r.ny = ny; r.nz = 1;
    return run(c, r, hmode, hs, strategy, cat, prec, out, flags, stats, WHAT_INTERP, nullptr, nullptr, nullptr);
}

PSB_API int psb_density(psb_ctx* c, int64_t ns, const void* sx, const void* sy, const void* sz, psb_hmode hmode,
                        const void* hs, psb_strategy strategy, psb_precision prec, void* out, uint32_t flags,
                        psb_stats* stats) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    DeviceGuard dg(c->device);
    int rc = check_samples(c, ns, sx, sy, sz);
    if (rc) return rc;
    void* outs[1] = {out};
    return run(c, points_req(ns, sx, sy, sz), hmode, hs, strategy, nullptr, prec, outs, flags, stats, WHAT_DENSITY,
               nullptr, nullptr, nullptr);
}

PSB_API int psb_neighbor_digest(psb_ctx* c, int32_t kind, int64_t ns, const void* ax, const void* ay, const void* az,
                                const void* dx, const void* dy, const void* dz, psb_hmode hmode, const void* hs,
                                psb_strategy strategy, int64_t* count_out, uint64_t* hash_out, void* ha_out,
                                uint32_t flags) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    DeviceGuard dg(c->device);
    if (kind != 0 && kind != 1) return fail(c, PSB_EINVAL, "kind must be 0 (points) or 1 (lines)");
    int rc = check_samples(c, ns, ax, ay, az);
    if (!rc && kind == 1) rc = check_samples(c, ns, dx, dy, dz);
    if (rc) return rc;
    SampleReq r = points_req(ns, ax, ay, az);
    if (kind == 1) {
        r.line = true;
        r.a[3] = dx; r.a[4] = dy; r.a[5] = dz;
    }
    // The digest follows the FP32C decision path (float tests with double
    // fallback) when flags bit 8 is set, otherwise the exact one.
    int prec = (flags & 0x100u) ? PREC_FP32C : PREC_FP64;
    return run(c, r, hmode, hs, strategy, nullptr, prec, nullptr, flags & PSB_FLAG_DEVICE_PTRS, nullptr, WHAT_DIGEST,
               count_out, hash_out, ha_out);
}

// ---- adjoint --------------------------------------------------------------
namespace psb {
int run_adjoint(psb_ctx* c, const SampleReq& rq, int hmode, const void* hs, int st, const psb_catalog* cat,
                const void* const* gout, double* gm, double* const* gcols, double* gx, double* gy, double* gz,
                uint32_t flags, psb_stats* stats);
}

PSB_API int psb_adjoint_points(psb_ctx* c, int64_t ns, const void* sx, const void* sy, const void* sz,
                               psb_hmode hmode, const void* hs, psb_strategy strategy, const psb_catalog* cat,
                               const void* const* gout, double* gm, double* const* gcols, double* gx, double* gy,
                               double* gz, uint32_t flags, psb_stats* stats) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    DeviceGuard dg(c->device);
    int rc = check_samples(c, ns, sx, sy, sz);
    if (rc) return rc;
    return run_adjoint(c, points_req(ns, sx, sy, sz), hmode, hs, strategy, cat, gout, gm, gcols, gx, gy, gz, flags,
                       stats);
}

PSB_API int psb_adjoint_grid(psb_ctx* c, const void* ax, int64_t nx, const void* ay, int64_t ny, const void* az,
                             int64_t nz, psb_hmode hmode, const void* hs, psb_strategy strategy,
                             const psb_catalog* cat, const void* const* gout, double* gm, double* const* gcols,
                             double* gx, double* gy, double* gz, uint32_t flags, psb_stats* stats) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    DeviceGuard dg(c->device);
    if (nx < 0 || ny < 0 || nz < 0) return fail(c, PSB_EINVAL, "grid sizes must be non-negative");
    if ((nx > 0 && !ax) || (ny > 0 && !ay) || (nz > 0 && !az)) return fail(c, PSB_EINVAL, "axis arrays must not be NULL");
    SampleReq r;
    r.kind = SRC_GRID;
    r.ns = nx * ny * nz;
    r.ax = ax; r.ay = ay; r.az = az;
    r.nx = nx; r.ny = ny; r.nz = nz;
    return run_adjoint(c, r, hmode, hs, strategy, cat, gout, gm, gcols, gx, gy, gz, flags, stats);
}

PSB_API int psb_adjoint_beam(psb_ctx* c, const void* frame, const void* params, int64_t nx, int64_t ny,
                             psb_hmode hmode, const void* hs, psb_strategy strategy, const psb_catalog* cat,
                             const void* const* gout, double* gm, double* const* gcols, double* gx, double* gy,
                             double* gz, uint32_t flags, psb_stats* stats) {
    if (!c) return PSB_EINVAL;
    c->err.clear();
    DeviceGuard dg(c->device);
    int rc = check_frame(c, frame, params, nx, ny, 1, false);
    if (rc) return rc;
    SampleReq r;
    r.kind = SRC_BEAM;
    r.line = true;
    r.ns = nx * ny;
    r.frame = frame; r.params = params;
    r.nx = nx; r.ny = ny; r.nz = 1;
    return run_adjoint(c, r, hmode, hs, strategy, cat, gout, gm, gcols, gx, gy, gz, flags, stats);
}
