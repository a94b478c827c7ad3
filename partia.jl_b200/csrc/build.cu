// build.cu -- LBVH construction on the device.
//
// Restates LinearBVH!(input) (src/julia/KernelInterpolation/interpolation_setup/InterpolationInput.jl:201-221):
//   1. per-axis min/max and normalisation     MortonEncoding/toolbox.jl:392-405
//   2. 21-bit quantisation + 3D interleave    MortonEncoding/toolbox.jl:224-229,375-383,422-447
//   3. stable sort of (code, index)           MortonEncoding/toolbox.jl:131-137 (sort.cu)
//   4. strictly-increasing dedup              MortonEncoding/toolbox.jl:138-142
//   5. permutation of every particle array    InterpolationInput.jl:205-214
//   6. Karras radix tree                      BinaryRadixTree/toolbox.jl:14-117, BinaryRadixTree.jl:105-109
//   7. escape links (internal, then leaves)   BinaryRadixTree/toolbox.jl:119-156, BinaryRadixTree.jl:111-126
//   8. bottom-up AABB / node-scale refit      LinearBVH/toolbox.jl:36-94, LinearBVH.jl:77-91
// plus the float traversal records used by the FP32C interpolation path.
//
// Step 4 is a sequential recurrence c'_i = max(c_i, c'_{i-1}+1) in the
// reference; it equals c'_i = i + max_{j<=i}(c_j - j), evaluated here as an
// inclusive prefix-max scan in signed 64-bit arithmetic.
#include "psb_ctx.hpp"

namespace psb {

constexpr int BT = 256;  // threads per block of the elementwise build kernels

static inline unsigned grid_for(int64_t n, int threads = BT) {
    int64_t g = (n + threads - 1) / threads;
    return (unsigned)(g < 1 ? 1 : g);
}

// ---- 1. min / max ----------------------------------------------------------
template <class T>
__global__ void k_minmax_partial(const T* x, const T* y, const T* z, int64_t n, T* part) {
    __shared__ T s[6][BT / 32];
    T v[6];
    v[0] = v[3] = x[0]; v[1] = v[4] = y[0]; v[2] = v[5] = z[0];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        T a = x[i], b = y[i], c = z[i];
        v[0] = (a < v[0]) ? a : v[0]; v[1] = (b < v[1]) ? b : v[1]; v[2] = (c < v[2]) ? c : v[2];
        v[3] = (a > v[3]) ? a : v[3]; v[4] = (b > v[4]) ? b : v[4]; v[5] = (c > v[5]) ? c : v[5];
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            T t = __shfl_xor_sync(PSB_FULL, v[k], o);
            v[k] = (k < 3) ? ((t < v[k]) ? t : v[k]) : ((t > v[k]) ? t : v[k]);
        }
    }
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 6; ++k) s[k][threadIdx.x >> 5] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < BT / 32; ++w)
            for (int k = 0; k < 6; ++k) {
                T t = s[k][w];
                v[k] = (k < 3) ? ((t < v[k]) ? t : v[k]) : ((t > v[k]) ? t : v[k]);
            }
        for (int k = 0; k < 6; ++k) part[(int64_t)blockIdx.x * 6 + k] = v[k];
    }
}

// bbox[0..5] = min xyz, max xyz; inv[0..2] = 1/(max-min) (0 marks an
// all-equal axis, which normalises to 0.5).
// One warp: each lane folds a strided share of the block partials, then the
// lanes are folded by shuffles (min and max are exact in any order).
template <class T>
__global__ void k_minmax_final(const T* part, int nparts, T* bbox, T* inv) {
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    T v[6];
    for (int k = 0; k < 6; ++k) v[k] = part[k];
    for (int b = lane; b < nparts; b += 32)
        for (int k = 0; k < 6; ++k) {
            T t = part[(int64_t)b * 6 + k];
            v[k] = (k < 3) ? ((t < v[k]) ? t : v[k]) : ((t > v[k]) ? t : v[k]);
        }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            T t = __shfl_xor_sync(PSB_FULL, v[k], o);
            v[k] = (k < 3) ? ((t < v[k]) ? t : v[k]) : ((t > v[k]) ? t : v[k]);
        }
    }
    if (lane != 0) return;
    for (int k = 0; k < 6; ++k) bbox[k] = v[k];
    for (int d = 0; d < 3; ++d) {
        T dv = X<T>::sub(v[3 + d], v[d]);
        inv[d] = (dv == T(0)) ? T(0) : X<T>::div(T(1), dv);
    }
}

// ---- 2. quantise + encode ------------------------------------------------------
template <class T>
__device__ __forceinline__ uint64_t quantise(T v, T vmin, T inv) {
    const T scale = T(2097151);  // exp2(21) - 1
    T f = (inv == T(0)) ? T(0.5) : X<T>::mul(X<T>::sub(v, vmin), inv);
    return (uint64_t)floor(X<T>::mul(scale, f));
}

template <class T>
__global__ void k_encode(const T* x, const T* y, const T* z, int64_t n, const T* bbox, const T* inv,
                         uint64_t* codes, uint32_t* idx, unsigned* err) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // UInt64(floor(NaN or Inf)) raises InexactError in the reference
    if (!isfinite(x[i]) || !isfinite(y[i]) || !isfinite(z[i])) atomicOr(err, PSB_DERR_INPUT);
    uint64_t ix = quantise(x[i], bbox[0], inv[0]);
    uint64_t iy = quantise(y[i], bbox[1], inv[1]);
    uint64_t iz = quantise(z[i], bbox[2], inv[2]);
    codes[i] = (spread3(ix) << 2) | (spread3(iy) << 1) | spread3(iz);
    idx[i] = (uint32_t)i;
}

// ---- 4. dedup ------------------------------------------------------------------
__global__ void k_dedup_prep(const uint64_t* codes, int64_t n, int64_t* v) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int64_t)codes[i] - i;
}
__global__ void k_dedup_apply(const int64_t* v, int64_t n, uint64_t* codes) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) codes[i] = (uint64_t)v[i] + (uint64_t)i;
}

// ---- 5. permutation -------------------------------------------------------------
template <class T>
__global__ void k_gather(const T* src, const uint32_t* idx, int64_t n, T* dst) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[idx[i]];
}
__global__ void k_order64(const uint32_t* idx, int64_t n, int64_t* order) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) order[i] = (int64_t)idx[i];
}
// a rebuild of arrays an earlier build already permuted: the caller's index of
// new position i is that of old position idx[i]
__global__ void k_compose_order(const uint32_t* idx, int64_t n, const int64_t* prev, int64_t* order) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) order[i] = prev[idx[i]];
}

// ---- 6. Karras radix tree ----------------------------------------------------------
// delta(i, j) with 1-based i, j: MortonEncoding/toolbox.jl:329-336
__device__ __forceinline__ int delta(const uint64_t* c, int64_t i, int64_t j) {
    uint64_t a = c[i - 1], b = c[j - 1];
    if (a == b) return __clzll((long long)((uint64_t)i ^ (uint64_t)j));
    return __clzll((long long)(a ^ b));
}

__global__ void k_karras(const uint64_t* c, int64_t n, int32_t* left, int32_t* right, int32_t* parent,
                         int32_t* range_lo, int32_t* range_hi) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n - 1) return;
    const int64_t i = t + 1;
    // _range_direction
    int64_t dL = (i > 1) ? delta(c, i, i - 1) : -1;
    int64_t dR = (i < n) ? delta(c, i, i + 1) : -1;
    int64_t s = dR - dL;
    int64_t d = (s > 0) ? 1 : ((s < 0) ? -1 : 1);
    // _find_range
    int64_t dmin = (1 <= i - d && i - d <= n) ? delta(c, i, i - d) : -1;
    int64_t lmax = 2;
    while (true) {
        int64_t j = i + lmax * d;
        if (j < 1 || j > n) break;
        if (delta(c, i, j) <= dmin) break;
        lmax *= 2;
    }
    int64_t l = 0;
    for (int64_t tt = lmax >> 1; tt > 0; tt >>= 1) {
        int64_t j = i + (l + tt) * d;
        if (j >= 1 && j <= n && delta(c, i, j) > dmin) l += tt;
    }
    int64_t j = i + l * d;
    int64_t lo = i < j ? i : j, hi = i < j ? j : i;
    range_lo[t] = (int32_t)lo;
    range_hi[t] = (int32_t)hi;
    // _split_position
    int64_t split;
    if (c[lo - 1] == c[hi - 1]) {
        int64_t mid = (lo + hi) >> 1;
        split = mid < lo ? lo : (mid > hi - 1 ? hi - 1 : mid);
    } else {
        int pfl = delta(c, lo, hi);
        split = lo;
        int64_t step = hi - lo;
        while (step > 1) {
            step = (step + 1) >> 1;
            int64_t ns = split + step;
            if (ns < hi && delta(c, lo, ns) > pfl) split = ns;
        }
    }
    // _build_child!
    int64_t li = (split == lo) ? lo + (n - 1) : split;
    int64_t ri = (split + 1 == hi) ? hi + (n - 1) : split + 1;
    left[t] = (int32_t)li;
    right[t] = (int32_t)ri;
    parent[li - 1] = (int32_t)i;
    parent[ri - 1] = (int32_t)i;
}

// ---- 7. escapes -----------------------------------------------------------------
__global__ void k_escape_internal(const uint64_t* c, int64_t n, const int32_t* range_hi, int32_t* escape) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n - 1) return;
    int64_t hi = range_hi[t];
    int32_t e;
    if (hi == n) e = 0;
    else if (hi == n - 1) e = (int32_t)((n - 1) + n);
    else {
        int64_t next = hi + 1;
        // adj[k] = delta(k, k+1) for k < n, adj[n] = typemax(Int32)
        int adj_next = (next < n) ? delta(c, next, next + 1) : 0x7fffffff;
        int adj_prev = delta(c, next - 1, next);
        e = (adj_next < adj_prev) ? (int32_t)((n - 1) + next) : (int32_t)next;
    }
    escape[t] = e;
}

__global__ void k_escape_leaf(int64_t n, const int32_t* parent, const int32_t* left, const int32_t* right,
                              int32_t* escape) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int64_t id = n + k;  // unified leaf id n..2n-1
    int32_t p = parent[id - 1];
    int32_t e;
    if (p == 0) e = 0;
    else if (left[p - 1] == (int32_t)id) e = right[p - 1];
    else e = escape[p - 1];
    escape[id - 1] = e;
}

// ---- 8. refit ("second arrival") ------------------------------------------------
template <class T>
__global__ void k_refit(int64_t n, const int32_t* parent, const int32_t* left, const int32_t* right,
                        const T* lx, const T* ly, const T* lz, const T* lh, unsigned* visited,
                        T* mnx, T* mny, T* mnz, T* mxx, T* mxy, T* mxz, T* nsc, unsigned* err) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int32_t p = parent[n + k - 1];
    int64_t guard = 0;
    while (p != 0) {
        if (++guard > n) { atomicOr(err, PSB_DERR_TRAVERSAL); return; }
        __threadfence();
        unsigned old = atomicAdd(&visited[p - 1], 1u);
        if (old == 0) return;  // first arrival: the sibling finishes this node
        if (old != 1) { atomicOr(err, PSB_DERR_REFIT); return; }
        const int32_t l = left[p - 1], r = right[p - 1];
        const bool ll = l >= (int32_t)n, rl = r >= (int32_t)n;
        // children written by other threads are read from L2 (__ldcg)
        T hl = ll ? lh[l - n] : __ldcg(&nsc[l - 1]);
        T hr = rl ? lh[r - n] : __ldcg(&nsc[r - 1]);
        nsc[p - 1] = (hl > hr) ? hl : hr;
        const T* lc[3] = {lx, ly, lz};
        T* mn[3] = {mnx, mny, mnz};
        T* mx[3] = {mxx, mxy, mxz};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            T lmin = ll ? lc[d][l - n] : __ldcg(&mn[d][l - 1]);
            T rmin = rl ? lc[d][r - n] : __ldcg(&mn[d][r - 1]);
            T lmax = ll ? lc[d][l - n] : __ldcg(&mx[d][l - 1]);
            T rmax = rl ? lc[d][r - n] : __ldcg(&mx[d][r - 1]);
            mn[d][p - 1] = (lmin < rmin) ? lmin : rmin;
            mx[d][p - 1] = (lmax > rmax) ? lmax : rmax;
        }
        p = parent[p - 1];
    }
}

__global__ void k_refit_check(const unsigned* visited, int64_t nint, unsigned* err) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nint && visited[t] != 2u) atomicOr(err, PSB_DERR_REFIT);
}

// (left, escape, range_lo, range_hi) of every internal node in one 16-byte record
__global__ void k_pack_links(int64_t nint, const int32_t* left, const int32_t* escape, const int32_t* rlo,
                             const int32_t* rhi, int4* links) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nint) links[t] = make_int4(left[t], escape[t], rlo[t], rhi[t]);
}

// ---- float traversal records ---------------------------------------------------------
template <class T>
__global__ void k_pack_nodes(int64_t nint, const T* mnx, const T* mny, const T* mnz, const T* mxx, const T* mxy,
                             const T* mxz, const T* nsc, float4* lo, float4* hi) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nint) return;
    float4 a, b;
    if (sizeof(T) == 8) {
        a = make_float4(__double2float_rd((double)mnx[t]), __double2float_rd((double)mny[t]),
                        __double2float_rd((double)mnz[t]), __double2float_ru((double)nsc[t]));
        b = make_float4(__double2float_ru((double)mxx[t]), __double2float_ru((double)mxy[t]),
                        __double2float_ru((double)mxz[t]), 0.f);
    } else {
        a = make_float4((float)mnx[t], (float)mny[t], (float)mnz[t], (float)nsc[t]);
        b = make_float4((float)mxx[t], (float)mxy[t], (float)mxz[t], 0.f);
    }
    lo[t] = a;
    hi[t] = b;
}

// First leaf (0-based) of the span of every leaf: the leaf's highest
// ancestor holding at most SPAN_LEAVES leaves, or the leaf itself when its
// parent holds more.  The traversals hand exactly these subtrees to their
// span handlers, so every span shares one anchor.  Unified ids: leaf i is
// n + i; parent[id - 1] (0 above the root).
__global__ void k_span_roots(int64_t n, const int32_t* parent, const int32_t* rlo, const int32_t* rhi,
                             int32_t* sfirst) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t first = (int32_t)i;
    int32_t p = parent[n + i - 1];
    for (int guard = 0; p > 0 && guard < 2 * SPAN_LEAVES; ++guard) {  // a span is at most 31 levels deep
        const int32_t lo = rlo[p - 1], hi = rhi[p - 1];
        if (hi - lo + 1 > SPAN_LEAVES) break;
        first = lo - 1;
        p = parent[p - 1];
    }
    sfirst[i] = first;
}

// Leaf records.  For double inputs the coordinates are stored relative to the
// first leaf of the leaf's span, so that float differences to a sample carry
// only the rounding of the (small) offset.  For float inputs they are the
// exact coordinates (anchor 0).
template <class T>
__global__ void k_pack_leaves(int64_t n, const T* x, const T* y, const T* z, const T* h, const T* m, const T* rho,
                              const int32_t* sfirst, float4* leaf4, float* mrho, float* mf, float4* leafK,
                              float2* spanb, float sig) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double ax = 0, ay = 0, az = 0;
    if (sizeof(T) == 8) {
        const int32_t a = sfirst[i];
        ax = (double)x[a]; ay = (double)y[a]; az = (double)z[a];
    }
    float4 r;
    if (sizeof(T) == 8) {
        r = make_float4((float)((double)x[i] - ax), (float)((double)y[i] - ay), (float)((double)z[i] - az),
                        (float)(double)h[i]);
    } else {
        r = make_float4((float)x[i], (float)y[i], (float)z[i], (float)h[i]);
    }
    leaf4[i] = r;
    const float mr = (float)((double)m[i] / (double)rho[i]);
    mrho[i] = mr;
    mf[i] = (float)m[i];
    // kernel-weight factors of the float pair bodies
    const float ih = 1.f / r.w;
    const float s3 = sig * ih * ih * ih;  // sig = the kernel's 3D norm
    leafK[i] = make_float4(ih, s3, s3 * ih, mr);
    // span bounds: max |offset|_1 and max h, rounded up (non-negative floats
    // order like their bit patterns); spanb starts at zero
    const float l1 = (fabsf(r.x) + fabsf(r.y) + fabsf(r.z)) * 1.0000005f;
    const float hu = __double2float_ru((double)h[i]);
    atomicMax((int*)&spanb[sfirst[i]].x, __float_as_int(l1));
    atomicMax((int*)&spanb[sfirst[i]].y, __float_as_int(hu));
}

__global__ void k_to_float(const double* src, int64_t n, float* dst) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = (float)src[i];
}

// A column of double inputs relative to the first leaf of each leaf's span,
// rounded once: the FP32C pair sums add a per-span shift to it
// (A[first leaf] - A0 in double, rounded once), so A - A0 carries the
// roundings of the two differences instead of those of A and A0 themselves.
__global__ void k_span_relative(const double* src, const int32_t* sfirst, int64_t n, float* dst) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = __double2float_rn(__dsub_rn(src[i], src[sfirst[i]]));
}

// float copies and span-relative copies of the columns (double inputs)
static int pack_columns(psb_ctx* c, cudaStream_t s) {
    const int64_t n = c->n;
    PSB_CUDA_TRY(c, dgrow_t(c, &c->colsf, sizeof(float) * n * c->ncol), "cudaMalloc float columns");
    PSB_CUDA_TRY(c, dgrow_t(c, &c->colsr, sizeof(float) * n * c->ncol), "cudaMalloc span-relative columns");
    for (int k = 0; k < c->ncol; ++k) {
        k_to_float<<<grid_for(n), BT, 0, s>>>((const double*)c->cols[k], n, c->colsf + (size_t)k * n);
        k_span_relative<<<grid_for(n), BT, 0, s>>>((const double*)c->cols[k], c->sfirst, n,
                                                   c->colsr + (size_t)k * n);
    }
    return PSB_OK;
}

// The mass-dependent parts of the leaf records (m/rho, m and leafK.w), with
// k_pack_leaves' arithmetic: a values-only update leaves them as a full
// build over the same particles would.
template <class T>
__global__ void k_pack_values(int64_t n, const T* m, const T* rho, float* mrho, float* mf, float4* leafK) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float mr = (float)((double)m[i] / (double)rho[i]);
    mrho[i] = mr;
    mf[i] = (float)m[i];
    reinterpret_cast<float*>(leafK + i)[3] = mr;
}

// ---------------------------------------------------------------------------
template <class T>
static int build_typed(psb_ctx* c) {
    const int64_t n = c->n;
    cudaStream_t s = c->stream;
    const size_t es = sizeof(T);
    int launches = 0;
    reset_tree(c);

    // 1. bounding box
    const int nparts = (int)std::min<int64_t>(grid_for(n), 148 * 4);
    T* part = (T*)scratch(c, 0, es * 6 * nparts);
    T* bb = (T*)scratch(c, 1, es * 9);
    if (!part || !bb) return fail(c, PSB_ENOMEM, "scratch allocation failed (bbox)");
    k_minmax_partial<T><<<nparts, BT, 0, s>>>((const T*)c->x, (const T*)c->y, (const T*)c->z, n, part);
    k_minmax_final<T><<<1, 32, 0, s>>>(part, nparts, bb, bb + 6);
    PSB_CUDA_TRY(c, cudaGetLastError(), "bbox kernels");

    // 2. codes
    uint32_t* idx = (uint32_t*)scratch(c, 2, sizeof(uint32_t) * n);
    PSB_CUDA_TRY(c, dgrow_t(c, &c->codes, sizeof(uint64_t) * n), "cudaMalloc codes");
    uint64_t* codes = c->codes;
    if (!idx) return fail(c, PSB_ENOMEM, "scratch allocation failed (index)");
    k_encode<T><<<grid_for(n), BT, 0, s>>>((const T*)c->x, (const T*)c->y, (const T*)c->z, n, bb, bb + 6, codes, idx, c->d_err);
    PSB_CUDA_TRY(c, cudaGetLastError(), "encode kernel");

    // 3. sort
    PSB_CUDA_TRY(c, radix_sort_pairs(codes, idx, n, c, 4, &launches), "radix sort");

    // 4. dedup
    int64_t* dv = (int64_t*)scratch(c, 3, sizeof(int64_t) * n);
    if (!dv) return fail(c, PSB_ENOMEM, "scratch allocation failed (dedup)");
    k_dedup_prep<<<grid_for(n), BT, 0, s>>>(codes, n, dv);
    PSB_CUDA_TRY(c, inclusive_max_scan_i64(dv, n, c, 12), "dedup scan");
    k_dedup_apply<<<grid_for(n), BT, 0, s>>>(dv, n, codes);
    PSB_CUDA_TRY(c, cudaGetLastError(), "dedup kernels");

    // 5. permute particle arrays into Morton order
    // order: the index each Morton position had when psb_set_particles gave
    // the arrays, also across repeated builds of the same (already permuted)
    // device arrays
    PSB_CUDA_TRY(c, dgrow_t(c, &c->order, sizeof(int64_t) * n), "cudaMalloc order");
    if (c->order_fresh) {
        k_order64<<<grid_for(n), BT, 0, s>>>(idx, n, c->order);
    } else {
        int64_t* ord2 = (int64_t*)scratch(c, 3, sizeof(int64_t) * n);  // dedup values are consumed
        if (!ord2) return fail(c, PSB_ENOMEM, "scratch allocation failed (order)");
        k_compose_order<<<grid_for(n), BT, 0, s>>>(idx, n, c->order, ord2);
        PSB_CUDA_TRY(c, cudaMemcpyAsync(c->order, ord2, sizeof(int64_t) * n, cudaMemcpyDeviceToDevice, s), "order copy");
    }
    c->order_fresh = false;
    T* tmp = (T*)scratch(c, 3, es * n);  // dedup values and the order copy are consumed
    if (!tmp) return fail(c, PSB_ENOMEM, "scratch allocation failed (permute)");
    std::vector<void*> arrays = {c->x, c->y, c->z, c->m, c->h, c->rho};
    for (void* col : c->cols) arrays.push_back(col);
    for (void* a : arrays) {
        k_gather<T><<<grid_for(n), BT, 0, s>>>((const T*)a, idx, n, tmp);
        PSB_CUDA_TRY(c, cudaMemcpyAsync(a, tmp, es * n, cudaMemcpyDeviceToDevice, s), "permute copy");
    }
    PSB_CUDA_TRY(c, cudaGetLastError(), "permute kernels");

    // 6-7. tree topology
    const int64_t tot = 2 * n - 1, nint = n - 1;
    PSB_CUDA_TRY(c, dgrow_t(c, &c->left, sizeof(int32_t) * tot), "cudaMalloc left");
    PSB_CUDA_TRY(c, dgrow_t(c, &c->right, sizeof(int32_t) * tot), "cudaMalloc right");
    PSB_CUDA_TRY(c, dgrow_t(c, &c->escape, sizeof(int32_t) * tot), "cudaMalloc escape");
    PSB_CUDA_TRY(c, dgrow_t(c, &c->parent, sizeof(int32_t) * tot), "cudaMalloc parent");
    PSB_CUDA_TRY(c, cudaMemsetAsync(c->left, 0, sizeof(int32_t) * tot, s), "memset");
    PSB_CUDA_TRY(c, cudaMemsetAsync(c->right, 0, sizeof(int32_t) * tot, s), "memset");
    PSB_CUDA_TRY(c, cudaMemsetAsync(c->escape, 0, sizeof(int32_t) * tot, s), "memset");
    PSB_CUDA_TRY(c, cudaMemsetAsync(c->parent, 0, sizeof(int32_t) * tot, s), "memset");
    const int64_t nalloc = nint > 0 ? nint : 1;
    PSB_CUDA_TRY(c, dgrow_t(c, &c->range_lo, sizeof(int32_t) * nalloc), "cudaMalloc range");
    PSB_CUDA_TRY(c, dgrow_t(c, &c->range_hi, sizeof(int32_t) * nalloc), "cudaMalloc range");
    for (int d = 0; d < 3; ++d) {
        PSB_CUDA_TRY(c, dgrow_t(c, &c->nmin[d], es * nalloc), "cudaMalloc node_min");
        PSB_CUDA_TRY(c, dgrow_t(c, &c->nmax[d], es * nalloc), "cudaMalloc node_max");
    }
    PSB_CUDA_TRY(c, dgrow_t(c, &c->nscale, es * nalloc), "cudaMalloc node_scale");
    c->root = (n >= 2) ? 1 : 0;
    if (nint > 0) {
        k_karras<<<grid_for(nint), BT, 0, s>>>(codes, n, c->left, c->right, c->parent, c->range_lo, c->range_hi);
        k_escape_internal<<<grid_for(nint), BT, 0, s>>>(codes, n, c->range_hi, c->escape);
        k_escape_leaf<<<grid_for(n), BT, 0, s>>>(n, c->parent, c->left, c->right, c->escape);
        PSB_CUDA_TRY(c, cudaGetLastError(), "tree kernels");
        // 8. refit
        unsigned* visited = (unsigned*)scratch(c, 2, sizeof(unsigned) * nint);  // index array consumed
        if (!visited) return fail(c, PSB_ENOMEM, "scratch allocation failed (refit)");
        PSB_CUDA_TRY(c, cudaMemsetAsync(visited, 0, sizeof(unsigned) * nint, s), "memset visited");
        k_refit<T><<<grid_for(n), BT, 0, s>>>(n, c->parent, c->left, c->right, (const T*)c->x, (const T*)c->y,
                                              (const T*)c->z, (const T*)c->h, visited, (T*)c->nmin[0],
                                              (T*)c->nmin[1], (T*)c->nmin[2], (T*)c->nmax[0], (T*)c->nmax[1],
                                              (T*)c->nmax[2], (T*)c->nscale, c->d_err);
        k_refit_check<<<grid_for(nint), BT, 0, s>>>(visited, nint, c->d_err);
        PSB_CUDA_TRY(c, cudaGetLastError(), "refit kernels");
    }

    // float traversal records
    PSB_CUDA_TRY(c, dgrow_t(c, &c->links, sizeof(int4) * nalloc), "cudaMalloc links");
    if (nint > 0) k_pack_links<<<grid_for(nint), BT, 0, s>>>(nint, c->left, c->escape, c->range_lo, c->range_hi, c->links);
    PSB_CUDA_TRY(c, dgrow_t(c, &c->node_lo, sizeof(float4) * nalloc), "cudaMalloc node_lo");
    PSB_CUDA_TRY(c, dgrow_t(c, &c->node_hi, sizeof(float4) * nalloc), "cudaMalloc node_hi");
    PSB_CUDA_TRY(c, dgrow_t(c, &c->leaf4, sizeof(float4) * n), "cudaMalloc leaf4");
    PSB_CUDA_TRY(c, dgrow_t(c, &c->mrho, sizeof(float) * n), "cudaMalloc mrho");
    PSB_CUDA_TRY(c, dgrow_t(c, &c->mf, sizeof(float) * n), "cudaMalloc mf");
    PSB_CUDA_TRY(c, dgrow_t(c, &c->leafK, sizeof(float4) * n), "cudaMalloc leafK");
    PSB_CUDA_TRY(c, dgrow_t(c, &c->spanb, sizeof(float2) * n), "cudaMalloc span bounds");
    PSB_CUDA_TRY(c, cudaMemsetAsync(c->spanb, 0, sizeof(float2) * n, s), "memset span bounds");
    if (nint > 0)
        k_pack_nodes<T><<<grid_for(nint), BT, 0, s>>>(nint, (const T*)c->nmin[0], (const T*)c->nmin[1],
                                                      (const T*)c->nmin[2], (const T*)c->nmax[0], (const T*)c->nmax[1],
                                                      (const T*)c->nmax[2], (const T*)c->nscale, c->node_lo, c->node_hi);
    PSB_CUDA_TRY(c, dgrow_t(c, &c->sfirst, sizeof(int32_t) * n), "cudaMalloc span roots");
    int32_t* sfirst = c->sfirst;
    k_span_roots<<<grid_for(n), BT, 0, s>>>(n, c->parent, c->range_lo, c->range_hi, sfirst);
    k_pack_leaves<T><<<grid_for(n), BT, 0, s>>>(n, (const T*)c->x, (const T*)c->y, (const T*)c->z, (const T*)c->h,
                                                (const T*)c->m, (const T*)c->rho, sfirst, c->leaf4, c->mrho, c->mf,
                                                c->leafK, c->spanb, (float)kern_norm3(c->kern));
    if (sizeof(T) == 8 && c->ncol > 0) {
        const int rc = pack_columns(c, s);
        if (rc != PSB_OK) return rc;
    }
    PSB_CUDA_TRY(c, cudaGetLastError(), "pack kernels");

    // bbox to host (used for sample ordering and float error bounds)
    T hb[6];
    PSB_CUDA_TRY(c, cudaMemcpyAsync(hb, bb, es * 6, cudaMemcpyDeviceToHost, s), "bbox copy");
    unsigned herr = 0;
    PSB_CUDA_TRY(c, cudaMemcpyAsync(&herr, c->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, s), "error word copy");
    PSB_CUDA_TRY(c, cudaStreamSynchronize(s), "build synchronize");
    if (herr) {
        cudaMemsetAsync(c->d_err, 0, sizeof(unsigned), s);
        cudaStreamSynchronize(s);
        reset_tree(c);
        if (herr & PSB_DERR_INPUT)
            return fail(c, PSB_EINVAL, "particle coordinates must be finite (NaN or Inf found)");
        if (herr & PSB_DERR_SORT) return device_error(c, herr);
        return fail(c, PSB_ETRAVERSAL, "LBVH refit did not combine every internal node exactly twice");
    }
    double maxabs = 0;
    for (int k = 0; k < 6; ++k) {
        c->bbox[k] = (double)hb[k];
        maxabs = std::max(maxabs, std::fabs((double)hb[k]));
    }
    // |float(v) - v| <= 2^-24 |v|; the node tests allow twice that
    c->coord_err = (float)(maxabs * 1.1920928955078125e-07);
    c->built = true;
    return PSB_OK;
}

template <class T>
static int repack_values_typed(psb_ctx* c) {
    const int64_t n = c->n;
    cudaStream_t s = c->stream;
    k_pack_values<T><<<grid_for(n), BT, 0, s>>>(n, (const T*)c->m, (const T*)c->rho, c->mrho, c->mf, c->leafK);
    if (sizeof(T) == 8 && c->ncol > 0) {
        const int rc = pack_columns(c, s);
        if (rc != PSB_OK) return rc;
    }
    PSB_CUDA_TRY(c, cudaGetLastError(), "value pack kernels");
    return PSB_OK;
}

int repack_values(psb_ctx* c) {
    return c->dt == PSB_F64 ? repack_values_typed<double>(c) : repack_values_typed<float>(c);
}

// Every escape link that ends a traversal (escape 0: the right spine and the
// last leaf) is pointed at the root instead.  Ids stay within 1..2n-1 and the
// ranges are untouched, so every access of a walk stays in bounds; the walks
// simply cycle until their step bound.
__global__ void k_loop_escapes(int64_t n, int4* links, int32_t* escape) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * n - 1) return;
    if (escape[i] == 0) escape[i] = 1;
    if (i < n - 1 && links[i].y == 0) links[i].y = 1;
}

int loop_escapes(psb_ctx* c) {
    if (!c->built) return fail(c, PSB_ESTATE, "psb_build_lbvh must run first");
    if (c->n < 2) return fail(c, PSB_EINVAL, "the LBVH needs at least two particles (a root node)");
    k_loop_escapes<<<grid_for(2 * c->n - 1), BT, 0, c->stream>>>(c->n, c->links, c->escape);
    PSB_CUDA_TRY(c, cudaGetLastError(), "escape kernel");
    PSB_CUDA_TRY(c, cudaStreamSynchronize(c->stream), "synchronize");
    return PSB_OK;
}

int build_lbvh(psb_ctx* c) {
    if (c->n < 1) return fail(c, PSB_EINVAL, "BinaryRadixTree: enc.codes must be non-empty (got n=0).");
    if (c->n > 1073741824ll)
        return fail(c, PSB_EINVAL, "BinaryRadixTree: n exceeds the Int32 node-id capacity (n <= 1073741824).");
    return c->dt == PSB_F64 ? build_typed<double>(c) : build_typed<float>(c);
}

}  // namespace psb
