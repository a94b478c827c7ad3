// sort.cu -- device prefix scans and the stable LSD radix sort of Morton keys.
//
// The sort replaces `sortperm(codes; alg=QuickSort)` of
// LinearBoundingVolumeHierarchy/MortonEncoding/toolbox.jl:131-144.  Julia's
// sortperm compares with the Perm ordering (ties broken by index), so the
// permutation it returns is the stable one; an LSD radix sort seeded with the
// identity permutation produces exactly that permutation.
//
// Layout: 8-bit digits, one pass per digit whose bits vary across the keys.
// Each pass is count -> exclusive scan (digit-major) -> stable scatter.  The
// scatter ranks keys inside a warp with __match_any_sync and orders warps and
// blocks by index, which keeps equal digits in input order.
#include "psb_ctx.hpp"

namespace psb {

// ---------------------------------------------------------------------------
// Block-wide scans (256 threads, 8 items per thread, blocked arrangement).
// ---------------------------------------------------------------------------
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

struct OpSum {
    template <class T> __device__ __forceinline__ T operator()(T a, T b) const { return a + b; }
};
struct OpMax {
    template <class T> __device__ __forceinline__ T operator()(T a, T b) const { return a > b ? a : b; }
};

// Inclusive scan of one value per thread across the block; returns the
// inclusive value and writes the block total to *total.
template <class T, class Op>
__device__ __forceinline__ T block_inclusive(T v, Op op, T* warp_tot, T* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(PSB_FULL, v, o);
        if (lane >= o) v = op(t, v);
    }
    if (lane == 31) warp_tot[wid] = v;
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        T w = (lane < nw) ? warp_tot[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T t = __shfl_up_sync(PSB_FULL, w, o);
            if (lane >= o && lane < nw) w = op(t, w);
        }
        if (lane < nw) warp_tot[lane] = w;
    }
    __syncthreads();
    if (wid > 0) v = op(warp_tot[wid - 1], v);
    if (total) *total = warp_tot[(blockDim.x >> 5) - 1];
    return v;
}

// Tile reduction: partial[b] = op-reduction of tile b.
template <class T, class Op>
__global__ void k_tile_reduce(const T* in, int64_t n, T* partial, Op op, T ident) {
    __shared__ T wt[32];
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    T acc = ident;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        int64_t i = base + (int64_t)k * SCAN_THREADS + threadIdx.x;
        if (i < n) acc = op(acc, in[i]);
    }
    T tot;
    block_inclusive(acc, op, wt, &tot);
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

// Scan each tile with a carry-in from the scanned partials (exclusive scan of
// tile totals).  inclusive=false produces an exclusive scan.
template <class T, class Op>
__global__ void k_tile_scan(const T* in, T* out, int64_t n, const T* carry, Op op, T ident, bool inclusive) {
    __shared__ T sm[SCAN_TILE];
    __shared__ T wt[32];
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        int i = k * SCAN_THREADS + threadIdx.x;
        sm[i] = (base + i < n) ? in[base + i] : ident;
    }
    __syncthreads();
    T v[SCAN_ITEMS];
    T acc = ident;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = sm[threadIdx.x * SCAN_ITEMS + k];
        acc = op(acc, v[k]);
    }
    T incl = block_inclusive(acc, op, wt, (T*)nullptr);
    // exclusive prefix of this thread's items
    T run = __shfl_up_sync(PSB_FULL, incl, 1);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) run = (wid > 0) ? wt[wid - 1] : ident;
    T c = carry ? carry[blockIdx.x] : ident;
    run = op(c, run);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        T nv = op(run, v[k]);
        sm[threadIdx.x * SCAN_ITEMS + k] = inclusive ? nv : run;
        run = nv;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        int i = k * SCAN_THREADS + threadIdx.x;
        if (base + i < n) out[base + i] = sm[i];
    }
}

// Recursive multi-level scan.  Scratch slots slot_base.. hold the partials of
// each level.
template <class T, class Op>
static cudaError_t scan_impl(const T* in, T* out, int64_t n, psb_ctx* c, int slot, Op op, T ident, bool inclusive) {
    if (n <= 0) return cudaSuccess;
    int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nb == 1) {
        k_tile_scan<T, Op><<<1, SCAN_THREADS, 0, c->stream>>>(in, out, n, nullptr, op, ident, inclusive);
        return cudaGetLastError();
    }
    T* part = (T*)scratch(c, slot, sizeof(T) * nb);
    if (!part) return cudaErrorMemoryAllocation;
    k_tile_reduce<T, Op><<<(unsigned)nb, SCAN_THREADS, 0, c->stream>>>(in, n, part, op, ident);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = scan_impl<T, Op>(part, part, nb, c, slot + 1, op, ident, false);
    if (e != cudaSuccess) return e;
    k_tile_scan<T, Op><<<(unsigned)nb, SCAN_THREADS, 0, c->stream>>>(in, out, n, part, op, ident, inclusive);
    return cudaGetLastError();
}

cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, psb_ctx* c, int slot_base) {
    return scan_impl<uint32_t, OpSum>(in, out, n, c, slot_base, OpSum(), 0u, false);
}

cudaError_t inclusive_max_scan_i64(int64_t* data, int64_t n, psb_ctx* c, int slot_base) {
    return scan_impl<long long, OpMax>((const long long*)data, (long long*)data, n, c, slot_base, OpMax(),
                                       (long long)INT64_MIN, true);
}

// ---------------------------------------------------------------------------
// Radix sort.
// ---------------------------------------------------------------------------
constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;   // 4096 keys per block
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_WSEG = RS_ITEMS * 32;           // keys per warp segment

__global__ void k_key_xor_or(const uint64_t* keys, int64_t n, unsigned long long* out) {
    __shared__ unsigned long long s[32];
    uint64_t k0 = keys[0];
    unsigned long long acc = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc |= (keys[i] ^ k0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc |= __shfl_xor_sync(PSB_FULL, acc, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t |= s[w];
        atomicOr(out, t);
    }
}

__global__ void k_rs_count(const uint64_t* keys, int64_t n, int shift, uint32_t* counts, int nblocks) {
    __shared__ uint32_t hist[256];
    for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[d] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * RS_TILE;
#pragma unroll 4
    for (int k = 0; k < RS_ITEMS; ++k) {
        int64_t i = base + (int64_t)k * RS_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&hist[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) counts[(int64_t)d * nblocks + blockIdx.x] = hist[d];
}

__global__ void k_rs_scatter(const uint64_t* kin, const uint32_t* vin, uint64_t* kout, uint32_t* vout, int64_t n,
                             int shift, const uint32_t* offs, int nblocks) {
    __shared__ uint32_t wcount[RS_WARPS][256];
    __shared__ uint32_t boff[256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < 256; d += blockDim.x) {
        boff[d] = offs[(int64_t)d * nblocks + blockIdx.x];
#pragma unroll
        for (int ww = 0; ww < RS_WARPS; ++ww) wcount[ww][d] = 0;
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    const int64_t seg = (int64_t)blockIdx.x * RS_TILE + (int64_t)w * RS_WSEG;
    uint64_t kk[RS_ITEMS];
    uint32_t vv[RS_ITEMS];
    uint32_t rk[RS_ITEMS];
#pragma unroll
    for (int r = 0; r < RS_ITEMS; ++r) {
        int64_t i = seg + r * 32 + lane;
        bool valid = i < n;
        uint64_t key = valid ? kin[i] : 0ull;
        kk[r] = key;
        vv[r] = valid ? vin[i] : 0u;
        unsigned d = valid ? (unsigned)((key >> shift) & 255u) : 256u;
        unsigned peers = __match_any_sync(PSB_FULL, d);
        unsigned before = __popc(peers & lt);
        uint32_t basec = valid ? wcount[w][d] : 0u;
        __syncwarp();
        if (valid && before == 0) wcount[w][d] = basec + (uint32_t)__popc(peers);
        __syncwarp();
        rk[r] = basec + before;
    }
    __syncthreads();
    // exclusive prefix over warps, per digit
    for (int d = threadIdx.x; d < 256; d += blockDim.x) {
        uint32_t run = 0;
#pragma unroll
        for (int ww = 0; ww < RS_WARPS; ++ww) {
            uint32_t t = wcount[ww][d];
            wcount[ww][d] = run;
            run += t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ITEMS; ++r) {
        int64_t i = seg + r * 32 + lane;
        if (i < n) {
            unsigned d = (unsigned)((kk[r] >> shift) & 255u);
            uint32_t pos = boff[d] + wcount[w][d] + rk[r];
            kout[pos] = kk[r];
            vout[pos] = vv[r];
        }
    }
}

cudaError_t radix_sort_pairs(uint64_t* keys, uint32_t* vals, int64_t n, psb_ctx* c, int slot_base, int* launches,
                             bool skip_constant_digits) {
    if (n <= 1) return cudaSuccess;
    cudaError_t e;
    unsigned long long vary = ~0ull;  // every digit sorted: no host round trip
    if (skip_constant_digits) {
        // the digits on which all keys agree, read back once (one host sync)
        unsigned long long* d_or = (unsigned long long*)scratch(c, slot_base, sizeof(unsigned long long));
        if (!d_or) return cudaErrorMemoryAllocation;
        e = cudaMemsetAsync(d_or, 0, sizeof(unsigned long long), c->stream);
        if (e != cudaSuccess) return e;
        int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
        k_key_xor_or<<<grid, 256, 0, c->stream>>>(keys, n, d_or);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        vary = 0;
        if ((e = cudaMemcpyAsync(&vary, d_or, sizeof(vary), cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess) return e;
        if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) return e;
        if (launches) *launches += 1;
    }

    const int nblocks = (int)((n + RS_TILE - 1) / RS_TILE);
    uint64_t* kalt = (uint64_t*)scratch(c, slot_base + 1, sizeof(uint64_t) * n);
    uint32_t* valt = (uint32_t*)scratch(c, slot_base + 2, sizeof(uint32_t) * n);
    uint32_t* cnt = (uint32_t*)scratch(c, slot_base + 3, sizeof(uint32_t) * 256 * (size_t)nblocks);
    if (!kalt || !valt || !cnt) return cudaErrorMemoryAllocation;
    uint64_t* ksrc = keys; uint32_t* vsrc = vals;
    uint64_t* kdst = kalt; uint32_t* vdst = valt;
    for (int shift = 0; shift < 64; shift += 8) {
        if (((vary >> shift) & 255ull) == 0) continue;
        k_rs_count<<<nblocks, RS_THREADS, 0, c->stream>>>(ksrc, n, shift, cnt, nblocks);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = exclusive_scan_u32(cnt, cnt, (int64_t)256 * nblocks, c, slot_base + 4)) != cudaSuccess) return e;
        k_rs_scatter<<<nblocks, RS_THREADS, 0, c->stream>>>(ksrc, vsrc, kdst, vdst, n, shift, cnt, nblocks);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (launches) *launches += 4;
        std::swap(ksrc, kdst); std::swap(vsrc, vdst);
    }
    if (ksrc != keys) {
        if ((e = cudaMemcpyAsync(keys, ksrc, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, c->stream)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(vals, vsrc, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, c->stream)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// ---------------------------------------------------------------------------
// The same sort on caller-provided scratch (no allocation).  Used by the
// no-allocation interpolation entry point; the scratch layout is
//   [vary (8 B) | alternate keys | alternate values | digit counts | scan partials]
// each part 256-byte aligned.
// ---------------------------------------------------------------------------
namespace {
inline size_t al256(size_t b) { return (b + 255) & ~size_t(255); }

size_t scan_partials_bytes(int64_t n) {
    size_t total = 0;
    while (n > SCAN_TILE) {
        n = (n + SCAN_TILE - 1) / SCAN_TILE;
        total += al256(sizeof(uint32_t) * n);
    }
    return total;
}

cudaError_t scan_u32_in(const uint32_t* in, uint32_t* out, int64_t n, char* part_space, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nb == 1) {
        k_tile_scan<uint32_t, OpSum><<<1, SCAN_THREADS, 0, s>>>(in, out, n, nullptr, OpSum(), 0u, false);
        return cudaGetLastError();
    }
    uint32_t* part = (uint32_t*)part_space;
    k_tile_reduce<uint32_t, OpSum><<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, part, OpSum(), 0u);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = scan_u32_in(part, part, nb, part_space + al256(sizeof(uint32_t) * nb), s);
    if (e != cudaSuccess) return e;
    k_tile_scan<uint32_t, OpSum><<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, out, n, part, OpSum(), 0u, false);
    return cudaGetLastError();
}
}  // namespace

size_t radix_sort_pairs_scratch_bytes(int64_t n) {
    const int64_t nblocks = (n + RS_TILE - 1) / RS_TILE;
    return al256(8) + al256(sizeof(uint64_t) * n) + al256(sizeof(uint32_t) * n) +
           al256(sizeof(uint32_t) * 256 * nblocks) + scan_partials_bytes(256 * nblocks);
}

cudaError_t radix_sort_pairs_in(uint64_t* keys, uint32_t* vals, int64_t n, void* scratch_space, size_t bytes,
                                cudaStream_t s, int* launches) {
    if (n <= 1) return cudaSuccess;
    if (bytes < radix_sort_pairs_scratch_bytes(n)) return cudaErrorInvalidValue;
    char* sp = (char*)scratch_space;
    unsigned long long* d_or = (unsigned long long*)sp;
    sp += al256(8);
    uint64_t* kalt = (uint64_t*)sp;
    sp += al256(sizeof(uint64_t) * n);
    uint32_t* valt = (uint32_t*)sp;
    sp += al256(sizeof(uint32_t) * n);
    const int nblocks = (int)((n + RS_TILE - 1) / RS_TILE);
    uint32_t* cnt = (uint32_t*)sp;
    sp += al256(sizeof(uint32_t) * 256 * (size_t)nblocks);
    char* parts = sp;

    cudaError_t e = cudaMemsetAsync(d_or, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    k_key_xor_or<<<grid, 256, 0, s>>>(keys, n, d_or);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    unsigned long long vary = 0;
    if ((e = cudaMemcpyAsync(&vary, d_or, sizeof(vary), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    if (launches) *launches += 1;
    uint64_t* ksrc = keys; uint32_t* vsrc = vals;
    uint64_t* kdst = kalt; uint32_t* vdst = valt;
    for (int shift = 0; shift < 64; shift += 8) {
        if (((vary >> shift) & 255ull) == 0) continue;
        k_rs_count<<<nblocks, RS_THREADS, 0, s>>>(ksrc, n, shift, cnt, nblocks);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = scan_u32_in(cnt, cnt, (int64_t)256 * nblocks, parts, s)) != cudaSuccess) return e;
        k_rs_scatter<<<nblocks, RS_THREADS, 0, s>>>(ksrc, vsrc, kdst, vdst, n, shift, cnt, nblocks);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (launches) *launches += 4;
        std::swap(ksrc, kdst); std::swap(vsrc, vdst);
    }
    if (ksrc != keys) {
        if ((e = cudaMemcpyAsync(keys, ksrc, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(vals, vsrc, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace psb
