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
// Radix sort: onesweep.  One upsweep pass builds the 256-bin histogram of
// every 8-bit digit of the keys at once (and the OR of key ^ key[0], which
// names the digits on which all keys agree); then one kernel per varying
// digit moves every key to its final place for that digit.  Each CTA of a
// digit pass takes the next tile of RS_TILE keys (an atomic ticket, so tiles
// are taken in order), ranks its keys per digit (stable: warps cover
// consecutive key segments, and __match_any_sync ranks the lanes of a round
// in key order), publishes its per-digit counts, and finds the counts of all
// earlier tiles by decoupled look-back: walking back over the status words of
// earlier tiles, each holding either that tile's own count (flag A) or its
// inclusive prefix (flag P), until a prefix is found.  A tile waits only on
// tiles taken before it, whose CTAs are running, so the wait always ends; it
// is nevertheless bounded, and a wait that runs out sets PSB_DERR_SORT.
// ---------------------------------------------------------------------------
constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;   // 4096 keys per tile
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_WSEG = RS_ITEMS * 32;           // keys per warp segment
constexpr int RS_DIGITS = 8;                     // 8-bit digits of a 64-bit key
constexpr unsigned long long RS_FLAG_A = 1ull << 32;  // status: the tile's own count
constexpr unsigned long long RS_FLAG_P = 2ull << 32;  // status: the inclusive prefix
constexpr long long RS_SPIN_LIMIT = 1ll << 26;

// hist[d * 256 + v]: keys whose digit d is v; *vary |= key ^ key[0]
__global__ void __launch_bounds__(RS_THREADS) k_rs_upsweep(const uint64_t* keys, int64_t n, uint32_t* hist,
                                                           unsigned long long* vary) {
    __shared__ uint32_t h[RS_DIGITS][256];
    __shared__ unsigned long long sv[RS_WARPS];
    for (int t = threadIdx.x; t < RS_DIGITS * 256; t += RS_THREADS) (&h[0][0])[t] = 0;
    __syncthreads();
    const uint64_t k0 = keys[0];
    unsigned long long acc = 0;
    for (int64_t i = (int64_t)blockIdx.x * RS_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * RS_THREADS) {
        const uint64_t k = keys[i];
        acc |= k ^ k0;
#pragma unroll
        for (int d = 0; d < RS_DIGITS; ++d) atomicAdd(&h[d][(k >> (8 * d)) & 255u], 1u);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc |= __shfl_xor_sync(PSB_FULL, acc, o);
    if ((threadIdx.x & 31) == 0) sv[threadIdx.x >> 5] = acc;
    __syncthreads();
    for (int t = threadIdx.x; t < RS_DIGITS * 256; t += RS_THREADS) {
        const uint32_t v = (&h[0][0])[t];
        if (v) atomicAdd(&hist[t], v);
    }
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < RS_WARPS; ++w) t |= sv[w];
        atomicOr(vary, t);
    }
}

__device__ __forceinline__ unsigned long long ld_status(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_status(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// One digit pass.  hist: this digit's 256 bins; status: ntiles x 256 words,
// zero at launch; ticket: zero at launch.
__global__ void __launch_bounds__(RS_THREADS) k_rs_onesweep(const uint64_t* kin, const uint32_t* vin, uint64_t* kout,
                                                            uint32_t* vout, int64_t n, int shift, const uint32_t* hist,
                                                            unsigned long long* status, unsigned* ticket,
                                                            unsigned* err) {
    __shared__ uint32_t wcount[RS_WARPS][256];
    __shared__ uint32_t base[256];     // global position of this tile's first key of each digit value
    __shared__ uint32_t wsum[RS_WARPS];
    __shared__ unsigned s_tile;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    for (int t = threadIdx.x; t < RS_WARPS * 256; t += RS_THREADS) (&wcount[0][0])[t] = 0;
    __syncthreads();
    const unsigned tile = s_tile;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t seg = (int64_t)tile * RS_TILE + (int64_t)w * RS_WSEG;
    uint64_t kk[RS_ITEMS];
    uint32_t vv[RS_ITEMS];
    uint32_t rk[RS_ITEMS];
#pragma unroll
    for (int r = 0; r < RS_ITEMS; ++r) {
        const int64_t i = seg + r * 32 + lane;
        const bool valid = i < n;
        const uint64_t key = valid ? kin[i] : 0ull;
        kk[r] = key;
        vv[r] = valid ? vin[i] : 0u;
        const unsigned d = valid ? (unsigned)((key >> shift) & 255u) : 256u;
        const unsigned peers = __match_any_sync(PSB_FULL, d);
        const unsigned before = __popc(peers & lt);
        const uint32_t basec = valid ? wcount[w][d] : 0u;
        __syncwarp();
        if (valid && before == 0) wcount[w][d] = basec + (uint32_t)__popc(peers);
        __syncwarp();
        rk[r] = basec + before;
    }
    __syncthreads();
    // thread v owns digit value v: the tile's count, the warps' exclusive
    // prefixes, the look-back, and the digit's global start
    const int v = threadIdx.x;
    uint32_t tot = 0;
#pragma unroll
    for (int ww = 0; ww < RS_WARPS; ++ww) {
        const uint32_t t = wcount[ww][v];
        wcount[ww][v] = tot;
        tot += t;
    }
    unsigned long long* my = status + (size_t)tile * 256 + v;
    if (tile == 0) st_status(my, RS_FLAG_P | tot);
    else st_status(my, RS_FLAG_A | tot);
    unsigned long long excl = 0;
    if (tile > 0) {
        long long spins = 0;
        for (int64_t j = (int64_t)tile - 1; j >= 0;) {
            const unsigned long long sw = ld_status(status + (size_t)j * 256 + v);
            const unsigned long long flag = sw & ~0xffffffffull;
            if (flag == 0) {
                if (++spins > RS_SPIN_LIMIT) {  // cannot happen while earlier tiles run; never loop without end
                    atomicOr(err, PSB_DERR_SORT);
                    break;
                }
                continue;
            }
            excl += sw & 0xffffffffull;
            if (flag == RS_FLAG_P) break;
            --j;
        }
        st_status(my, RS_FLAG_P | (excl + tot));
    }
    // exclusive scan of the digit histogram over digit values (the digit's start)
    const uint32_t hv = hist[v];
    uint32_t incl = hv;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(PSB_FULL, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    uint32_t off = 0;
    for (int ww = 0; ww < w; ++ww) off += wsum[ww];
    base[v] = off + incl - hv + (uint32_t)excl;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ITEMS; ++r) {
        const int64_t i = seg + r * 32 + lane;
        if (i < n) {
            const unsigned d = (unsigned)((kk[r] >> shift) & 255u);
            const uint32_t pos = base[d] + wcount[w][d] + rk[r];
            kout[pos] = kk[r];
            vout[pos] = vv[r];
        }
    }
}

namespace {
inline size_t al256(size_t b) { return (b + 255) & ~size_t(255); }

struct SortSpace {
    unsigned long long* vary;   // 8 B
    uint32_t* hist;             // 8 x 256
    unsigned* tickets;          // 8
    unsigned long long* status; // ntiles x 256
    uint64_t* kalt;
    uint32_t* valt;
};

size_t sort_space_bytes(int64_t n, int64_t ntiles) {
    return al256(8) + al256(sizeof(uint32_t) * RS_DIGITS * 256) + al256(sizeof(unsigned) * RS_DIGITS) +
           al256(sizeof(unsigned long long) * 256 * (size_t)ntiles) + al256(sizeof(uint64_t) * n) +
           al256(sizeof(uint32_t) * n);
}

SortSpace carve(char* sp, int64_t n, int64_t ntiles) {
    SortSpace S;
    S.vary = (unsigned long long*)sp;
    sp += al256(8);
    S.hist = (uint32_t*)sp;
    sp += al256(sizeof(uint32_t) * RS_DIGITS * 256);
    S.tickets = (unsigned*)sp;
    sp += al256(sizeof(unsigned) * RS_DIGITS);
    S.status = (unsigned long long*)sp;
    sp += al256(sizeof(unsigned long long) * 256 * (size_t)ntiles);
    S.kalt = (uint64_t*)sp;
    sp += al256(sizeof(uint64_t) * n);
    S.valt = (uint32_t*)sp;
    return S;
}

// The sort on carved space.  skip_constant_digits reads the varying digits
// back (one host synchronisation) and runs only their passes; otherwise all
// eight passes run without a host round trip.
cudaError_t onesweep(uint64_t* keys, uint32_t* vals, int64_t n, const SortSpace& S, cudaStream_t s, unsigned* err,
                     int* launches, bool skip_constant_digits, int key_bits = 64) {
    const int64_t ntiles = (n + RS_TILE - 1) / RS_TILE;
    cudaError_t e;
    // vary | hist | tickets are contiguous: one memset
    if ((e = cudaMemsetAsync(S.vary, 0, (char*)S.status - (char*)S.vary, s)) != cudaSuccess) return e;
    const int grid = (int)std::min<int64_t>((n + RS_THREADS - 1) / RS_THREADS, 148 * 4);
    k_rs_upsweep<<<grid, RS_THREADS, 0, s>>>(keys, n, S.hist, S.vary);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (launches) *launches += 1;
    unsigned long long vary = ~0ull;
    if (skip_constant_digits) {
        if ((e = cudaMemcpyAsync(&vary, S.vary, sizeof(vary), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    }
    uint64_t* ksrc = keys; uint32_t* vsrc = vals;
    uint64_t* kdst = S.kalt; uint32_t* vdst = S.valt;
    for (int d = 0; d < RS_DIGITS && 8 * d < key_bits; ++d) {
        if (((vary >> (8 * d)) & 255ull) == 0) continue;
        if ((e = cudaMemsetAsync(S.status, 0, sizeof(unsigned long long) * 256 * (size_t)ntiles, s)) != cudaSuccess)
            return e;
        k_rs_onesweep<<<(unsigned)ntiles, RS_THREADS, 0, s>>>(ksrc, vsrc, kdst, vdst, n, 8 * d, S.hist + 256 * d,
                                                              S.status, S.tickets + d, err);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (launches) *launches += 1;
        std::swap(ksrc, kdst); std::swap(vsrc, vdst);
    }
    if (ksrc != keys) {
        if ((e = cudaMemcpyAsync(keys, ksrc, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(vals, vsrc, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}
}  // namespace

cudaError_t radix_sort_pairs(uint64_t* keys, uint32_t* vals, int64_t n, psb_ctx* c, int slot_base, int* launches,
                             bool skip_constant_digits, int key_bits) {
    if (n <= 1) return cudaSuccess;
    const int64_t ntiles = (n + RS_TILE - 1) / RS_TILE;
    char* sp = (char*)scratch(c, slot_base, sort_space_bytes(n, ntiles));
    if (!sp) return cudaErrorMemoryAllocation;
    return onesweep(keys, vals, n, carve(sp, n, ntiles), c->stream, c->d_err, launches, skip_constant_digits,
                    key_bits);
}

size_t radix_sort_pairs_scratch_bytes(int64_t n) {
    return sort_space_bytes(n, (n + RS_TILE - 1) / RS_TILE);
}

cudaError_t radix_sort_pairs_in(uint64_t* keys, uint32_t* vals, int64_t n, void* scratch_space, size_t bytes,
                                cudaStream_t s, unsigned* err, int* launches) {
    if (n <= 1) return cudaSuccess;
    if (bytes < radix_sort_pairs_scratch_bytes(n)) return cudaErrorInvalidValue;
    const int64_t ntiles = (n + RS_TILE - 1) / RS_TILE;
    return onesweep(keys, vals, n, carve((char*)scratch_space, n, ntiles), s, err, launches, true);
}

}  // namespace psb
