// interp.cuh -- device pieces of the interpolation kernels: sample sources,
// M4 kernel functions, the line-integrated lookup, compensated accumulators
// and the warp-cooperative stackless traversal.
#pragma once

#include "psb_common.cuh"

namespace psb {

enum { PREC_FP64 = 0, PREC_FP32C = 1 };
enum { ST_GATHER = 0, ST_SCATTER = 1, ST_SYMMETRIC = 2 };
enum { SRC_ARRAYS = 0, SRC_GRID = 1, SRC_BOX = 2, SRC_BEAM = 3 };
enum { WHAT_INTERP = 0, WHAT_DENSITY = 1, WHAT_DIGEST = 2 };

constexpr int MAX_OUT = 64;
constexpr int MAX_KC = 8;   // distinct catalog columns per call
constexpr int LUT_N = 4096;
constexpr int LUT_SHORT_N = 1000;  // the optional short float table of line kernels

// Output recipes: each output field is a function of the per-sample sums
// S1 = sum w, G = sum g, Sw[c] = sum A_c w, Sg[c] = sum A_c g,
// Dm = sum m W, Dg = sum m gradW  (w = m/rho W, g = m/rho gradW), which is
// the algebra of general_interpolation.jl:128-214 regrouped.
enum { OP_SCALAR = 0, OP_GRADC = 1, OP_GRADD = 2, OP_DIV = 3, OP_CURL = 4 };
struct Recipe {
    int32_t L;
    int32_t kc;           // distinct columns used
    int32_t need_dg;      // density gradient requested
    int8_t op[MAX_OUT];
    int8_t a0[MAX_OUT], a1[MAX_OUT], a2[MAX_OUT], a3[MAX_OUT];
};

// ---------------------------------------------------------------------------
// Sample sources.  A warp owns one tile of 32 samples; tiles are ordered so
// that the 32 samples of a tile are spatially close.
// ---------------------------------------------------------------------------
template <class T> struct SampleSrc {
    int kind;
    int64_t ns;
    const T* a[6];               // SRC_ARRAYS: x,y,z (points) or ox,oy,oz,dx,dy,dz (lines)
    const uint32_t* order;       // SRC_ARRAYS: Morton order of the samples (nullable)
    const T* ax; const T* ay; const T* az;
    int64_t nx, ny, nz;
    T frame[12];                 // position, right, up, forward
    T params[6];                 // xmin,xmax, ymin,ymax, zmin,zmax
    int64_t ntiles;
};

// sample index of (tile, lane), or -1
template <class T> __device__ __forceinline__ int64_t sample_of(const SampleSrc<T>& s, int64_t tile, int lane) {
    if (s.kind == SRC_ARRAYS) {
        int64_t k = tile * 32 + lane;
        if (k >= s.ns) return -1;
        return s.order ? (int64_t)s.order[k] : k;
    }
    if (s.kind == SRC_BEAM) {  // 8 x 4 pixel tiles
        int64_t nbx = (s.nx + 7) >> 3;
        int64_t bx = tile % nbx, by = tile / nbx;
        int64_t i = bx * 8 + (lane & 7), j = by * 4 + (lane >> 3);
        if (i >= s.nx || j >= s.ny) return -1;
        return i + s.nx * j;
    }
    // 4 x 4 x 2 voxel tiles
    int64_t nbx = (s.nx + 3) >> 2, nby = (s.ny + 3) >> 2;
    int64_t bx = tile % nbx, r = tile / nbx;
    int64_t by = r % nby, bz = r / nby;
    int64_t i = bx * 4 + (lane & 3), j = by * 4 + ((lane >> 2) & 3), k = bz * 2 + (lane >> 4);
    if (i >= s.nx || j >= s.ny || k >= s.nz) return -1;
    return i + s.nx * (j + s.ny * k);
}

// coordinates of sample k (points) or origin + direction (lines)
template <class T> __device__ __forceinline__ void sample_coords(const SampleSrc<T>& s, int64_t k, T p[3], T d[3]) {
    if (s.kind == SRC_ARRAYS) {
        p[0] = s.a[0][k]; p[1] = s.a[1][k]; p[2] = s.a[2][k];
        if (s.a[3]) { d[0] = s.a[3][k]; d[1] = s.a[4][k]; d[2] = s.a[5][k]; }
        return;
    }
    if (s.kind == SRC_GRID) {
        int64_t i = k % s.nx, r = k / s.nx;
        p[0] = s.ax[i]; p[1] = s.ay[r % s.ny]; p[2] = s.az[r / s.ny];
        return;
    }
    // Frame-based Cartesian plane / box, src/julia/Grids/grids/coordinate.jl:37-151:
    // delta = (max - min) / (n - 1); xi = min + (i - 1) * delta;
    // x = x0 + xi * rx + eta * ux [+ zeta * fx], evaluated left to right.
    const T* f = s.frame;
    int64_t i = k % s.nx, r = k / s.nx;
    int64_t j = r % s.ny, l = r / s.ny;
    T dx = X<T>::div(X<T>::sub(s.params[1], s.params[0]), (T)(s.nx - 1));
    T dy = X<T>::div(X<T>::sub(s.params[3], s.params[2]), (T)(s.ny - 1));
    T xi = X<T>::add(s.params[0], X<T>::mul((T)i, dx));
    T eta = X<T>::add(s.params[2], X<T>::mul((T)j, dy));
#pragma unroll
    for (int c = 0; c < 3; ++c)
        p[c] = X<T>::add(X<T>::add(f[c], X<T>::mul(xi, f[3 + c])), X<T>::mul(eta, f[6 + c]));
    if (s.kind == SRC_BOX) {
        T dz = X<T>::div(X<T>::sub(s.params[5], s.params[4]), (T)(s.nz - 1));
        T zeta = X<T>::add(s.params[4], X<T>::mul((T)l, dz));
#pragma unroll
        for (int c = 0; c < 3; ++c) p[c] = X<T>::add(p[c], X<T>::mul(zeta, f[9 + c]));
    } else {  // SRC_BEAM: every direction is the frame forward
        d[0] = f[9]; d[1] = f[10]; d[2] = f[11];
    }
}

// ---------------------------------------------------------------------------
// M4 spline (kernel_function/kernels/M4_spline.jl:13-36; 3D norm 1/pi).
// The fast path evaluates f and f' together from q = r / h.
// ---------------------------------------------------------------------------
template <class C> __device__ __forceinline__ void m4_fdf(C q, C& f, C& df) {
    // inner piece expanded to avoid cancellation at small q:
    //   1/4 (2-q)^3 - (1-q)^3 = 1 + q^2 (3/4 q - 3/2),  its derivative q (9/4 q - 3)
    C a = C(2) - q;
    C a2 = a * a;
    C fo = C(0.25) * a2 * a;      // 1 <= q < 2
    C dfo = C(-0.75) * a2;
    C fi = C(1) + q * q * (C(0.75) * q - C(1.5));
    C dfi = q * (C(2.25) * q - C(3));
    f = (q < C(1)) ? fi : ((q < C(2)) ? fo : C(0));
    df = (q < C(1)) ? dfi : ((q < C(2)) ? dfo : C(0));
}
// M4 f and f' for the float pair sums.  The inner piece (q < 1) comes from
// q in float.  The outer piece, f = a^3 / 4 and f' = -3 a^2 / 4 with
// a = 2 - q, takes a = (4 h^2 - d2) / (h (2 h + r)), with 4 h^2 - d2 formed
// in double from the exact squared separation (num): from the float q alone,
// a would carry an absolute error of a few float ulps, a relative error of
// about 1e-6 at q = 1 that grows without bound towards the support edge,
// where a sample with few neighbours still gets most of its weight.
//
// Every rounding of the float pair terms is written out (__fmul_rn,
// __fmaf_rn, ...), here, in kern_fdf_f32 and in f32c_pair_weights: a product
// and a sum left to the compiler may or may not be contracted into one fused
// multiply-add depending on the code around the inlined call, and the single
// kernel and the pair-sum kernel must give a pair the same bits.
__device__ __forceinline__ void m4_fdf_edge(float q, float r, float num, float hf, float& f, float& df) {
    if (q < 1.f) {
        f = __fmaf_rn(__fmul_rn(q, q), __fmaf_rn(0.75f, q, -1.5f), 1.f);
        df = __fmul_rn(q, __fmaf_rn(2.25f, q, -3.f));
        return;
    }
    const float a = fmaxf(__fdividef(num, __fmul_rn(hf, __fmaf_rn(2.f, hf, r))), 0.f);
    const float a2 = __fmul_rn(a, a);
    f = __fmul_rn(__fmul_rn(0.25f, a2), a);
    df = __fmul_rn(-0.75f, a2);
}

// f, f' of the kernel family: KF = 0 is M4 (its own forms above), KF = 1 any
// other family, selected by kern (warp-uniform).
template <int KF, class C> __device__ __forceinline__ void kfdf(int kern, C q, C& f, C& df) {
    if constexpr (KF == 0) m4_fdf<C>(q, f, df);
    else kern_fdf<C>(kern, q, f, df);
}
// the float pair sums' form: num = K^2 h^2 - d^2 formed in double
template <int KF> __device__ __forceinline__ void kfdf_edge(int kern, float q, float r, float num, float hf, float Kf,
                                                            float& f, float& df) {
    if constexpr (KF == 0) m4_fdf_edge(q, r, num, hf, f, df);
    else kern_fdf_f32(kern, q, r, num, hf, Kf, f, df);
}

// FP32C weights of one pair for the Wendland families (support 2h).  Their
// f and f' carry a = 1 - q/2 to the 4th to 8th power, so a relative error e
// of a becomes 4-8 e in the pair term.  From the float q (rsqrtf, two
// roundings of the separation) a carries up to about 3.5 float ulps near
// q = 1, which put C4 and C6 above 1e-6 of the field maxima.  Here
// t = r / (2 h) is formed in double from the exact squared separation (one
// double rsqrt) and 1/(2h): per sample for h_a, and for h_b the float 1/h_b
// refined by one Newton step against 2 h_b in double.  Then a = 1 - t and
// q = 2 t are each rounded once to float.  A pair outside one h's support
// (accepted for the other h of a symmetric pair) gets a = 0, so f = f' = 0.
template <int ST, class ExactD2, class HbK>
__device__ __forceinline__ void f32c_wendland_weights(int kern, float sa3, float sa4, double ika, float4 K,
                                                      ExactD2 exact_d2, HbK hb_K, float& Wsum, float& csum) {
    const double d2d = exact_d2();
    const double ir = d2d > 0.0 ? rsqrt(d2d) : 0.0;
    const double rd = __dmul_rn(d2d, ir);
    Wsum = 0.f;
    csum = 0.f;
    if (ST != ST_SCATTER) {
        const double t = __dmul_rn(rd, ika);  // r / (2 h_a)
        const float a = fmaxf(__double2float_rn(__dsub_rn(1.0, t)), 0.f);
        float f, df;
        wendland_fdf_f32(kern, __double2float_rn(__dadd_rn(t, t)), a, f, df);
        Wsum = __fmul_rn(sa3, f);
        csum = __fmul_rn(sa4, df);
    }
    if (ST != ST_GATHER) {
        // 1/(2 h_b): the float record's 1/h_b, halved, and one Newton step
        const double hbK = hb_K();
        const double i0 = (double)__fmul_rn(0.5f, K.x);
        const double ikb = __fma_rn(i0, __fma_rn(-hbK, i0, 1.0), i0);
        const double t = __dmul_rn(rd, ikb);  // r / (2 h_b)
        const float a = fmaxf(__double2float_rn(__dsub_rn(1.0, t)), 0.f);
        float f, df;
        wendland_fdf_f32(kern, __double2float_rn(__dadd_rn(t, t)), a, f, df);
        if (ST == ST_SCATTER) {
            Wsum = __fmul_rn(K.y, f);
            csum = __fmul_rn(K.z, df);
        } else {
            Wsum = __fmul_rn(0.5f, __fmaf_rn(K.y, f, Wsum));
            csum = __fmul_rn(0.5f, __fmaf_rn(K.z, df, csum));
        }
    }
    csum = __fmul_rn(csum, __double2float_rn(ir));
}

// The FP32C weights of one pair of a double particle set (both pair-sum
// kernels): d = (dx, dy, dz) is the sample minus the particle in float, ia,
// sa3, sa4 the sample's 1/h, sigma/h^3, sigma/h^4, fa2 = (K h_a)^2, ika =
// 1/(2 h_a) in double (Wendland families only) and haf = h_a; K is the
// particle's leafK record (1/h, sigma/h^3, sigma/h^4, m/rho),
// hbf its h in float.  exact_d2() returns the squared separation in double
// (called only for the outer kernel piece), hb_K() K h_b in double.  Returns
// the weight W (Wsum) and the gradient factor csum (grad W = csum d).
template <int ST, int KF, class ExactD2, class HbK>
__device__ __forceinline__ void f32c_pair_weights(int kern, float Kf, float qe, float dx, float dy, float dz, float ia,
                                                  float sa3, float sa4, double fa2, double ika, float haf,
                                                  float4 K, float hbf, ExactD2 exact_d2, HbK hb_K, float& Wsum,
                                                  float& csum) {
    if constexpr (KF == 1) {
        if (kern >= KERN_C2) {  // warp-uniform
            f32c_wendland_weights<ST>(kern, sa3, sa4, ika, K, exact_d2, hb_K, Wsum, csum);
            return;
        }
    }
    const float d2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
    const float invr = d2 > 0.f ? rsqrtf(d2) : 0.f;
    const float r = __fmul_rn(d2, invr);
    const float qa = (ST != ST_SCATTER) ? __fmul_rn(r, ia) : 0.f;
    const float qb = (ST != ST_GATHER) ? __fmul_rn(r, K.x) : 0.f;
    double d2d = 0.0;
    if (qa >= qe || qb >= qe) d2d = exact_d2();
    Wsum = 0.f;
    csum = 0.f;
    if (ST != ST_SCATTER) {
        float f, df;
        kfdf_edge<KF>(kern, qa, r, (float)__dadd_rn(fa2, -d2d), haf, Kf, f, df);
        Wsum = __fmul_rn(sa3, f);
        csum = __fmul_rn(sa4, df);
    }
    if (ST != ST_GATHER) {
        float f, df;
        const double hbK = qb >= qe ? hb_K() : 0.0;
        kfdf_edge<KF>(kern, qb, r, (float)__fma_rn(hbK, hbK, -d2d), hbf, Kf, f, df);
        if (ST == ST_SCATTER) {
            Wsum = __fmul_rn(K.y, f);
            csum = __fmul_rn(K.z, df);
        } else {
            Wsum = __fmul_rn(0.5f, __fmaf_rn(K.y, f, Wsum));
            csum = __fmul_rn(0.5f, __fmaf_rn(K.z, df, csum));
        }
    }
    csum = __fmul_rn(csum, invr);
}

template <class C> __device__ __forceinline__ C m4_f(C q) {
    C a = C(2) - q, b = C(1) - q;
    C fo = C(0.25) * a * a * a;
    C fi = fo - b * b * b;
    return (q < C(1)) ? fi : ((q < C(2)) ? fo : C(0));
}
template <class C> __device__ __forceinline__ C inv_pi();
template <> __device__ __forceinline__ double inv_pi<double>() { return 0.31830988618379067154; }
template <> __device__ __forceinline__ float inv_pi<float>() { return 0.318309886183790671538f; }

// ---------------------------------------------------------------------------
// Compensated float accumulator (Kahan).  The _rn intrinsics keep the
// compensation exact (no contraction).
// ---------------------------------------------------------------------------
struct KahanF {
    float s, c;
    __device__ __forceinline__ void zero() { s = 0.f; c = 0.f; }
    __device__ __forceinline__ void add(float v) {
        float y = __fsub_rn(v, c);
        float t = __fadd_rn(s, y);
        c = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
    }
    __device__ __forceinline__ double get() const { return (double)s - (double)c; }
};
// FP32C sums of double inputs of the kernel families other than M4
// accumulate A - A0 (A0: the column values of the sample's first accepted
// neighbour) as colR[leaf] + shift, with colR the column relative to the
// first leaf of the leaf's span (k_span_relative) and this shift, A[span's
// first leaf] - A0, formed in double and rounded once.  A - A0 then carries
// the roundings of those two differences, not those of A and A0 themselves,
// which the steeper kernels' gradient sums amplify (M4 keeps the cheaper
// float A - A0).
template <class T>
__device__ __forceinline__ float span_shift(const T* col, int64_t lo, int64_t first) {
    return __double2float_rn(__dsub_rn((double)__ldg(&col[lo]), (double)__ldg(&col[first])));
}

struct PlainD {
    double s;
    __device__ __forceinline__ void zero() { s = 0.0; }
    __device__ __forceinline__ void add(double v) { s += v; }
    __device__ __forceinline__ double get() const { return s; }
};

// ---------------------------------------------------------------------------
// Warp-cooperative stackless DFS over left + escape links
// (LinearBVHTraversalMacros.jl:26-108 and variants).  All lanes walk the same
// node sequence.  A lane that prunes node X waits until the warp reaches
// escape[X], which is exactly the node the lane's own stackless traversal
// would visit next, so every lane sees the same leaves in the same order as
// the reference's per-sample traversal.  The warp descends into X when any
// active lane wants it.  The loop is bounded by 4n+8 steps.
// node_fn(ni) -> true to descend (internal node record ni = id-1);
// leaf_fn(li) -> processes 0-based Morton leaf li.
// ---------------------------------------------------------------------------
template <class NodeFn, class LeafFn>
__device__ __forceinline__ bool warp_traverse(int32_t start, int64_t n, const int32_t* __restrict__ left,
                                              const int32_t* __restrict__ escape, bool lane_valid,
                                              NodeFn node_fn, LeafFn leaf_fn) {
    int32_t node = start;
    int32_t resume = lane_valid ? -1 : 0;
    const int64_t bound = 4 * n + 8;
    int64_t steps = 0;
    const int64_t maxid = 2 * n - 1;
    while (node != 0) {
        // corrupt links (an id outside 1..2n-1) or a cycle end the walk with an error
        if (++steps > bound || node < 0 || (int64_t)node > maxid) return false;
        if (resume == node) resume = -1;
        const bool active = (resume == -1);
        if (node >= n) {
            const int32_t esc = __ldg(&escape[node - 1]);
            if (active) leaf_fn((int64_t)node - n);
            node = esc;
        } else {
            const int32_t ni = node - 1;
            const int32_t esc = __ldg(&escape[ni]);
            bool want = false;
            if (active) {
                if (node_fn(ni)) want = true;
                else resume = esc;
            }
            node = __any_sync(PSB_FULL, want) ? __ldg(&left[ni]) : esc;
        }
        if (__all_sync(PSB_FULL, resume == 0)) break;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Warp-cooperative stackless DFS with leaf spans.  Same walk as
// warp_traverse, but an internal node whose subtree holds at most SPAN leaves
// (a contiguous Morton range [range_lo, range_hi]) is handed to span_fn as a
// whole instead of being descended, and the walk continues at its escape.
// links[ni] = (left, escape, range_lo, range_hi) of internal node ni (1-based
// ids / leaf indices), one 16-byte load per step.  span_fn(lo, cnt, part)
// receives the 0-based first leaf, the leaf count and whether this lane takes
// part; it is called by all 32 lanes (it may use warp-synchronous code).
// For point queries this visits, for every lane, exactly the leaves whose
// inclusion test can succeed: point-box distances are monotone in every
// rounding (a box distance never exceeds the distance to a point inside it),
// so skipping the pruning tests inside a span cannot add or lose a neighbour,
// and leaves are still visited in increasing index (DFS) order.
// ---------------------------------------------------------------------------
constexpr int SPAN = SPAN_LEAVES;

template <class NodeFn, class SpanFn>
__device__ __forceinline__ bool warp_traverse_spans(int32_t start, int64_t n, const int4* __restrict__ links,
                                                    const int32_t* __restrict__ escape, bool lane_valid,
                                                    NodeFn node_fn, SpanFn span_fn, int64_t& steps) {
    int32_t node = start;
    int32_t resume = lane_valid ? -1 : 0;
    // A DFS visits each of the 2n - 1 nodes at most once; the bound (4n + 8
    // steps, capped below 2^32) only ends a walk over a corrupted tree.  32-bit
    // counters and ids keep the per-step bookkeeping short (n <= 2^30).
    const uint32_t bound = (uint32_t)(4 * n + 8 < 0xFFFFFFFFll ? 4 * n + 8 : 0xFFFFFFFFll);
    const uint32_t maxid = (uint32_t)(2 * n - 1);
    const int32_t n32 = (int32_t)n;
    uint32_t k = 0;
    bool ok = true;
    while (node != 0) {
        if (++k >= bound || (uint32_t)node > maxid) { ok = false; break; }
        if (resume == node) resume = -1;
        const bool active = (resume == -1);
        if (node >= n32) {  // a leaf reached directly: a span of one
            const int32_t esc = __ldg(&escape[node - 1]);
            span_fn((int64_t)node - n, 1, active);
            node = esc;
        } else {
            const int32_t ni = node - 1;
            const int4 lk = __ldg(&links[ni]);
            bool want = false;
            if (active) {
                if (node_fn(ni)) want = true;
                else resume = lk.y;
            }
            if (!__any_sync(PSB_FULL, want)) {
                node = lk.y;
            } else {
                const int cnt = lk.w - lk.z + 1;
                if (cnt <= SPAN) {
                    span_fn((int64_t)lk.z - 1, cnt, want);
                    if (want) resume = lk.y;
                    node = lk.y;
                } else {
                    node = lk.x;
                }
            }
        }
        if (__all_sync(PSB_FULL, resume == 0)) break;
    }
    steps += k;
    return ok;
}

}  // namespace psb
