// interp.cu -- point and line interpolation kernels (forward path).
//
// Per-sample semantics follow
//   grid_interpolation/kernels/PointSamples_kernel.jl:7-139   (nearest h, output order)
//   single_point_interpolation/kernels/general_interpolation.jl:1-669
//   single_point_interpolation/kernels/scalar_interpolation.jl:1-75 (_density_kernel)
//   line_integrated_interpolation/kernels/line_integrated_scalar_interpolation.jl:76-214
//   LinearBVH/LinearBVHQueries.jl:118-140 (LBVH_find_nearest_h)
// with the traversal of LinearBVH/LinearBVHTraversalMacros.jl:26-953.
//
// Precision modes
//  * exact geometry (double inputs in PSB_PREC_FP64, and every float input):
//    distances, radii and the inclusion test use the reference's operation
//    order with exactly rounded intrinsics, so neighbour sets are identical.
//  * FP32C with double inputs: nodes are tested in float against boxes rounded
//    outward (a conservative superset); a leaf is accepted or rejected in
//    float only when it lies outside an error band around the support
//    radius, otherwise the reference's double test decides.  Neighbour sets
//    are therefore identical too.  Float differences use leaf coordinates
//    relative to the first leaf of their span, so their error is relative to
//    the separation.
#pragma once
#include <type_traits>
#include "interp.cuh"

namespace psb {

// Buffers of the two-kernel point path (one batch of tiles): the collect
// kernel writes, for every sample, its accepted leaves as one entry per span
// (the span's first leaf, a mask over its <= 32 leaves, and the sample's
// position relative to that first leaf, rounded to float from double), and
// its smoothing length; the body kernel reads them.  A tile with a sample of
// more than RCAP entries is marked (cnt = 0xFF for all its lanes) and listed
// in ovf_tiles; the single-kernel path computes those tiles instead.
constexpr int RCAP = 32;
struct SplitBufs {
    float4* ent4;        // [tile][RCAP][32]: (rx, ry, rz, first leaf as int bits)
    uint32_t* emask;     // [tile][RCAP][32]
    float* eshift;       // FP32C sums of double inputs, kernels other than M4, else null:
                         // [tile][RCAP][kc][32], the column shifts A[first leaf] - A0 of each entry
                         // (span_shift)
    uint8_t* cnt;        // [tile][32]
    void* ha;            // [tile][32], element type T
    int32_t* ovf_tiles;  // absolute tile ids
    unsigned* ovf_count;
    int64_t tile0;       // first tile of the batch
    int64_t ntiles;      // tiles in the batch
};

template <class T> struct Args {
    TreeView<T> tv;
    SampleSrc<T> src;
    int hmode;
    const T* hs;
    Recipe rec;
    const T* colT[MAX_KC];
    const float* colF[MAX_KC];
    const float* colR[MAX_KC];  // double inputs: the columns relative to each leaf's span anchor (span_shift)
    T* out[MAX_OUT];
    int64_t* dig_count;
    uint64_t* dig_hash;
    T* ha_out;
    const double* lut_d;
    const float* lut_f;
    const float* lut_fs;  // short float table (LUT_SHORT_N entries), used when lut_n == LUT_SHORT_N
    int lut_n;            // entries of the line table in use
    unsigned* err;
    unsigned long long* stats;  // [0] accepted pairs, [1] exact re-tests, [2] traversal steps
    SplitBufs sp;
    // adjoint (FP64 interpolation only): with lam set, the output stage
    // writes the cotangents of the per-sample sums, from the output
    // cotangents gout[L][ns], to lam[q * lam_stride + k] instead of fields
    const double* const* gout;
    double* lam;
    int64_t lam_stride;
    // single-kernel path over a device list of tiles (nullptr: every tile)
    const int32_t* tile_list;
    const unsigned* tile_count;
    // WHAT_DENSITY: every particle mass taken as 1, the number density
    // sum W of _number_density_kernel (scalar_interpolation.jl:86-166)
    int unit_mass;
};

// ---------------------------------------------------------------------------
// Exact geometry (reference operation order), LinearBVHTraversalMacros.jl:800-953
// ---------------------------------------------------------------------------
template <class T> __device__ __forceinline__ T ex_d2_pp(const T p[3], T x, T y, T z) {
    T s = T(0), d;
    d = X<T>::sub(p[0], x); s = X<T>::add(s, X<T>::mul(d, d));
    d = X<T>::sub(p[1], y); s = X<T>::add(s, X<T>::mul(d, d));
    d = X<T>::sub(p[2], z); s = X<T>::add(s, X<T>::mul(d, d));
    return s;
}

template <class T> __device__ __forceinline__ T ex_d2_pbox(const T p[3], const TreeView<T>& tv, int ni) {
    T s = T(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        T a = __ldg(&tv.nmin[d][ni]), b = __ldg(&tv.nmax[d][ni]);
        T t = p[d] < a ? X<T>::sub(a, p[d]) : (p[d] > b ? X<T>::sub(p[d], b) : T(0));
        s = X<T>::add(s, X<T>::mul(t, t));
    }
    return s;
}

// _squared_distance_line_coords: delta = x - o
template <class T> __device__ __forceinline__ T ex_d2_line(const T o[3], const T m[3], T x, T y, T z) {
    T c[3] = {x, y, z};
    T D2 = T(0), Dm = T(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        T D = X<T>::sub(c[d], o[d]);
        D2 = X<T>::add(D2, X<T>::mul(D, D));
        Dm = X<T>::add(Dm, X<T>::mul(D, m[d]));
    }
    return X<T>::sub(D2, X<T>::mul(Dm, Dm));
}

// _squared_distance_line_aabb_lower_bound (with _line_intersects_aabb)
template <class T> __device__ __forceinline__ T ex_d2_line_box(const T o[3], const T m[3], const TreeView<T>& tv, int ni) {
    T a[3], b[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) { a[d] = __ldg(&tv.nmin[d][ni]); b[d] = __ldg(&tv.nmax[d][ni]); }
    bool hit = true;
    T tmin = -(T)INFINITY, tmax = (T)INFINITY;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (!hit) break;
        if (m[d] == T(0)) {
            if (o[d] < a[d] || o[d] > b[d]) hit = false;
        } else {
            T t0 = X<T>::div(X<T>::sub(a[d], o[d]), m[d]);
            T t1 = X<T>::div(X<T>::sub(b[d], o[d]), m[d]);
            if (t0 > t1) { T tt = t0; t0 = t1; t1 = tt; }
            tmin = jmax(tmin, t0);
            tmax = jmin(tmax, t1);
            if (tmin > tmax) hit = false;
        }
    }
    if (hit) return T(0);
    const T half = T(0.5);
    T c[3], r2 = T(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        c[d] = X<T>::mul(X<T>::add(a[d], b[d]), half);
        T hh = X<T>::mul(X<T>::sub(b[d], a[d]), half);
        r2 = X<T>::add(r2, X<T>::mul(hh, hh));
    }
    // _squared_distance_point_line(center, origin, direction): delta = p - o
    T D2 = T(0), Dm = T(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        T D = X<T>::sub(c[d], o[d]);
        D2 = X<T>::add(D2, X<T>::mul(D, D));
        Dm = X<T>::add(Dm, X<T>::mul(D, m[d]));
    }
    T dc2 = X<T>::sub(D2, X<T>::mul(Dm, Dm));
    if (dc2 <= r2) return T(0);
    T dl = X<T>::sub(X<T>::sqrt(dc2), X<T>::sqrt(r2));
    return X<T>::mul(dl, dl);
}

// radius^2 of a leaf or node: gather (K ha)^2, scatter (K hb)^2, symmetric
// max; K = the kernel's support in units of h (Kvalid * h, then squared:
// LinearBVHTraversalMacros.jl:189,246)
template <int ST, class T> __device__ __forceinline__ T ex_r2(T ra2, T hb, T K) {
    if (ST == ST_GATHER) return ra2;
    T r = X<T>::mul(K, hb);
    T r2 = X<T>::mul(r, r);
    if (ST == ST_SCATTER) return r2;
    return jmax(ra2, r2);
}

// ---------------------------------------------------------------------------
// Conservative float geometry (FP32C with double inputs).
// ---------------------------------------------------------------------------
constexpr float U1 = 1.1920928955078125e-07f;  // 2^-23
constexpr float RELM = 4.76837158203125e-07f;  // 2^-21

// lower bound of the exact squared point-box distance
__device__ __forceinline__ float lb_d2_pbox(const float pf[3], float pem, float4 lo, float4 hi) {
    float tx = fmaxf(fmaxf(lo.x - pf[0], pf[0] - hi.x), 0.f);
    float ty = fmaxf(fmaxf(lo.y - pf[1], pf[1] - hi.y), 0.f);
    float tz = fmaxf(fmaxf(lo.z - pf[2], pf[2] - hi.z), 0.f);
    tx = fmaxf(tx * (1.f - 2.f * U1) - pem, 0.f);
    ty = fmaxf(ty * (1.f - 2.f * U1) - pem, 0.f);
    tz = fmaxf(tz * (1.f - 2.f * U1) - pem, 0.f);
    return (tx * tx + ty * ty + tz * tz) * (1.f - RELM);
}

// upper bound of the node radius^2 (node scale is rounded up; K = support)
template <int ST> __device__ __forceinline__ float hi_r2_node(float ra2_hi, float scale_up, float Kf) {
    if (ST == ST_GATHER) return ra2_hi;
    float r = Kf * scale_up;
    float r2 = r * r * (1.f + 2.f * RELM);
    if (ST == ST_SCATTER) return r2;
    return fmaxf(ra2_hi, r2);
}

// lower bound of the squared distance between a line and a node box.
// o, m: float line; el: absolute error allowance of the float line near the
// box (origin and direction rounding).
__device__ __forceinline__ float lb_d2_line_box(const float o[3], const float m[3], float el, float4 lo, float4 hi) {
    float a[3] = {lo.x, lo.y, lo.z}, b[3] = {hi.x, hi.y, hi.z};
    // centre / half-diagonal of the outward-rounded box
    float c[3], r2 = 0.f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        c[d] = 0.5f * (a[d] + b[d]);
        float hh = 0.5f * (b[d] - a[d]);
        r2 += hh * hh;
    }
    float rb = sqrtf(r2) * (1.f + 4.f * U1);
    float v[3], vm = 0.f, vv = 0.f;
#pragma unroll
    for (int d = 0; d < 3; ++d) { v[d] = c[d] - o[d]; vm += v[d] * m[d]; }
    float pp = 0.f;
#pragma unroll
    for (int d = 0; d < 3; ++d) { float w = v[d] - vm * m[d]; pp += w * w; vv += v[d] * v[d]; }
    float dc = sqrtf(pp);
    float err = el + 8.f * U1 * sqrtf(vv);
    float g = dc - rb - err;
    if (g <= 0.f) return 0.f;
    return g * g * (1.f - RELM);
}

// ---------------------------------------------------------------------------
// Line kernel (line-integrated scalars, LUT kernel)
// ---------------------------------------------------------------------------
// _lin_lut, kernel_function/line_integrated_kernel.jl:13-19, with the
// q >= q_max cut (:90-94) and the 1/h factor (:132-137).
// n = entries of the table, dq its spacing (idq = 1/dq: the float path
// multiplies, FP64 divides as the reference does), K the kernel's support.
template <class C> __device__ __forceinline__ C line_W(C r, C h, C invh, const C* lut, C dq, C idq, int n, C K) {
    C q = r * invh;
    if (q >= K) return C(0);
    C idxf = (sizeof(C) == 4 ? q * idq : q / dq) + C(1);
    int i = (int)idxf;  // q >= 0
    i = i < 1 ? 1 : (i > n - 1 ? n - 1 : i);
    C t = idxf - C(i);
    C v = lut[i - 1] * (C(1) - t) + lut[i] * t;
    return invh * v;
}

// Per-warp shared-memory stage of a span of leaves (FP32C line path).
template <int KC> struct LStage {
    float4 L[SPAN];
    float ih[SPAN];  // 1/h (float)
    float mr[SPAN];
    float col[KC][SPAN];
};

template <class T, int PREC, int ST, int KC, int WHAT>
__global__ void __launch_bounds__(128) k_lines(const Args<T> A) {
    using CT = typename std::conditional<PREC == PREC_FP64, double, float>::type;
    using Acc = typename std::conditional<PREC == PREC_FP64, PlainD, KahanF>::type;
    // FP32C with double inputs: float tests with a double fallback, leaf
    // spans.  Otherwise the reference's own arithmetic node by node, so that
    // the pruning decisions (including the rounding of the line-box lower
    // bound) are the reference's.
    constexpr bool BAND = (PREC == PREC_FP32C) && (sizeof(T) == 8);
    // The line table is read from global memory: one copy (16 or 32 KB) in
    // each SM's L1 serves every CTA there, where a copy per CTA in shared
    // memory took up to 256 KB an SM from the L1 that holds the leaf records
    // (C3: FP32C 35.7 -> 35.0 ms, FP64 145.9 -> 130.8 ms).  Only the FP64 sums
    // over the short float table convert it into shared memory.
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ LStage<KC> lstage_all[4];
    const int nlut = A.lut_n;
    const bool short_lut = nlut == LUT_SHORT_N;
    const CT* lut;
    if (PREC == PREC_FP64 && short_lut) {
        CT* sl = (CT*)smem_raw;
        for (int i = threadIdx.x; i < nlut; i += blockDim.x) sl[i] = (CT)A.lut_fs[i];
        __syncthreads();
        lut = sl;
    } else {
        lut = short_lut ? (const CT*)A.lut_fs : ((PREC == PREC_FP64) ? (const CT*)A.lut_d : (const CT*)A.lut_f);
    }
    // dq = Q[2] - Q[1] of the n-point table over [0, K] = K/(n-1) rounded to CT
    const CT dq = (CT)(A.tv.Kd / (double)(nlut - 1));
    const CT Kc = (CT)A.tv.Kd;
    const CT idq = CT(1) / dq;

    const TreeView<T>& tv = A.tv;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    LStage<KC>& st = lstage_all[wib];
    int64_t tile = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    if (tile >= A.src.ntiles) return;
    if (A.tile_list) tile = A.tile_list[tile];  // a permutation of the tiles (heavy first)
    const int64_t k = sample_of(A.src, tile, lane);
    const bool valid = k >= 0;
    T o[3] = {T(0), T(0), T(0)}, m[3] = {T(0), T(0), T(1)};
    if (valid) sample_coords(A.src, k, o, m);
    const float of[3] = {(float)o[0], (float)o[1], (float)o[2]};
    const float mf3[3] = {(float)m[0], (float)m[1], (float)m[2]};
    // |o|_1 and the particle coordinate scale S (coord_err = 2^-23 S)
    const float onorm = fabsf(of[0]) + fabsf(of[1]) + fabsf(of[2]);
    const float S = tv.coord_err / U1;
    const float el = 4.f * U1 * (onorm + 6.f * S) + 1e-30f;
    const float e64 = 4.5e-16f * (onorm + 6.f * S) * (onorm + 6.f * S);
    const int32_t start = (tv.root == 0) ? (int32_t)tv.n : tv.root;
    unsigned long long n_pairs = 0, n_retest = 0;
    int64_t steps = 0;

    T ha = T(0);
    if (ST != ST_SCATTER && valid) ha = (A.hmode == PSB_H_PER_SAMPLE) ? A.hs[k] : A.hs[0];
    const T Kt = (T)tv.Kd;
    const T ra = X<T>::mul(Kt, ha);
    const T ra2 = X<T>::mul(ra, ra);
    float ra2_hi = 0.f, ra2_lo = 0.f;
    if (BAND && ST != ST_SCATTER) {
        ra2_hi = __double2float_ru((double)ra2) * (1.f + RELM);
        ra2_lo = __double2float_rd((double)ra2) * (1.f - RELM);
    }
    const CT ia = (ST != ST_SCATTER) ? CT(1) / (CT)ha : CT(0);

    Acc S1, Sw[KC];
    S1.zero();
#pragma unroll
    for (int c = 0; c < KC; ++c) Sw[c].zero();
    uint64_t hsum = 0;
    int64_t hcount = 0;
    const int kc = A.rec.kc;

    // line-integrated weight of one accepted pair (s = squared distance)
    // dr = the line's distance from the particle, ib = 1/hb
    auto body = [&](int64_t li, CT dr, CT hb, CT ib, CT mr, const CT* cols) {
        ++n_pairs;
        if (WHAT == WHAT_DIGEST) {
            ++hcount;
            hsum += mix64((uint64_t)(li + 1));
            return;
        }
        CT W;
        if (ST == ST_GATHER) W = line_W<CT>(dr, (CT)ha, ia, lut, dq, idq, nlut, Kc);
        else {
            CT Wb = line_W<CT>(dr, hb, ib, lut, dq, idq, nlut, Kc);
            W = (ST == ST_SCATTER) ? Wb : CT(0.5) * (line_W<CT>(dr, (CT)ha, ia, lut, dq, idq, nlut, Kc) + Wb);
        }
        const CT w = mr * W;
        S1.add(w);
#pragma unroll
        for (int c = 0; c < KC; ++c)
            if (c < kc) Sw[c].add(cols[c] * w);
    };

    bool ok;
    if constexpr (BAND) {
        auto node_fn = [&](int ni) -> bool {
            float4 lo = __ldg(&tv.node_lo[ni]), hi = __ldg(&tv.node_hi[ni]);
            float lb = lb_d2_line_box(of, mf3, el, lo, hi);
            return !(lb > hi_r2_node<ST>(ra2_hi, lo.w, tv.Kf));
        };
        // perpendicular offset of a span's anchor (its first leaf) from the
        // line, in double
        auto perp_anchor = [&](int64_t a, float c[3], float& cerr) {
            double q0 = (double)__ldg(&tv.x[a]) - (double)o[0];
            double q1 = (double)__ldg(&tv.y[a]) - (double)o[1];
            double q2 = (double)__ldg(&tv.z[a]) - (double)o[2];
            double t0 = q0 * (double)m[0] + q1 * (double)m[1] + q2 * (double)m[2];
            c[0] = (float)(q0 - t0 * (double)m[0]);
            c[1] = (float)(q1 - t0 * (double)m[1]);
            c[2] = (float)(q2 - t0 * (double)m[2]);
            cerr = 1e-15f * (float)(fabs(q0) + fabs(q1) + fabs(q2) + 1.0);
        };
        auto span_fn = [&](int64_t lo, int cnt, bool part) {
            __syncwarp();
            if (lane < cnt) {
                const int64_t li = lo + lane;
                st.L[lane] = __ldg(&tv.leaf4[li]);
                if (WHAT != WHAT_DIGEST) {
                    st.ih[lane] = __ldg(&tv.leafK[li]).x;
                    st.mr[lane] = __ldg(&tv.mrho[li]);
#pragma unroll
                    for (int c = 0; c < KC; ++c)
                        if (c < kc) st.col[c][lane] = __ldg(&A.colF[c][li]);
                }
            }
            __syncwarp();
            if (!part) return;
            float cf[3], cerr;
            perp_anchor(lo, cf, cerr);
            // one error bound for every leaf of the span: |v|_1 <= |L|_1 + |cf|_1
            // with |L|_1 <= spanb.x (the span's largest, rounded up)
            const float sbx = __ldg(&tv.spanb[lo]).x;
            const float ev = 8.f * U1 * (2.f * sbx + fabsf(cf[0]) + fabsf(cf[1]) + fabsf(cf[2])) * (1.f + 4.f * U1) +
                             cerr + 1e-30f;
            for (int j = 0; j < cnt; ++j) {
                const float4 L = st.L[j];
                float v0 = L.x + cf[0], v1 = L.y + cf[1], v2 = L.z + cf[2];
                float vm = v0 * mf3[0] + v1 * mf3[1] + v2 * mf3[2];
                float w0 = v0 - vm * mf3[0], w1 = v1 - vm * mf3[1], w2 = v2 - vm * mf3[2];
                float fs = w0 * w0 + w1 * w1 + w2 * w2;
                float r = sqrtf(fs);
                float up = r + ev, dn = fmaxf(r - ev, 0.f);
                const float kb = tv.Kf * L.w;
                float rb2 = kb * kb;
                float r2lo, r2hi;
                if (ST == ST_GATHER) { r2lo = ra2_lo; r2hi = ra2_hi; }
                else if (ST == ST_SCATTER) { r2lo = rb2 * (1.f - 2.f * RELM); r2hi = rb2 * (1.f + 2.f * RELM); }
                else {
                    r2lo = fmaxf(ra2_lo, rb2 * (1.f - 2.f * RELM));
                    r2hi = fmaxf(ra2_hi, rb2 * (1.f + 2.f * RELM));
                }
                bool acc;
                if (up * up * (1.f + RELM) + e64 < r2lo) acc = true;
                else if (dn * dn * (1.f - RELM) - e64 > r2hi) acc = false;
                else {
                    ++n_retest;
                    const int64_t li = lo + j;
                    T e2 = ex_d2_line<T>(o, m, tv.x[li], tv.y[li], tv.z[li]);
                    acc = e2 <= ex_r2<ST, T>(ra2, tv.h[li], Kt);
                }
                if (!acc) continue;
                CT cols[KC];
#pragma unroll
                for (int c = 0; c < KC; ++c) cols[c] = (c < kc) ? (CT)st.col[c][j] : CT(0);
                body(lo + j, (CT)r, (CT)L.w, (CT)st.ih[j], (CT)st.mr[j], cols);
            }
        };
        ok = warp_traverse_spans(start, tv.n, tv.links, tv.escape, valid, node_fn, span_fn, steps);
    } else {
        auto node_fn = [&](int ni) -> bool {
            ++steps;
            T d2n = ex_d2_line_box<T>(o, m, tv, ni);
            T r2 = (ST == ST_GATHER) ? ra2 : ex_r2<ST, T>(ra2, __ldg(&tv.nscale[ni]), Kt);
            return !(d2n > r2);
        };
        auto leaf_fn = [&](int64_t li) {
            T e2 = ex_d2_line<T>(o, m, __ldg(&tv.x[li]), __ldg(&tv.y[li]), __ldg(&tv.z[li]));
            T hb = __ldg(&tv.h[li]);
            if (!(e2 <= ex_r2<ST, T>(ra2, hb, Kt))) return;
            CT cols[KC];
#pragma unroll
            for (int c = 0; c < KC; ++c) cols[c] = (c < kc) ? (CT)__ldg(&A.colT[c][li]) : CT(0);
            CT mr = (WHAT == WHAT_DIGEST) ? CT(0) : (CT)((double)tv.m[li] / (double)tv.rho[li]);
            const CT s2 = (CT)e2;
            body(li, sqrt(s2 < CT(0) ? CT(0) : s2), (CT)hb, CT(1) / (CT)hb, mr, cols);
        };
        ok = warp_traverse(start, tv.n, tv.left, tv.escape, valid, node_fn, leaf_fn);
    }

    if (valid) {
        if (WHAT == WHAT_DIGEST) {
            A.dig_count[k] = hcount;
            A.dig_hash[k] = hsum;
            if (A.ha_out) A.ha_out[k] = ha;
        } else if (A.lam) {
            // adjoint: cotangents of S1 (q = 0) and Sw_c (q = 1 + c), zero where S1 = 0
            const double s1 = S1.get();
            double l[1 + MAX_KC];
            for (int q = 0; q <= kc; ++q) l[q] = 0.0;
            if (s1 != 0.0) {
                const double inv = 1.0 / s1;
                for (int q = 0; q < A.rec.L; ++q) {
                    const double go = A.gout[q][k];
                    const int c = A.rec.a0[q];
                    l[1 + c] += A.rec.a1[q] ? go * inv : go;
                }
                // Shepard terms: d(Sw_c/S1)/dS1 = -Sw_c/S1^2
                for (int q = 0; q < A.rec.L; ++q) {
                    if (!A.rec.a1[q]) continue;
                    const int c = A.rec.a0[q];
                    double swc = 0.0;
#pragma unroll
                    for (int cc = 0; cc < KC; ++cc)
                        if (cc == c) swc = Sw[cc].get();
                    l[0] -= A.gout[q][k] * swc * inv * inv;
                }
            }
            for (int q = 0; q <= kc; ++q) A.lam[q * A.lam_stride + k] = l[q];
        } else {
            const double s1 = S1.get();
            const int L = A.rec.L;
            if (s1 == 0.0) {
                for (int q = 0; q < L; ++q) A.out[q][k] = qnan<T>();
            } else {
                double sw[MAX_KC];
#pragma unroll
                for (int c = 0; c < KC; ++c) sw[c] = Sw[c].get();
                const double inv = 1.0 / s1;
                for (int q = 0; q < L; ++q) {
                    const int a0 = A.rec.a0[q];
                    A.out[q][k] = (T)(A.rec.a1[q] ? sw[a0] * inv : sw[a0]);
                }
            }
        }
    }
#pragma unroll
    for (int q = 16; q > 0; q >>= 1) {
        n_pairs += __shfl_xor_sync(PSB_FULL, n_pairs, q);
        n_retest += __shfl_xor_sync(PSB_FULL, n_retest, q);
    }
    if (lane == 0 && A.stats) {
        atomicAdd(&A.stats[0], n_pairs);
        atomicAdd(&A.stats[1], n_retest);
        atomicAdd(&A.stats[2], (unsigned long long)steps);
    }
    if (!ok && lane == 0) atomicOr(A.err, PSB_DERR_TRAVERSAL);
}

// ---------------------------------------------------------------------------
// Sample ordering: Morton codes of sample positions (line origins) in the
// particle bounding box, clamped, then the stable radix sort.
// ---------------------------------------------------------------------------
// Explicit samples are put in the order of a coarser Morton curve than the
// particles': the order only groups nearby samples into tiles (every sample's
// result is independent of its tile), and 10 bits per axis of the particle
// box (1024 cells) make 30-bit keys, four radix passes instead of eight.
constexpr int SAMPLE_AXIS_BITS = 10;
constexpr int SAMPLE_KEY_BITS = 3 * SAMPLE_AXIS_BITS;

template <class T>
__global__ void k_sample_codes(const T* x, const T* y, const T* z, int64_t ns, double3 lo, double3 sc,
                               uint64_t* codes, uint32_t* idx) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    double v[3] = {(double)x[i], (double)y[i], (double)z[i]};
    double l[3] = {lo.x, lo.y, lo.z}, s[3] = {sc.x, sc.y, sc.z};
    uint64_t q[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double f = (v[d] - l[d]) * s[d];
        f = f < 0.0 ? 0.0 : (f > 2097151.0 ? 2097151.0 : f);
        q[d] = (uint64_t)f >> (21 - SAMPLE_AXIS_BITS);
    }
    codes[i] = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
    idx[i] = (uint32_t)i;
}

}  // namespace psb
