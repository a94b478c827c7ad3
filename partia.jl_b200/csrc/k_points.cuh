// k_points.cuh -- point-sample interpolation kernel.
//
// One warp owns a tile of 32 spatially close samples (one per lane) and walks
// the LBVH once for all of them (warp_traverse_spans).  A span of <= 32
// consecutive leaves is processed "transposed": lane j holds leaf j of the
// span; for every sample s that wants the span (a ballot), all lanes test
// their leaf against sample s at once and the ballot of the results is sample
// s's accept mask.  Each lane then runs the pair bodies of its own mask, in
// increasing leaf order (the reference's DFS order).
//
// Inclusion decisions: exact reference arithmetic for double inputs in
// PSB_PREC_FP64 and for float inputs; with double inputs in PSB_PREC_FP32C a
// float test classifies each pair as surely in, surely out or undecided, and
// undecided pairs are decided by the reference's double test.
#pragma once

#include "interp_kernels.cuh"

namespace psb {

// Per-warp shared memory: the span's leaves and the tile's samples.
template <class T, bool BAND, int KC> struct PStage {
    // leaves
    T x[SPAN], y[SPAN], z[SPAN], h[SPAN], m[SPAN], rho[SPAN];
    T col[KC][SPAN];
    // samples
    T px[SPAN], py[SPAN], pz[SPAN], ra2[SPAN], best[SPAN];
};
template <class T, int KC> struct PStage<T, true, KC> {
    static constexpr int NB = 1;            // spans batched before the pair bodies run
    static constexpr int SB = NB * SPAN;
    // leaves of up to NB spans (slot b*32 + j = leaf j of batched span b)
    float4 Q[SB];       // position relative to the warp anchor, h (inclusion tests)
    float4 Lr[SB];      // position relative to the span's first leaf (pair bodies)
    float4 K[SB];       // 1/h, sigma/h^3, sigma/h^4, m/rho
    float mf[SB];       // m
    float col[KC][SB];
    int64_t lo[NB];     // first leaf of each batched span
    float eq[SPAN];     // nearest search: error bound of Q
    // samples: position relative to the warp anchor + its error, radius bounds
    float4 P[SPAN];
    float2 R[SPAN];
    float2 AB[SPAN];    // per-span squared thresholds: surely in below A, surely out above B
    float thr[SPAN];    // nearest search: candidate threshold on the float d2
};

// Adjoint: cotangents of the per-sample sums S1, G, Dm, Dg, Sw_c, Sg_c for a
// loss sum_o gout[o][k] out_o(k), i.e. the derivative of the output recipes
// below.  Layout q: 0 S1 | 1-3 G | 4 Dm | 5-7 Dg | 8+c Sw_c | 8+kc+3c+d Sg_c.
// Sums shifted by a0 (FP32C) are shifted back first.  All zero where S1 = 0
// (every output NaN, nothing flows back).
template <class T, class Acc, class CT, int KC>
__device__ __forceinline__ void write_sum_cotangents(const Args<T>& A, int64_t k, const Acc& S1, const Acc (&G)[3],
                                                     const Acc (&Sw)[KC], const Acc (&Sg)[KC][3], const Acc& Dm,
                                                     const Acc (&Dg)[3], const double (&a0)[KC]) {
    const int kc = A.rec.kc;
    const double s1 = S1.get();
    const double g[3] = {G[0].get(), G[1].get(), G[2].get()};
    double sw[MAX_KC], sg[MAX_KC][3];
#pragma unroll
    for (int c = 0; c < KC; ++c) {
        sw[c] = Sw[c].get() + a0[c] * s1;
#pragma unroll
        for (int d = 0; d < 3; ++d) sg[c][d] = Sg[c][d].get() + a0[c] * g[d];
    }
    const double dm = Dm.get();
    double l[8 + 4 * MAX_KC];
    for (int q = 0; q < 8 + 4 * kc; ++q) l[q] = 0.0;
    double* lS1 = &l[0];
    double* lG = &l[1];
    double* lDm = &l[4];
    double* lDg = &l[5];
    double* lSw = &l[8];
    double* lSg = &l[8 + kc];
    if (s1 != 0.0) {
        const double inv = 1.0 / s1, inv2 = inv * inv;
        for (int o = 0; o < A.rec.L; ++o) {
            const double go = A.gout[o][k];
            const int op = A.rec.op[o];
            const int a0i = A.rec.a0[o], a1 = A.rec.a1[o], a2 = A.rec.a2[o], a3 = A.rec.a3[o];
            if (op == OP_SCALAR) {
                if (a1) { lSw[a0i] += go * inv; *lS1 -= go * sw[a0i] * inv2; }
                else lSw[a0i] += go;
            } else if (op == OP_GRADC) {  // Sg_c[d] - G[d] Sw_c / S1
                lSg[3 * a0i + a1] += go; lG[a1] -= go * sw[a0i] * inv; lSw[a0i] -= go * g[a1] * inv;
                *lS1 += go * g[a1] * sw[a0i] * inv2;
            } else if (op == OP_GRADD) {
                if (a2) {  // plain form Dg[d] - G[d] Dm (NaN, no cotangent, where Dm = 0)
                    if (dm != 0.0) { lDg[a1] += go; lG[a1] -= go * dm; *lDm -= go * g[a1]; }
                } else {   // Dg[d] - G[d] Dm / S1
                    lDg[a1] += go; lG[a1] -= go * dm * inv; *lDm -= go * g[a1] * inv;
                    *lS1 += go * g[a1] * dm * inv2;
                }
            } else if (op == OP_DIV) {
                const int cs[3] = {a0i, a1, a2};
                for (int d = 0; d < 3; ++d) {
                    const int c = cs[d];
                    lSg[3 * c + d] += go; lG[d] -= go * sw[c] * inv; lSw[c] -= go * g[d] * inv;
                    *lS1 += go * sw[c] * g[d] * inv2;
                }
            } else {  // OP_CURL: -Sg_a[ka] + Sg_b[kb] + Sw_a/S1 G[ka] - Sw_b/S1 G[kb]
                int a, ka, b, kb;
                if (a3 == 0) { a = a1; ka = 2; b = a2; kb = 1; }
                else if (a3 == 1) { a = a2; ka = 0; b = a0i; kb = 2; }
                else { a = a0i; ka = 1; b = a1; kb = 0; }
                lSg[3 * a + ka] -= go; lSg[3 * b + kb] += go;
                lG[ka] += go * sw[a] * inv; lG[kb] -= go * sw[b] * inv;
                lSw[a] += go * g[ka] * inv; lSw[b] -= go * g[kb] * inv;
                *lS1 -= go * (sw[a] * g[ka] - sw[b] * g[kb]) * inv2;
            }
        }
    }
    for (int q = 0; q < 8 + 4 * kc; ++q) A.lam[q * A.lam_stride + k] = l[q];
    (void)dm;
    (void)Dg;
}

// Output fields of one sample from its sums (general_interpolation.jl:128-214):
// NaN everywhere when S1 = 0, then each recipe op in catalog order.
template <class T, class Acc, class CT, int KC>
__device__ __forceinline__ void write_interp_outputs(const Args<T>& A, int64_t k, const Acc& S1, const Acc (&G)[3],
                                                     const Acc (&Sw)[KC], const Acc (&Sg)[KC][3], const Acc& Dm,
                                                     const Acc (&Dg)[3], const double (&a0)[KC]) {
    if (A.lam) {
        write_sum_cotangents<T, Acc, CT, KC>(A, k, S1, G, Sw, Sg, Dm, Dg, a0);
        return;
    }
    const double s1 = S1.get();
    const int L = A.rec.L;
    if (s1 == 0.0) {
        for (int o = 0; o < L; ++o) A.out[o][k] = qnan<T>();
    } else {
        // sums of (A - A0) w and (A - A0) g; gradients, divergences and
        // curls are invariant under the shift, scalars add A0 back.
        double sw[MAX_KC], sg[MAX_KC][3], sh[MAX_KC];
#pragma unroll
        for (int c = 0; c < KC; ++c) {
            sw[c] = Sw[c].get();
            sh[c] = a0[c];
#pragma unroll
            for (int d = 0; d < 3; ++d) sg[c][d] = Sg[c][d].get();
        }
        const double g[3] = {G[0].get(), G[1].get(), G[2].get()};
        const double inv = 1.0 / s1;
        for (int o = 0; o < L; ++o) {
            const int op = A.rec.op[o];
            const int a0i = A.rec.a0[o], a1 = A.rec.a1[o], a2 = A.rec.a2[o], a3 = A.rec.a3[o];
            double v;
            if (op == OP_SCALAR) {
                v = a1 ? sw[a0i] * inv + sh[a0i] : sw[a0i] + sh[a0i] * s1;
            } else if (op == OP_GRADC) {
                v = sg[a0i][a1] - g[a1] * (sw[a0i] * inv);
            } else if (op == OP_GRADD) {
                // a2 set: the plain density rho(r) = Dm replaces the Shepard-normalised
                // Dm / S1 (_gradient_density_kernel, gradient_interpolation.jl:1-170)
                const double dm = Dm.get();
                v = a2 ? (dm == 0.0 ? (double)NAN : Dg[a1].get() - g[a1] * dm) : Dg[a1].get() - g[a1] * (dm * inv);
            } else if (op == OP_DIV) {
                double f = sg[a0i][0] + sg[a1][1] + sg[a2][2];
                double b = (sw[a0i] * inv) * g[0] + (sw[a1] * inv) * g[1] + (sw[a2] * inv) * g[2];
                v = f - b;
            } else {  // OP_CURL, component a3
                double Ax = sw[a0i] * inv, Ay = sw[a1] * inv, Az = sw[a2] * inv;
                double f, b;
                if (a3 == 0) { f = sg[a1][2] - sg[a2][1]; b = Ay * g[2] - Az * g[1]; }
                else if (a3 == 1) { f = sg[a2][0] - sg[a0i][2]; b = Az * g[0] - Ax * g[2]; }
                else { f = sg[a0i][1] - sg[a1][0]; b = Ax * g[1] - Ay * g[0]; }
                v = -(f - b);
            }
            A.out[o][k] = (T)v;
        }
    }
}

// LBVH_find_nearest_h (LinearBVHQueries.jl:118-140) for the warp's samples:
// the smoothing length of the nearest particle, NaN without particles.  The
// reference starts its search with an infinite bound.  Here the bound starts
// at the exact distance to the particle next to the sample in Morton order
// (found by binary search of the sorted codes), and ties are resolved towards
// the smaller leaf index, so the result is the same argmin -- the first leaf
// in DFS order with the minimum distance.  stage_span(lo, cnt, false) stages
// the positions of leaves [lo, lo+cnt) in st (Q and eq for float tests, x y z
// otherwise); st.P / st.px.. hold the samples.
constexpr int64_t NEAREST_SEED = 8;

template <class T, bool BAND, class Stage, class StageSpan>
__device__ __forceinline__ T nearest_h_pass(const TreeView<T>& tv, Stage& st, StageSpan& stage_span, int lane,
                                            bool valid, const T p[3], const float pf[3], float pem, int32_t start,
                                            int64_t& steps, bool& ok) {
    double best = INFINITY;
    int64_t bidx = -1;
    if (valid) {
        uint64_t q[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double f = ((double)p[d] - tv.qlo[d]) * tv.qscale[d];
            f = f < 0.0 ? 0.0 : (f > 2097151.0 ? 2097151.0 : f);
            q[d] = (uint64_t)f;
        }
        const uint64_t code = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
        int64_t lo = 0, hi = tv.n;  // first index with codes[i] >= code
        while (lo < hi) {
            int64_t mid = (lo + hi) >> 1;
            if (__ldg(&tv.codes[mid]) < code) lo = mid + 1;
            else hi = mid;
        }
        // the (up to) 2 NEAREST_SEED particles around that position in Morton
        // order, in increasing index: the first strict minimum keeps the
        // smallest index.  A closer seed prunes more of the walk.
        const int64_t c0 = lo >= NEAREST_SEED ? lo - NEAREST_SEED : 0;
        const int64_t c1 = (lo + NEAREST_SEED <= tv.n) ? lo + NEAREST_SEED : tv.n;
        for (int64_t ci = c0; ci < c1; ++ci) {
            const double dc = (double)ex_d2_pp<T>(p, tv.x[ci], tv.y[ci], tv.z[ci]);
            if (dc < best) { best = dc; bidx = ci; }
        }
    }
    auto better = [&](double d2, int64_t li) { return d2 < best || (d2 == best && li < bidx); };
    // the node test compares in float against best rounded up (lb > bestf
    // implies lb > best): one conversion per improvement, not per step
    float bestf = __double2float_ru(best);
    auto node_fn = [&](int ni) -> bool {
        if constexpr (BAND) {
            float lb = lb_d2_pbox(pf, pem, __ldg(&tv.node_lo[ni]), __ldg(&tv.node_hi[ni]));
            return !(lb > bestf);
        } else {
            return !((double)ex_d2_pbox<T>(p, tv, ni) > best);
        }
    };
    auto span_fn = [&](int64_t lo, int cnt, bool part) {
        float eqmax = stage_span(lo, cnt, false);
        const unsigned parts = __ballot_sync(PSB_FULL, part);
        if (!parts) return;
        unsigned cand = 0;
        if constexpr (BAND) {
            // candidates: float d2 not above (sqrt(best) + error)^2 (eqmax is the span's bound)
            {
                const float4 Pme = st.P[lane];
                float bs = (float)sqrt(best);
                float e = 1.7320508f * (Pme.w + eqmax) + 4.f * U1 * bs + 1e-30f;
                float t = (bs + e) * (1.f + 4.f * U1);
                st.thr[lane] = isinf(best) ? INFINITY : t * t;
            }
            __syncwarp();
            if (3 * __popc(parts) >= 2 * cnt) {  // warp-uniform: many samples take part
                // each taking lane tests its sample against every leaf
                if (part) {
                    const float4 P = st.P[lane];
                    const float thr = st.thr[lane];
#pragma unroll 4
                    for (int j = 0; j < cnt; ++j) {
                        const float4 Q = st.Q[j];
                        float dx = P.x - Q.x, dy = P.y - Q.y, dz = P.z - Q.z;
                        cand |= (unsigned)(dx * dx + dy * dy + dz * dz <= thr) << j;
                    }
                }
            } else {  // lane j tests leaf j against each taking sample
                const float4 Q = st.Q[lane < cnt ? lane : 0];
                for (unsigned pp = parts; pp; pp &= pp - 1) {
                    const int s = __ffs(pp) - 1;
                    const float4 P = st.P[s];
                    const float thr = st.thr[s];
                    float dx = P.x - Q.x, dy = P.y - Q.y, dz = P.z - Q.z;
                    bool c = (lane < cnt) && (dx * dx + dy * dy + dz * dz <= thr);
                    unsigned b = __ballot_sync(PSB_FULL, c);
                    if (lane == s) cand = b;
                }
            }
            for (; cand; cand &= cand - 1) {
                const int64_t li = lo + __ffs(cand) - 1;
                double d2 = (double)ex_d2_pp<T>(p, tv.x[li], tv.y[li], tv.z[li]);
                if (better(d2, li)) { best = d2; bidx = li; bestf = __double2float_ru(best); }
            }
        } else {
            st.best[lane] = (T)best;
            __syncwarp();
            const int j = lane < cnt ? lane : 0;
            const T xj = st.x[j], yj = st.y[j], zj = st.z[j];
            for (unsigned pp = parts; pp; pp &= pp - 1) {
                const int s = __ffs(pp) - 1;
                const T ps[3] = {st.px[s], st.py[s], st.pz[s]};
                bool c = (lane < cnt) && (ex_d2_pp<T>(ps, xj, yj, zj) <= st.best[s]);
                unsigned b = __ballot_sync(PSB_FULL, c);
                if (lane == s) cand = b;
            }
            for (; cand; cand &= cand - 1) {
                const int jj = __ffs(cand) - 1;
                double d2 = (double)ex_d2_pp<T>(p, st.x[jj], st.y[jj], st.z[jj]);
                if (better(d2, lo + jj)) { best = d2; bidx = lo + jj; }
            }
        }
    };
    ok = warp_traverse_spans(start, tv.n, tv.links, tv.escape, valid, node_fn, span_fn, steps) && ok;
    return valid ? ((bidx >= 0) ? tv.h[bidx] : qnan<T>()) : T(0);
}

template <class T, int PREC, int ST, int KC, int WHAT, int KF>
__global__ void __launch_bounds__(128) k_points(const Args<T> A) {
    using CT = typename std::conditional<PREC == PREC_FP64, double, float>::type;
    using Acc = typename std::conditional<PREC == PREC_FP64, PlainD, KahanF>::type;
    constexpr bool BAND = (PREC == PREC_FP32C) && (sizeof(T) == 8);
    constexpr bool SHIFT = (PREC == PREC_FP32C);  // accumulate A - A0 (cancellation-free gradients)
    constexpr bool EXS = BAND && KF == 1;         // A - A0 from span-relative columns (span_shift)
    __shared__ PStage<T, BAND, KC> stage_all[4];
    const TreeView<T>& tv = A.tv;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    auto& st = stage_all[wib];
    int64_t tile = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    if (A.tile_list) {  // the tiles the two-kernel path handed back
        if (tile >= (int64_t)*A.tile_count) return;
        tile = A.tile_list[tile];
    } else if (tile >= A.src.ntiles) {
        return;  // warp-uniform
    }

    const int64_t k = sample_of(A.src, tile, lane);
    const bool valid = k >= 0;
    T p[3] = {T(0), T(0), T(0)}, dd[3];
    if (valid) sample_coords(A.src, k, p, dd);
    const float pf[3] = {(float)p[0], (float)p[1], (float)p[2]};
    const float pem = U1 * fmaxf(fmaxf(fabsf(pf[0]), fabsf(pf[1])), fabsf(pf[2])) + 1e-30f;
    const int32_t start = (tv.root == 0) ? (int32_t)tv.n : tv.root;
    const int kc = A.rec.kc;
    const bool need_dg = A.rec.need_dg != 0;
    unsigned long long n_pairs = 0, n_retest = 0;
    unsigned long long n_spans = 0, n_parts = 0, n_bodyit = 0;  // main-pass work counters (warp-uniform)
    int64_t steps = 0;
    bool ok = true;

    // warp anchor: the first valid sample of the tile
    const unsigned vmask = __ballot_sync(PSB_FULL, valid);
    const int first = vmask ? __ffs(vmask) - 1 : 0;
    const double cw[3] = {__shfl_sync(PSB_FULL, (double)p[0], first), __shfl_sync(PSB_FULL, (double)p[1], first),
                          __shfl_sync(PSB_FULL, (double)p[2], first)};
    if constexpr (BAND) {
        float sr[3] = {(float)((double)p[0] - cw[0]), (float)((double)p[1] - cw[1]), (float)((double)p[2] - cw[2])};
        float es = U1 * (fabsf(sr[0]) + fabsf(sr[1]) + fabsf(sr[2])) + 1e-30f;
        st.P[lane] = make_float4(sr[0], sr[1], sr[2], es);
    } else {
        st.px[lane] = p[0]; st.py[lane] = p[1]; st.pz[lane] = p[2];
    }

    // stage leaves [lo, lo+cnt): lane j takes leaf lo+j (all lanes call).
    // Returns the error bound of the float leaf positions Q (the same for the
    // whole span): |Q - exact| <= U1 (|L|_1 + |o|_1 + |Q|_1) per leaf, and
    // |Q|_1 <= (|L|_1 + |o|_1)(1 + U1), with max |L|_1 over the span stored.
    auto stage_span = [&](int64_t lo, int cnt, bool with_cols) -> float {
        __syncwarp();
        float eqmax = 0.f;
        if constexpr (BAND) {
            // the span's leaves are stored relative to its first leaf
            const float o0 = (float)((double)__ldg(&tv.x[lo]) - cw[0]);
            const float o1 = (float)((double)__ldg(&tv.y[lo]) - cw[1]);
            const float o2 = (float)((double)__ldg(&tv.z[lo]) - cw[2]);
            const float lm = __ldg(&tv.spanb[lo]).x;
            eqmax = U1 * (2.f * lm + 2.f * (fabsf(o0) + fabsf(o1) + fabsf(o2))) * (1.f + 4.f * U1);
            if (lane < cnt) {
                const float4 L = __ldg(&tv.leaf4[lo + lane]);
                st.Q[lane] = make_float4(L.x + o0, L.y + o1, L.z + o2, L.w);
            }
        } else if (lane < cnt) {
            const int64_t li = lo + lane;
            {
                st.x[lane] = __ldg(&tv.x[li]); st.y[lane] = __ldg(&tv.y[li]); st.z[lane] = __ldg(&tv.z[li]);
                st.h[lane] = __ldg(&tv.h[li]);
                if (with_cols) {
                    st.m[lane] = __ldg(&tv.m[li]); st.rho[lane] = __ldg(&tv.rho[li]);
#pragma unroll
                    for (int c = 0; c < KC; ++c)
                        if (c < kc) st.col[c][lane] = __ldg(&A.colT[c][li]);
                }
            }
        }
        __syncwarp();
        return eqmax;
    };

    // ---- sample smoothing length (LBVH_find_nearest_h or given) ----
    T ha = T(0);
    if (ST != ST_SCATTER) {
        if (A.hmode == PSB_H_NEAREST) {
            ha = nearest_h_pass<T, BAND>(tv, st, stage_span, lane, valid, p, pf, pem, start, steps, ok);
        } else if (valid) {
            ha = (A.hmode == PSB_H_PER_SAMPLE) ? A.hs[k] : A.hs[0];
        }
    }
    // radius = Kvalid * ha; radius2 = radius * radius (general_interpolation.jl:20-21)
    const T Kt = (T)tv.Kd;
    const T ra = X<T>::mul(Kt, ha);
    const T ra2 = X<T>::mul(ra, ra);
    if constexpr (BAND) {
        float ralo = 0.f, rahi = 0.f;
        if (ST != ST_SCATTER) {
            ralo = __double2float_rd((double)ra) * (1.f - 2.f * U1);
            rahi = __double2float_ru((double)ra) * (1.f + 2.f * U1);
        }
        st.R[lane] = make_float2(ralo, rahi);
    } else {
        st.ra2[lane] = ra2;
    }
    float ra2_hi = 0.f;
    if (BAND && ST != ST_SCATTER) ra2_hi = __double2float_ru((double)ra2) * (1.f + RELM);

    // ---- per-sample constants of the kernel weights ----
    const CT sig = (KF == 0) ? inv_pi<CT>() : (CT)tv.sig;
    CT ia = CT(0), sa3 = CT(0), sa4 = CT(0);
    if (ST != ST_SCATTER) {
        ia = CT(1) / (CT)ha;
        sa3 = sig * ia * ia * ia;
        sa4 = sa3 * ia;
    }
    const double kha = tv.Kd * (double)ha;
    const double fa2 = kha * kha;  // (K ha)^2 for the kernel piece at the support edge
    const double ika = (KF == 1 && ST != ST_SCATTER) ? 0.5 / (double)ha : 0.0;  // Wendland pair terms
    const float qe = (KF == 0) ? 1.f : tv.qedge;

    // ---- accumulators ----
    Acc S1, G[3], Sw[KC], Sg[KC][3], Dm, Dg[3];
    CT dens = CT(0);
    CT a0[KC];
    bool have0 = false;
    int64_t first0 = -1;  // EXS: the first accepted leaf (its column values are A0)
    S1.zero(); Dm.zero();
#pragma unroll
    for (int d = 0; d < 3; ++d) { G[d].zero(); Dg[d].zero(); }
#pragma unroll
    for (int c = 0; c < KC; ++c) {
        Sw[c].zero();
        a0[c] = CT(0);
#pragma unroll
        for (int d = 0; d < 3; ++d) Sg[c][d].zero();
    }
    uint64_t hsum = 0;
    int64_t hcount = 0;

    // kernel weights and accumulation of one accepted pair (leaf j of the stage)
    auto body = [&](int64_t li, int j, CT dx, CT dy, CT dz, CT d2, CT hb) {
        ++n_pairs;
        if (WHAT == WHAT_DIGEST) {
            ++hcount;
            hsum += mix64((uint64_t)(li + 1));
            return;
        }
        const CT r = sqrt(d2);
        const CT invr = (d2 > CT(0)) ? CT(1) / r : CT(0);
        CT Wsum = CT(0), csum = CT(0);  // kernel value and gradient coefficient (grad W = c * delta)
        if (ST != ST_SCATTER) {
            CT f, df;
            kfdf<KF, CT>(tv.kern, r * ia, f, df);
            Wsum = sa3 * f;
            csum = sa4 * df * invr;
        }
        if (ST != ST_GATHER) {
            CT ib = CT(1) / hb;
            CT sb3 = sig * ib * ib * ib;
            CT f, df;
            kfdf<KF, CT>(tv.kern, r * ib, f, df);
            CT Wb = sb3 * f, cb = sb3 * ib * df * invr;
            if (ST == ST_SCATTER) { Wsum = Wb; csum = cb; }
            else { Wsum = CT(0.5) * (Wsum + Wb); csum = CT(0.5) * (csum + cb); }
        }
        CT mb, mr;
        if constexpr (BAND) {
            mr = (CT)st.K[j].w;
            mb = (CT)st.mf[j];
        } else {
            mb = (CT)st.m[j];
            mr = (CT)((double)st.m[j] / (double)st.rho[j]);
        }
        if (WHAT == WHAT_DENSITY) {
            dens += (A.unit_mass ? CT(1) : mb) * Wsum;
            return;
        }
        const CT w = mr * Wsum;
        const CT gc = mr * csum;
        const CT gx = gc * dx, gy = gc * dy, gz = gc * dz;
        S1.add(w);
        G[0].add(gx); G[1].add(gy); G[2].add(gz);
        if (SHIFT && !have0) {
            have0 = true;
#pragma unroll
            for (int c = 0; c < KC; ++c)
                if (c < kc) a0[c] = (CT)st.col[c][j];
        }
#pragma unroll
        for (int c = 0; c < KC; ++c) {
            if (c < kc) {
                CT a = (CT)st.col[c][j];
                if (SHIFT) a -= a0[c];
                Sw[c].add(a * w);
                Sg[c][0].add(a * gx); Sg[c][1].add(a * gy); Sg[c][2].add(a * gz);
            }
        }
        if (need_dg) {
            Dm.add(mb * Wsum);
            CT mc = mb * csum;
            Dg[0].add(mc * dx); Dg[1].add(mc * dy); Dg[2].add(mc * dz);
        }
    };

    auto node_fn = [&](int ni) -> bool {
        if constexpr (BAND) {
            float4 lo = __ldg(&tv.node_lo[ni]), hi = __ldg(&tv.node_hi[ni]);
            float lb = lb_d2_pbox(pf, pem, lo, hi);
            return !(lb > hi_r2_node<ST>(ra2_hi, lo.w, tv.Kf));
        } else {
            T d2n = ex_d2_pbox<T>(p, tv, ni);
            T r2 = (ST == ST_GATHER) ? ra2 : ex_r2<ST, T>(ra2, __ldg(&tv.nscale[ni]), Kt);
            return !(d2n > r2);
        }
    };

    if constexpr (BAND) {
        // ---- FP32C main pass: batched spans, transposed tests, flattened pair loop ----
        constexpr int NB = PStage<T, true, KC>::NB;
        int nb = 0;                                   // batched spans (warp-uniform)
        unsigned acc0 = 0, acc1 = 0, acc2 = 0, acc3 = 0;
        unsigned unc0 = 0, unc1 = 0, unc2 = 0, unc3 = 0;
        const float4 Pme = st.P[lane];
        const float2 Rme = st.R[lane];
        float R0[3] = {0.f, 0.f, 0.f};  // the sample relative to the current span's first leaf
        float esmax = Pme.w, rahimax = Rme.y;  // tile-wide maxima (sample error, sample radius)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            esmax = fmaxf(esmax, __shfl_xor_sync(PSB_FULL, esmax, o));
            rahimax = fmaxf(rahimax, __shfl_xor_sync(PSB_FULL, rahimax, o));
        }

        auto pair_body = [&](int b, int j) {
            const int slot = b * SPAN + j;
            ++n_pairs;
            if (WHAT == WHAT_DIGEST) {
                ++hcount;
                hsum += mix64((uint64_t)(st.lo[b] + j + 1));
                return;
            }
            const float4 Lj = st.Lr[slot];
            const float4 K = st.K[slot];
            const float dx = __fsub_rn(R0[0], Lj.x);
            const float dy = __fsub_rn(R0[1], Lj.y);
            const float dz = __fsub_rn(R0[2], Lj.z);
            const int64_t li = st.lo[b] + j;
            float Wsum, csum;
            f32c_pair_weights<ST, KF>(
                tv.kern, tv.Kf, qe, dx, dy, dz, (float)ia, (float)sa3, (float)sa4, fa2, ika, (float)ha, K, Lj.w,
                [&]() {
                    const double ex = __dsub_rn((double)p[0], (double)tv.x[li]);
                    const double ey = __dsub_rn((double)p[1], (double)tv.y[li]);
                    const double ez = __dsub_rn((double)p[2], (double)tv.z[li]);
                    return __fma_rn(ex, ex, __fma_rn(ey, ey, __dmul_rn(ez, ez)));
                },
                [&]() { return __dmul_rn(tv.Kd, (double)tv.h[li]); }, Wsum, csum);
            if (WHAT == WHAT_DENSITY) {
                Dm.add(__fmul_rn(A.unit_mass ? 1.f : st.mf[slot], Wsum));
                return;
            }
            const float w = __fmul_rn(K.w, Wsum);
            const float gc = __fmul_rn(K.w, csum);
            const float gx = __fmul_rn(gc, dx), gy = __fmul_rn(gc, dy), gz = __fmul_rn(gc, dz);
            S1.add(w);
            G[0].add(gx); G[1].add(gy); G[2].add(gz);
            if (EXS && first0 < 0) first0 = li;
            if (!EXS && !have0) {
                have0 = true;
#pragma unroll
                for (int c = 0; c < KC; ++c)
                    if (c < kc) a0[c] = st.col[c][slot];
            }
#pragma unroll
            for (int c = 0; c < KC; ++c) {
                if (c < kc) {
                    // A - A0 as in k_bodies: for EXS the span-relative column
                    // plus the span's shift A[first leaf] - A0 (double, rounded
                    // once), else the float column less the float A0
                    const float a = EXS ? __fadd_rn(st.col[c][slot], span_shift(A.colT[c], st.lo[b], first0))
                                        : __fsub_rn(st.col[c][slot], (float)a0[c]);
                    Sw[c].add(__fmul_rn(a, w));
                    Sg[c][0].add(__fmul_rn(a, gx)); Sg[c][1].add(__fmul_rn(a, gy)); Sg[c][2].add(__fmul_rn(a, gz));
                }
            }
            if (need_dg) {
                const float mb = st.mf[slot];
                Dm.add(__fmul_rn(mb, Wsum));
                const float mc = __fmul_rn(mb, csum);
                Dg[0].add(__fmul_rn(mc, dx)); Dg[1].add(__fmul_rn(mc, dy)); Dg[2].add(__fmul_rn(mc, dz));
            }
        };

        auto flush = [&]() {
            // undecided pairs: the reference's double test
            for (int b = 0; b < nb; ++b) {
                unsigned u = b == 0 ? unc0 : b == 1 ? unc1 : b == 2 ? unc2 : unc3;
                unsigned add = 0;
                for (; u; u &= u - 1) {
                    const int jj = __ffs(u) - 1;
                    const int64_t li = st.lo[b] + jj;
                    ++n_retest;
                    T e2 = ex_d2_pp<T>(p, tv.x[li], tv.y[li], tv.z[li]);
                    if (e2 <= ex_r2<ST, T>(ra2, tv.h[li], Kt)) add |= 1u << jj;
                }
                if (b == 0) acc0 |= add; else if (b == 1) acc1 |= add; else if (b == 2) acc2 |= add; else acc3 |= add;
            }
            unc0 = unc1 = unc2 = unc3 = 0;
            n_bodyit += __reduce_max_sync(PSB_FULL, (unsigned)(__popc(acc0) + __popc(acc1) + __popc(acc2) + __popc(acc3)));
            // one flattened loop over the pairs of all batched spans, in leaf order
            while (true) {
                int b;
                unsigned* m;
                if (acc0) { b = 0; m = &acc0; }
                else if (acc1) { b = 1; m = &acc1; }
                else if (acc2) { b = 2; m = &acc2; }
                else if (acc3) { b = 3; m = &acc3; }
                else break;
                const int jj = __ffs(*m) - 1;
                *m &= *m - 1;
                pair_body(b, jj);
            }
            nb = 0;
            __syncwarp();
        };

        auto span_fn = [&](int64_t lo, int cnt, bool part) {
            const unsigned parts = __ballot_sync(PSB_FULL, part);
            if (!parts) return;
            const int b = nb;
            const int slot = b * SPAN + lane;
            float eq = 0.f, Aj = 0.f, Bj = 0.f, hb = 0.f;
            if (lane < cnt) {
                const int64_t li = lo + lane;
                const float4 L = __ldg(&tv.leaf4[li]);
                const float o0 = (float)((double)__ldg(&tv.x[lo]) - cw[0]);
                const float o1 = (float)((double)__ldg(&tv.y[lo]) - cw[1]);
                const float o2 = (float)((double)__ldg(&tv.z[lo]) - cw[2]);
                const float q0 = L.x + o0, q1 = L.y + o1, q2 = L.z + o2;
                hb = L.w;
                st.Q[slot] = make_float4(q0, q1, q2, hb);
                st.Lr[slot] = L;
                eq = U1 * (fabsf(L.x) + fabsf(L.y) + fabsf(L.z) + fabsf(o0) + fabsf(o1) + fabsf(o2) +
                           fabsf(q0) + fabsf(q1) + fabsf(q2));
                if (WHAT != WHAT_DIGEST) {
                    const float ih = 1.f / hb;
                    const float s3 = (float)sig * ih * ih * ih;
                    st.K[slot] = make_float4(ih, s3, s3 * ih, __ldg(&tv.mrho[li]));
                    if (need_dg || WHAT == WHAT_DENSITY) st.mf[slot] = __ldg(&tv.mf[li]);
#pragma unroll
                    for (int c = 0; c < KC; ++c)
                        if (c < kc) st.col[c][slot] = __ldg(&(EXS ? A.colR : A.colF)[c][li]);
                }
            }
            if (lane == 0) st.lo[b] = lo;
            // this lane's sample relative to the span's first leaf, in double
            // then rounded: the pair separation R - L then carries only the
            // rounding of two small vectors
            R0[0] = (float)((double)p[0] - (double)__ldg(&tv.x[lo]));
            R0[1] = (float)((double)p[1] - (double)__ldg(&tv.y[lo]));
            R0[2] = (float)((double)p[2] - (double)__ldg(&tv.z[lo]));
            // error bound of float distances for this span, the same for every pair
            float eqm = eq;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) eqm = fmaxf(eqm, __shfl_xor_sync(PSB_FULL, eqm, o));
            const float rbhi = tv.Kf * hb * (1.f + 3.f * U1), rblo = tv.Kf * hb * (1.f - 3.f * U1);
            // the rounding of r itself enters through 4 U1 r (r <= the larger radius)
            float rmax = rahimax;
            if (ST != ST_GATHER) {
                float rb = rbhi;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) rb = fmaxf(rb, __shfl_xor_sync(PSB_FULL, rb, o));
                rmax = fmaxf(rmax, rb);
            }
            const float E = 1.7320508f * (esmax + eqm) + 4.f * U1 * rmax + 1e-30f;
            if (ST != ST_GATHER && lane < cnt) {
                const float il = fmaxf((rblo - E) * (1.f - 4.f * U1), 0.f), ih2 = (rbhi + E) * (1.f + 4.f * U1);
                Aj = il * il;
                Bj = ih2 * ih2;
            }
            {
                float As = 0.f, Bs = 0.f;
                if (ST != ST_SCATTER) {
                    const float il = fmaxf((Rme.x - E) * (1.f - 4.f * U1), 0.f), ih2 = (Rme.y + E) * (1.f + 4.f * U1);
                    As = il * il;
                    Bs = ih2 * ih2;
                }
                st.AB[lane] = make_float2(As, Bs);
            }
            __syncwarp();
            const float4 Q = st.Q[lane < cnt ? slot : b * SPAN];
            unsigned myacc = 0, myunc = 0;
            for (unsigned pp = parts; pp; pp &= pp - 1) {
                const int s = __ffs(pp) - 1;
                const float4 P = st.P[s];
                const float2 AB = st.AB[s];
                const float dx = P.x - Q.x, dy = P.y - Q.y, dz = P.z - Q.z;
                const float d2 = dx * dx + dy * dy + dz * dz;
                const bool in = (lane < cnt) && d2 < fmaxf(AB.x, Aj);
                const bool un = (lane < cnt) && !in && !(d2 > fmaxf(AB.y, Bj));
                const unsigned bi = __ballot_sync(PSB_FULL, in), bu = __ballot_sync(PSB_FULL, un);
                if (lane == s) { myacc = bi; myunc = bu; }
            }
            if (b == 0) { acc0 = myacc; unc0 = myunc; }
            else if (b == 1) { acc1 = myacc; unc1 = myunc; }
            else if (b == 2) { acc2 = myacc; unc2 = myunc; }
            else { acc3 = myacc; unc3 = myunc; }
            ++n_spans;
            n_parts += __popc(parts);
            nb = b + 1;
            __syncwarp();
            if (nb == NB) flush();  // pair bodies of this span (R0 / R1 belong to it)
        };
        ok = warp_traverse_spans(start, tv.n, tv.links, tv.escape, valid, node_fn, span_fn, steps) && ok;
        if (nb > 0) flush();
        if (WHAT == WHAT_DENSITY) dens = (CT)Dm.get();
    } else {
        const bool with_cols = (WHAT != WHAT_DIGEST);
        auto span_fn = [&](int64_t lo, int cnt, bool part) {
            stage_span(lo, cnt, with_cols);
            const unsigned parts = __ballot_sync(PSB_FULL, part);
            if (!parts) return;
            ++n_spans;
            n_parts += __popc(parts);
            unsigned acc = 0, unc = 0;
            const int j = lane < cnt ? lane : 0;
            if constexpr (BAND) {
                const float4 Q = st.Q[j];
                const float eq = st.eq[j];
                const float rblo = tv.Kf * Q.w * (1.f - 3.f * U1), rbhi = tv.Kf * Q.w * (1.f + 3.f * U1);
                for (unsigned pp = parts; pp; pp &= pp - 1) {
                    const int s = __ffs(pp) - 1;
                    const float4 P = st.P[s];
                    const float2 R = st.R[s];
                    float dx = P.x - Q.x, dy = P.y - Q.y, dz = P.z - Q.z;
                    float d2 = dx * dx + dy * dy + dz * dz;
                    float rlo, rhi;
                    if (ST == ST_GATHER) { rlo = R.x; rhi = R.y; }
                    else if (ST == ST_SCATTER) { rlo = rblo; rhi = rbhi; }
                    else { rlo = fmaxf(R.x, rblo); rhi = fmaxf(R.y, rbhi); }
                    float e = 1.7320508f * (P.w + eq) + 4.f * U1 * rhi + 1e-30f;
                    float il = (rlo - e) * (1.f - 4.f * U1), ih = (rhi + e) * (1.f + 4.f * U1);
                    bool in = (lane < cnt) && il > 0.f && d2 < il * il;
                    bool un = (lane < cnt) && !in && !(d2 > ih * ih);
                    unsigned bi = __ballot_sync(PSB_FULL, in), bu = __ballot_sync(PSB_FULL, un);
                    if (lane == s) { acc = bi; unc = bu; }
                }
                // undecided pairs: the reference's double test
                for (unsigned u = unc; u; u &= u - 1) {
                    const int jj = __ffs(u) - 1;
                    const int64_t li = lo + jj;
                    ++n_retest;
                    T e2 = ex_d2_pp<T>(p, tv.x[li], tv.y[li], tv.z[li]);
                    if (e2 <= ex_r2<ST, T>(ra2, tv.h[li], Kt)) acc |= 1u << jj;
                }
                const float sr0 = st.P[lane].x, sr1 = st.P[lane].y, sr2 = st.P[lane].z;
                n_bodyit += __reduce_max_sync(PSB_FULL, (unsigned)__popc(acc));
                for (; acc; acc &= acc - 1) {
                    const int jj = __ffs(acc) - 1;
                    const float4 Qj = st.Q[jj];
                    float fx = sr0 - Qj.x, fy = sr1 - Qj.y, fz = sr2 - Qj.z;
                    body(lo + jj, jj, (CT)fx, (CT)fy, (CT)fz, (CT)(fx * fx + fy * fy + fz * fz), (CT)Qj.w);
                }
            } else {
                const T xj = st.x[j], yj = st.y[j], zj = st.z[j], hj = st.h[j];
                const T r2b = ex_r2<ST_SCATTER, T>(T(0), hj, Kt);  // (K hb)^2
                for (unsigned pp = parts; pp; pp &= pp - 1) {
                    const int s = __ffs(pp) - 1;
                    const T ps[3] = {st.px[s], st.py[s], st.pz[s]};
                    const T ra2s = st.ra2[s];
                    T e2 = ex_d2_pp<T>(ps, xj, yj, zj);
                    T r2 = (ST == ST_GATHER) ? ra2s : ((ST == ST_SCATTER) ? r2b : jmax(ra2s, r2b));
                    bool in = (lane < cnt) && (e2 <= r2);
                    unsigned bi = __ballot_sync(PSB_FULL, in);
                    if (lane == s) acc = bi;
                }
                n_bodyit += __reduce_max_sync(PSB_FULL, (unsigned)__popc(acc));
                for (; acc; acc &= acc - 1) {
                    const int jj = __ffs(acc) - 1;
                    const T xb = st.x[jj], yb = st.y[jj], zb = st.z[jj];
                    const T e2 = ex_d2_pp<T>(p, xb, yb, zb);
                    body(lo + jj, jj, (CT)(p[0] - xb), (CT)(p[1] - yb), (CT)(p[2] - zb), (CT)e2, (CT)st.h[jj]);
                }
            }
        };

        ok = warp_traverse_spans(start, tv.n, tv.links, tv.escape, valid, node_fn, span_fn, steps) && ok;
    }

    // ---- outputs ----
    if (valid) {
        if (WHAT != WHAT_DIGEST && A.ha_out) A.ha_out[k] = ha;
        if (WHAT == WHAT_DIGEST) {
            A.dig_count[k] = hcount;
            A.dig_hash[k] = hsum;
            if (A.ha_out) A.ha_out[k] = ha;
        } else if (WHAT == WHAT_DENSITY) {
            A.out[0][k] = (T)dens;
        } else {
            double a0o[KC];
#pragma unroll
            for (int c = 0; c < KC; ++c)
                a0o[c] = EXS ? ((c < kc && first0 >= 0) ? (double)A.colT[c][first0] : 0.0) : (double)a0[c];
            write_interp_outputs<T, Acc, CT, KC>(A, k, S1, G, Sw, Sg, Dm, Dg, a0o);
        }
    }
    // ---- statistics and errors ----
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n_pairs += __shfl_xor_sync(PSB_FULL, n_pairs, o);
        n_retest += __shfl_xor_sync(PSB_FULL, n_retest, o);
    }
    if (lane == 0 && A.stats) {
        atomicAdd(&A.stats[0], n_pairs);
        atomicAdd(&A.stats[1], n_retest);
        atomicAdd(&A.stats[2], (unsigned long long)steps);
        atomicAdd(&A.stats[3], n_spans);
        atomicAdd(&A.stats[4], n_parts);
        atomicAdd(&A.stats[5], n_bodyit);
    }
    if (!ok && lane == 0) atomicOr(A.err, PSB_DERR_TRAVERSAL);
}

}  // namespace psb
