// k_split.cuh -- the two-kernel point path.
//
// k_collect walks the LBVH for a tile of 32 samples (one warp, the same walk,
// spans and inclusion decisions as k_points) and records, per sample, the
// accepted leaves as one entry per span (first leaf, 32-bit mask, the sample's
// offset from the first leaf) plus the sample's smoothing length.  It keeps no accumulators, so it runs with few registers.
// k_bodies then evaluates the kernel weights and sums of every recorded pair:
// each lane runs through its own sample's list in one flattened loop, so a
// warp iteration does 32 pair bodies until the shortest lists run out, instead
// of idling lanes once per span.  Pairs are visited in the same order as in
// k_points (span order, then leaf order), with the same arithmetic.
#pragma once

#include "k_points.cuh"

namespace psb {

template <class T, bool BAND> struct CStage {
    T x[SPAN], y[SPAN], z[SPAN], h[SPAN];
    T px[SPAN], py[SPAN], pz[SPAN], ra2[SPAN], best[SPAN];
};
template <class T> struct CStage<T, true> {
    float4 Q[SPAN];   // leaf position relative to the warp anchor, h (nearest search)
    float4 P[SPAN];   // sample position relative to the warp anchor, error bound
    float2 R[SPAN];   // sample radius bounds
    float2 AB[SPAN];  // per-span squared thresholds of each leaf
    float2 SAB[SPAN]; // per-span squared thresholds of each sample
    float thr[SPAN];  // nearest search: candidate threshold
};

// 12 CTAs (48 warps) per SM, 40 registers: the walk is bound by issue and
// by its node loads, and more resident warps beat the few spills this costs
// (C2: FP32C step 5.52 -> 5.42 ms, FP64 7.95 -> 7.37 ms; 16 CTAs at 32
// registers spill too much: 5.67 / 8.18 ms).
template <class T, int PREC, int ST>
__global__ void __launch_bounds__(128, 12) k_collect(const Args<T> A) {
    constexpr bool BAND = (PREC == PREC_FP32C) && (sizeof(T) == 8);
    __shared__ CStage<T, BAND> stage_all[4];
    const TreeView<T>& tv = A.tv;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    auto& st = stage_all[wib];
    const int64_t bt = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    if (bt >= A.sp.ntiles) return;  // warp-uniform
    const int64_t tile = A.sp.tile0 + bt;

    const int64_t k = sample_of(A.src, tile, lane);
    const bool valid = k >= 0;
    T p[3] = {T(0), T(0), T(0)}, dd[3];
    if (valid) sample_coords(A.src, k, p, dd);
    const float pf[3] = {(float)p[0], (float)p[1], (float)p[2]};
    const float pem = U1 * fmaxf(fmaxf(fabsf(pf[0]), fabsf(pf[1])), fabsf(pf[2])) + 1e-30f;
    const int32_t start = (tv.root == 0) ? (int32_t)tv.n : tv.root;
    uint32_t n_pairs = 0, n_retest = 0, n_spans = 0, n_parts = 0;  // per lane / warp, widened below
    int64_t steps = 0;
    bool ok = true;

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

    // positions of leaves [lo, lo+cnt): lane j takes leaf lo+j (all lanes call)
    // (the span's float error bound is the same for every leaf; see k_points)
    auto stage_span = [&](int64_t lo, int cnt, bool) -> float {
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
            st.x[lane] = __ldg(&tv.x[li]); st.y[lane] = __ldg(&tv.y[li]); st.z[lane] = __ldg(&tv.z[li]);
            st.h[lane] = __ldg(&tv.h[li]);
        }
        __syncwarp();
        return eqmax;
    };

    T ha = T(0);
    if (ST != ST_SCATTER) {
        if (A.hmode == PSB_H_NEAREST) {
            ha = nearest_h_pass<T, BAND>(tv, st, stage_span, lane, valid, p, pf, pem, start, steps, ok);
        } else if (valid) {
            ha = (A.hmode == PSB_H_PER_SAMPLE) ? A.hs[k] : A.hs[0];
        }
    }
    const T Kt = (T)tv.Kd;
    const T ra = X<T>::mul(Kt, ha);
    const T ra2 = X<T>::mul(ra, ra);
    float ra2_hi = 0.f;
    if constexpr (BAND) {
        float ralo = 0.f, rahi = 0.f;
        if (ST != ST_SCATTER) {
            ralo = __double2float_rd((double)ra) * (1.f - 2.f * U1);
            rahi = __double2float_ru((double)ra) * (1.f + 2.f * U1);
            ra2_hi = __double2float_ru((double)ra2) * (1.f + RELM);
        }
        st.R[lane] = make_float2(ralo, rahi);
    } else {
        st.ra2[lane] = ra2;
    }

    // this lane's pair list
    float4* ent4 = A.sp.ent4 + (size_t)bt * RCAP * 32 + lane;
    uint32_t* emask = A.sp.emask + (size_t)bt * RCAP * 32 + lane;
    int nent = 0;
    bool ovf = false;
    auto emit = [&](int64_t lo, unsigned acc) {
        if (!acc) return;
        n_pairs += __popc(acc);
        if (nent < RCAP) {
            // the sample relative to the span's first leaf, in double then
            // rounded: the pair separation R - L carries only the rounding of
            // two small vectors
            float r0 = 0.f, r1 = 0.f, r2 = 0.f;
            if (BAND) {
                r0 = (float)((double)p[0] - (double)__ldg(&tv.x[lo]));
                r1 = (float)((double)p[1] - (double)__ldg(&tv.y[lo]));
                r2 = (float)((double)p[2] - (double)__ldg(&tv.z[lo]));
            }
            ent4[(size_t)nent * 32] = make_float4(r0, r1, r2, __int_as_float((int)lo));
            emask[(size_t)nent * 32] = acc;
            ++nent;
        } else {
            ovf = true;
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
        const float4 Pme = st.P[lane];
        const float2 Rme = st.R[lane];
        float esmax = Pme.w, rahimax = Rme.y;  // tile-wide maxima (sample error, sample radius)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            esmax = fmaxf(esmax, __shfl_xor_sync(PSB_FULL, esmax, o));
            rahimax = fmaxf(rahimax, __shfl_xor_sync(PSB_FULL, rahimax, o));
        }
        auto span_fn = [&](int64_t lo, int cnt, bool part) {
            const unsigned parts = __ballot_sync(PSB_FULL, part);
            if (!parts) return;
            // the span's anchor (first leaf) relative to the warp anchor and its
            // bounds: one error bound E for every float distance of the span
            const float o0 = (float)((double)__ldg(&tv.x[lo]) - cw[0]);
            const float o1 = (float)((double)__ldg(&tv.y[lo]) - cw[1]);
            const float o2 = (float)((double)__ldg(&tv.z[lo]) - cw[2]);
            const float2 sb = __ldg(&tv.spanb[lo]);
            const float eqm = U1 * (2.f * sb.x + 2.f * (fabsf(o0) + fabsf(o1) + fabsf(o2))) * (1.f + 4.f * U1);
            // the rounding of r itself enters through 4 U1 r (r <= the larger radius)
            float rmax = rahimax;
            if (ST != ST_GATHER) rmax = fmaxf(rmax, tv.Kf * sb.y * (1.f + 3.f * U1));
            const float E = 1.7320508f * (esmax + eqm) + 4.f * U1 * rmax + 1e-30f;
            // this lane's sample thresholds
            float As = 0.f, Bs = 0.f;
            if (ST != ST_SCATTER) {
                const float il = fmaxf((Rme.x - E) * (1.f - 4.f * U1), 0.f), ih2 = (Rme.y + E) * (1.f + 4.f * U1);
                As = il * il;
                Bs = ih2 * ih2;
            }
            // few samples take part: lane j tests leaf j against each of them;
            // otherwise each taking lane tests its sample against every leaf
            const bool by_sample = 3 * __popc(parts) >= 2 * cnt;  // warp-uniform
            // the span's leaves (and their radius thresholds) in shared memory
            __syncwarp();
            float4 Qme = make_float4(0.f, 0.f, 0.f, 0.f);
            float Aj = 0.f, Bj = 0.f;
            if (lane < cnt) {
                const float4 L = __ldg(&tv.leaf4[lo + lane]);
                Qme = make_float4(L.x + o0, L.y + o1, L.z + o2, L.w);
                st.Q[lane] = Qme;
                if (ST != ST_GATHER) {
                    const float rbhi = tv.Kf * L.w * (1.f + 3.f * U1), rblo = tv.Kf * L.w * (1.f - 3.f * U1);
                    const float il = fmaxf((rblo - E) * (1.f - 4.f * U1), 0.f), ih2 = (rbhi + E) * (1.f + 4.f * U1);
                    Aj = il * il;
                    Bj = ih2 * ih2;
                    st.AB[lane] = make_float2(Aj, Bj);
                }
            }
            if (!by_sample) st.SAB[lane] = make_float2(As, Bs);
            __syncwarp();
            // surely in: d2 < A; maybe in: d2 <= B (undecided = maybe and not surely)
            unsigned myacc = 0, mymaybe = 0;
            if (!by_sample) {
                for (unsigned pp = parts; pp; pp &= pp - 1) {
                    const int s = __ffs(pp) - 1;
                    const float4 Ps = st.P[s];
                    const float2 sab = st.SAB[s];
                    const float dx = Ps.x - Qme.x, dy = Ps.y - Qme.y, dz = Ps.z - Qme.z;
                    const float d2 = dx * dx + dy * dy + dz * dz;
                    const float At = (ST == ST_GATHER) ? sab.x : ((ST == ST_SCATTER) ? Aj : fmaxf(sab.x, Aj));
                    const float Bt = (ST == ST_GATHER) ? sab.y : ((ST == ST_SCATTER) ? Bj : fmaxf(sab.y, Bj));
                    const unsigned bi = __ballot_sync(PSB_FULL, lane < cnt && d2 < At);
                    const unsigned bm = __ballot_sync(PSB_FULL, lane < cnt && d2 <= Bt);
                    if (lane == s) { myacc = bi; mymaybe = bm; }
                }
            } else if (part) {
#pragma unroll 4
                for (int j = 0; j < cnt; ++j) {
                    const float4 Q = st.Q[j];
                    const float dx = Pme.x - Q.x, dy = Pme.y - Q.y, dz = Pme.z - Q.z;
                    const float d2 = dx * dx + dy * dy + dz * dz;
                    float At = As, Bt = Bs;
                    if (ST != ST_GATHER) {
                        const float2 ab = st.AB[j];
                        At = (ST == ST_SCATTER) ? ab.x : fmaxf(As, ab.x);
                        Bt = (ST == ST_SCATTER) ? ab.y : fmaxf(Bs, ab.y);
                    }
                    myacc |= (unsigned)(d2 < At) << j;
                    mymaybe |= (unsigned)(d2 <= Bt) << j;
                }
            }
            const unsigned myunc = mymaybe & ~myacc;
            // undecided pairs: the reference's double test
            for (unsigned u = myunc; u; u &= u - 1) {
                const int jj = __ffs(u) - 1;
                const int64_t li = lo + jj;
                ++n_retest;
                T e2 = ex_d2_pp<T>(p, tv.x[li], tv.y[li], tv.z[li]);
                if (e2 <= ex_r2<ST, T>(ra2, tv.h[li], Kt)) myacc |= 1u << jj;
            }
            emit(lo, myacc);
            ++n_spans;
            n_parts += __popc(parts);
        };
        ok = warp_traverse_spans(start, tv.n, tv.links, tv.escape, valid, node_fn, span_fn, steps) && ok;
    } else {
        auto span_fn = [&](int64_t lo, int cnt, bool part) {
            stage_span(lo, cnt, false);
            const unsigned parts = __ballot_sync(PSB_FULL, part);
            if (!parts) return;
            ++n_spans;
            n_parts += __popc(parts);
            unsigned acc = 0;
            const int j = lane < cnt ? lane : 0;
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
            emit(lo, acc);
        };
        ok = warp_traverse_spans(start, tv.n, tv.links, tv.escape, valid, node_fn, span_fn, steps) && ok;
    }

    const bool tovf = __any_sync(PSB_FULL, ovf);
    if (BAND && A.sp.eshift && !tovf && nent > 0) {
        // the column shifts of this lane's entries, A[lo] - A0 (span_shift),
        // after the walk: here the entries' loads are independent and overlap,
        // where inside the walk each would stall it.  A0 are the column values
        // of the first accepted leaf.
        const int kc = A.rec.kc;
        float* esh = A.sp.eshift + (size_t)bt * RCAP * kc * 32 + lane;
        const int32_t fl = __float_as_int(ent4[0].w) + __ffs(emask[0]) - 1;
        for (int c = 0; c < kc; ++c) {
#pragma unroll 4
            for (int e = 0; e < nent; ++e)
                esh[((size_t)e * kc + c) * 32] = span_shift(A.colT[c], (int64_t)__float_as_int(ent4[(size_t)e * 32].w), fl);
        }
    }
    if (valid && A.ha_out) A.ha_out[k] = ha;
    A.sp.cnt[bt * 32 + lane] = tovf ? (uint8_t)0xFF : (uint8_t)nent;
    ((T*)A.sp.ha)[bt * 32 + lane] = ha;
    if (tovf && lane == 0) {
        const unsigned slot = atomicAdd(A.sp.ovf_count, 1u);
        A.sp.ovf_tiles[slot] = (int32_t)tile;
    }
    // the single-kernel pass counts the pairs of an overflowed tile
    unsigned long long t_pairs = tovf ? 0ull : n_pairs, t_retest = n_retest;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        t_pairs += __shfl_xor_sync(PSB_FULL, t_pairs, o);
        t_retest += __shfl_xor_sync(PSB_FULL, t_retest, o);
    }
    if (lane == 0 && A.stats) {
        atomicAdd(&A.stats[0], t_pairs);
        atomicAdd(&A.stats[1], t_retest);
        atomicAdd(&A.stats[2], (unsigned long long)steps);
        atomicAdd(&A.stats[3], (unsigned long long)n_spans);
        atomicAdd(&A.stats[4], (unsigned long long)n_parts);
    }
    if (!ok && lane == 0) atomicOr(A.err, PSB_DERR_TRAVERSAL);
}

// The data of one pair for k_bodies: float records for the FP32C path of
// double inputs, the exact particle values otherwise.
template <class T, bool BAND, int KC> struct PairData {
    T x, y, z, h, m, rho;
    T col[KC];
    __device__ __forceinline__ void load(const TreeView<T>& tv, const Args<T>& A, int64_t li, int kc, bool,
                                         const float*, const float* const*) {
        x = __ldg(&tv.x[li]); y = __ldg(&tv.y[li]); z = __ldg(&tv.z[li]);
        h = __ldg(&tv.h[li]); m = __ldg(&tv.m[li]); rho = __ldg(&tv.rho[li]);
#pragma unroll
        for (int c = 0; c < KC; ++c) col[c] = (c < kc) ? __ldg(&A.colT[c][li]) : T(0);
    }
};
template <class T, int KC> struct PairData<T, true, KC> {
    float4 L, K;      // leaf4 and leafK of the particle
    float col[KC];    // the column in float, or for EXS span-relative (A - A0 once the entry's shift is added)
    float mb;         // mass (density gradient only)
    float r[3];       // the sample relative to the span's first leaf
    int64_t li;       // leaf index
    double xd, yd, zd, hd;  // the particle in double (outer kernel piece)
    __device__ __forceinline__ void load(const TreeView<T>& tv, const Args<T>& A, int64_t li, int kc, bool need_dg,
                                         const float* Rs, const float* const* cols) {
        L = __ldg(&tv.leaf4[li]);
        K = __ldg(&tv.leafK[li]);
#pragma unroll
        for (int c = 0; c < KC; ++c) col[c] = (c < kc) ? __ldg(&cols[c][li]) : 0.f;
        mb = need_dg ? __ldg(&tv.mf[li]) : 0.f;
        r[0] = Rs[0]; r[1] = Rs[1]; r[2] = Rs[2];
        this->li = li;
        xd = __ldg(&tv.x[li]); yd = __ldg(&tv.y[li]); zd = __ldg(&tv.z[li]); hd = __ldg(&tv.h[li]);
    }
};

template <class T, int PREC, int ST, int KC, int KF, bool DG>
__global__ void __launch_bounds__(128, (KC <= 4) ? 4 : 2) k_bodies(const Args<T> A) {
    using CT = typename std::conditional<PREC == PREC_FP64, double, float>::type;
    using Acc = typename std::conditional<PREC == PREC_FP64, PlainD, KahanF>::type;
    constexpr bool BAND = (PREC == PREC_FP32C) && (sizeof(T) == 8);
    constexpr bool SHIFT = (PREC == PREC_FP32C);
    constexpr bool EXS = BAND && KF == 1;  // column shifts formed in double (span_shift), from k_collect
    const TreeView<T>& tv = A.tv;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int64_t bt = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    if (bt >= A.sp.ntiles) return;  // warp-uniform
    const int n = A.sp.cnt[bt * 32 + lane];
    if (n == 0xFF) return;  // overflowed tile (every lane): the single-kernel pass owns it
    const int64_t tile = A.sp.tile0 + bt;
    const int64_t k = sample_of(A.src, tile, lane);
    const bool valid = k >= 0;
    T p[3] = {T(0), T(0), T(0)}, dd[3];
    if (valid) sample_coords(A.src, k, p, dd);
    const T ha = ((const T*)A.sp.ha)[bt * 32 + lane];
    const int kc = A.rec.kc;
    constexpr bool need_dg = DG;  // A.rec.need_dg (the launch picks the instantiation)

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
    Acc S1, G[3], Sw[KC], Sg[KC][3], Dm, Dg[3];
    CT a0[KC];
    bool have0 = false;
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

    // Kernel weights and sums of one pair; weights as in k_points.
    // (FP32C: every product rounded on its own, as in k_points; FP64 as written)
    auto mul = [](CT a, CT b) -> CT {
        if constexpr (std::is_same<CT, float>::value) return __fmul_rn(a, b);
        else return a * b;
    };
    auto sub = [](CT a, CT b) -> CT {
        if constexpr (std::is_same<CT, float>::value) return __fsub_rn(a, b);
        else return a - b;
    };
    auto accumulate = [&](const auto& col, CT dx, CT dy, CT dz, CT Wsum, CT csum, CT mr, CT mb) {
        const CT w = mul(mr, Wsum);
        const CT gc = mul(mr, csum);
        const CT gx = mul(gc, dx), gy = mul(gc, dy), gz = mul(gc, dz);
        S1.add(w);
        G[0].add(gx); G[1].add(gy); G[2].add(gz);
        if (SHIFT && !EXS && !have0) {
            have0 = true;
#pragma unroll
            for (int c = 0; c < KC; ++c)
                if (c < kc) a0[c] = (CT)col[c];
        }
#pragma unroll
        for (int c = 0; c < KC; ++c) {
            if (c < kc) {
                CT a = (CT)col[c];  // EXS: already A - A0
                if constexpr (SHIFT && !EXS) a = sub(a, a0[c]);
                Sw[c].add(mul(a, w));
                Sg[c][0].add(mul(a, gx)); Sg[c][1].add(mul(a, gy)); Sg[c][2].add(mul(a, gz));
            }
        }
        if (need_dg) {
            Dm.add(mul(mb, Wsum));
            const CT mc = mul(mb, csum);
            Dg[0].add(mul(mc, dx)); Dg[1].add(mul(mc, dy)); Dg[2].add(mul(mc, dz));
        }
    };

    // The pairs of this lane's list, one ahead: the loads of the next pair are
    // in flight while the current pair is summed.
    const float4* ent4 = A.sp.ent4 + (size_t)bt * RCAP * 32 + lane;
    const uint32_t* emask = A.sp.emask + (size_t)bt * RCAP * 32 + lane;
    const float* esh = EXS ? A.sp.eshift + (size_t)bt * RCAP * kc * 32 + lane : nullptr;
    int e = 0;
    unsigned m = 0;
    int64_t lo = 0;
    float Rs[3] = {0.f, 0.f, 0.f};
    float sh[KC];          // EXS: the entry's column shifts A[lo] - A0 (written by k_collect)
#pragma unroll
    for (int c = 0; c < KC; ++c) sh[c] = 0.f;
    PairData<T, BAND, KC> nx;
    bool hn = false;
    auto fetch = [&]() {
        if (m == 0 && e < n) {
            const float4 q = ent4[(size_t)e * 32];
            m = emask[(size_t)e * 32];  // never 0: k_collect writes entries with accepted leaves only
            ++e;
            lo = (int64_t)__float_as_int(q.w);
            Rs[0] = q.x; Rs[1] = q.y; Rs[2] = q.z;
            if constexpr (EXS) {
#pragma unroll
                for (int c = 0; c < KC; ++c) sh[c] = (c < kc) ? esh[((size_t)(e - 1) * kc + c) * 32] : 0.f;
            }
        }
        hn = m != 0;
        if (hn) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            nx.load(tv, A, lo + j, kc, need_dg, Rs, EXS ? A.colR : A.colF);
        }
    };
    unsigned long long n_bodyit = 0;
    fetch();
    while (__any_sync(PSB_FULL, hn)) {
        const bool hc = hn;
        PairData<T, BAND, KC> cur = nx;
        if constexpr (EXS) {
            // A - A0: the shifts of cur's entry (fetch may start the next one);
            // added here, an iteration after the loads, not as they return
#pragma unroll
            for (int c = 0; c < KC; ++c) cur.col[c] = __fadd_rn(cur.col[c], sh[c]);
        }
        fetch();
        ++n_bodyit;
        if (!hc) continue;
        if constexpr (BAND) {
            const float dx = __fsub_rn(cur.r[0], cur.L.x);
            const float dy = __fsub_rn(cur.r[1], cur.L.y);
            const float dz = __fsub_rn(cur.r[2], cur.L.z);
            float Wsum, csum;
            f32c_pair_weights<ST, KF>(
                tv.kern, tv.Kf, qe, dx, dy, dz, (float)ia, (float)sa3, (float)sa4, fa2, ika, (float)ha, cur.K, cur.L.w,
                [&]() {
                    const double ex = __dsub_rn((double)p[0], cur.xd);
                    const double ey = __dsub_rn((double)p[1], cur.yd);
                    const double ez = __dsub_rn((double)p[2], cur.zd);
                    return __fma_rn(ex, ex, __fma_rn(ey, ey, __dmul_rn(ez, ez)));
                },
                [&]() { return __dmul_rn(tv.Kd, cur.hd); }, Wsum, csum);
            accumulate(cur.col, dx, dy, dz, Wsum, csum, cur.K.w, cur.mb);
        } else {
            const T e2 = ex_d2_pp<T>(p, cur.x, cur.y, cur.z);
            const CT d2 = (CT)e2;
            const CT r = sqrt(d2);
            const CT invr = (d2 > CT(0)) ? CT(1) / r : CT(0);
            CT Wsum = CT(0), csum = CT(0);
            if (ST != ST_SCATTER) {
                CT f, df;
                kfdf<KF, CT>(tv.kern, r * ia, f, df);
                Wsum = sa3 * f;
                csum = sa4 * df * invr;
            }
            if (ST != ST_GATHER) {
                const CT hb = (CT)cur.h;
                CT ib = CT(1) / hb;
                CT sb3 = sig * ib * ib * ib;
                CT f, df;
                kfdf<KF, CT>(tv.kern, r * ib, f, df);
                CT Wb = sb3 * f, cb = sb3 * ib * df * invr;
                if (ST == ST_SCATTER) { Wsum = Wb; csum = cb; }
                else { Wsum = CT(0.5) * (Wsum + Wb); csum = CT(0.5) * (csum + cb); }
            }
            const CT mb = (CT)cur.m;
            const CT mr = (CT)((double)cur.m / (double)cur.rho);
            CT cc[KC];
#pragma unroll
            for (int c = 0; c < KC; ++c) cc[c] = (CT)cur.col[c];
            accumulate(cc, (CT)(p[0] - cur.x), (CT)(p[1] - cur.y), (CT)(p[2] - cur.z), Wsum, csum, mr, mb);
        }
    }

    if (valid) {
        // EXS: A0 are the column values of the first accepted leaf (the first
        // pair of the first entry)
        int64_t first = -1;
        if (EXS && n > 0) first = (int64_t)__float_as_int(ent4[0].w) + __ffs(emask[0]) - 1;
        double a0o[KC];
#pragma unroll
        for (int c = 0; c < KC; ++c)
            a0o[c] = EXS ? ((c < kc && first >= 0) ? (double)A.colT[c][first] : 0.0) : (double)a0[c];
        write_interp_outputs<T, Acc, CT, KC>(A, k, S1, G, Sw, Sg, Dm, Dg, a0o);
    }
    if (lane == 0 && A.stats) atomicAdd(&A.stats[5], n_bodyit);
}

}  // namespace psb
