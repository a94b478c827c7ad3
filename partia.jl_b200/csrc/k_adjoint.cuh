// k_adjoint.cuh -- adjoint (vector-Jacobian product) kernels for every kernel
// family: M4's Hessian is written out below (m4_whess), the others take f'/q
// and its q-derivative from kern_g12; the support K enters every radius rule.
//
// For a loss L = sum_s sum_k gout_k(s) out_k(s) the forward pass in FP64 first
// writes, per sample, the cotangents lambda of its sums (S1, G, Dm, Dg, Sw_c,
// Sg_c; write_sum_cotangents).  The kernels here then sum the pair terms per
// PARTICLE, so that every gradient is accumulated by one thread and no float
// atomics are needed:
//   dL/dm_b   = sum_s (aS W + aG.gradW) / rho_b + lDm W + lDg.gradW
//   dL/dA_c,b = sum_s m_b/rho_b (lSw_c W + lSg_c.gradW)
//   dL/dx_b   = -sum_s m_b/rho_b (aS gradW + H aG) + m_b (lDm gradW + H lDg)
// with aS = lS1 + sum_c lSw_c A_c,b, aG = lG + sum_c A_c,b lSg_c, W, gradW and
// the Hessian H of the kernel at delta = x_s - x_b (averaged over h_a and h_b
// in the symmetric strategy).  Densities and smoothing lengths are held fixed
// (h_a from the nearest particle is piecewise constant in the positions).
//
// Point samples: one warp per 32 Morton-consecutive particles walks a second
// LBVH built over the samples (node scale = subtree max of h_a) with the
// forward's radius rules seen from the particle, and re-decides every pair
// with the forward's exact arithmetic, so the pair set is the forward's.
// Parallel-beam lines: one thread per particle visits the pixels whose lines
// can pass within its support (the particle projected onto the frame plane)
// and re-decides each pair with the forward's line distance.
#pragma once

#include "k_points.cuh"

namespace psb {

// Pair lists of the two-kernel adjoint: one chain of blocks per tile of 32
// particles, taken from a pool with an atomic counter.  A block holds up to
// ADJ_CH entries per lane; an entry is a span of the sample tree (its first
// sample) and the mask of the samples that pair with the lane's particle.
// The warp takes a new block when any lane's is full, so where a chain's
// blocks begin and end follows from the walk alone.  A tile for which the
// pool runs out is marked and listed (the host grows the pool and walks
// again).
constexpr int ADJ_CH = 16;
struct AdjLists {
    uint2* ent;           // [block][ADJ_CH][32]: (first sample of the span, mask)
    uint8_t* bcnt;        // [block][32]: entries of each lane in the block
    int32_t* bnext;       // [block]: the tile's next block, -1 after its last
    int32_t* btile;       // [block]: the block's tile
    double* part;         // [block][8 + KC][32]: the block's partial sums (AdjAcc fields)
    int32_t* head;        // [tile]: first block, -1 without pairs, -2 overflowed
    unsigned* top;        // blocks taken
    int64_t nblocks;      // pool size
    int32_t* ovf_tiles;   // overflowed tiles
    unsigned* ovf_count;
};

struct AdjArgs {
    TreeView<double> pt;          // particles (Morton order)
    TreeView<double> sv;          // samples, in the order of their own LBVH; h = h_a
    const double* colT[MAX_KC];   // the catalog's distinct columns (particle Morton order)
    int kc;
    const double* lam;            // sum cotangents [q][sample] (sample-tree order for points)
    int64_t lam_stride;
    const int64_t* porder;        // particle Morton position -> caller's index
    double* gm;
    double* gx;
    double* gy;
    double* gz;
    double* gcol[MAX_KC];         // gradient of catalog column c (caller's order), may be null
    // parallel-beam lines
    SampleSrc<double> beam;
    int hmode;
    const double* hs;
    double ha_max;
    const double* lut;
    unsigned* err;
    unsigned long long* stats;    // [0] pairs, [2] walk steps
    // the two-kernel point path (k_adj_points' list form, k_adj_bodies, k_adj_combine)
    AdjLists al;
    const double* lamT;           // records of the samples for k_adj_bodies (AdjRec, sample-tree order)
    const int32_t* tile_list;     // k_adj_points over these particle tiles only (the lists' overflow), or null
    const unsigned* tile_count;
};

// M4 at delta = x_s - x_b: W, gradW = sigma/h^5 g1(q) delta and the Hessian
// (xx, yy, zz, xy, xz, yz) = sigma/h^5 (g1 I + g2 q delta delta^T / r^2), with
// g1 = f'(q)/q and g2 = d g1/dq (kernels/M4_spline.jl:13-36).  r = |delta|,
// ir = 1/r (0 at r = 0), h and invh = 1/h: 1/q = h ir, so no pair needs a
// division.  HESS = false leaves H untouched (scalar catalogs need W and
// gradW only).
template <bool HESS = true>
__device__ __forceinline__ void m4_whess(const double dl[3], double r, double ir, double h, double invh, double& W,
                                         double g[3], double H[6]) {
    const double q = r * invh;
    const double iq = h * ir;
    const double sig = inv_pi<double>();
    const double ih3 = invh * invh * invh, ih5 = ih3 * invh * invh;
    double f, g1, g2;
    if (q < 1.0) {
        f = 1.0 + q * q * (0.75 * q - 1.5);
        g1 = 2.25 * q - 3.0;
        g2 = 2.25;
    } else if (q < 2.0) {
        const double a = 2.0 - q;
        f = 0.25 * a * a * a;
        g1 = -0.75 * a * a * iq;
        g2 = 0.75 * a * (q + 2.0) * (iq * iq);
    } else {
        f = 0.0; g1 = 0.0; g2 = 0.0;
    }
    W = sig * ih3 * f;
    const double c = sig * ih5 * g1;
    g[0] = c * dl[0]; g[1] = c * dl[1]; g[2] = c * dl[2];
    if (!HESS) return;
    const double e = sig * ih5 * g2 * q * (ir * ir);  // 0 at r = 0 (ir = 0)
    H[0] = c + e * dl[0] * dl[0]; H[1] = c + e * dl[1] * dl[1]; H[2] = c + e * dl[2] * dl[2];
    H[3] = e * dl[0] * dl[1]; H[4] = e * dl[0] * dl[2]; H[5] = e * dl[1] * dl[2];
}

// The same for a kernel other than M4 (id k, 3D norm sig): f from kern_fdf,
// g1 = f'(q)/q and g2 = d g1/dq from kern_g12, with 1/q = h ir.
template <bool HESS = true>
__device__ __forceinline__ void kern_whess(int k, double sig, const double dl[3], double r, double ir, double h,
                                           double invh, double& W, double g[3], double H[6]) {
    const double q = r * invh;
    double f, df, g1, g2;
    kern_fdf<double>(k, q, f, df);
    kern_g12(k, q, h * ir, g1, g2);
    const double ih3 = invh * invh * invh, ih5 = ih3 * invh * invh;
    W = sig * ih3 * f;
    const double c = sig * ih5 * g1;
    g[0] = c * dl[0]; g[1] = c * dl[1]; g[2] = c * dl[2];
    if (!HESS) return;
    const double e = sig * ih5 * g2 * q * (ir * ir);  // 0 at r = 0 (ir = 0)
    H[0] = c + e * dl[0] * dl[0]; H[1] = c + e * dl[1] * dl[1]; H[2] = c + e * dl[2] * dl[2];
    H[3] = e * dl[0] * dl[1]; H[4] = e * dl[0] * dl[2]; H[5] = e * dl[1] * dl[2];
}

// W, gradW (and H) of the context's kernel: KF = 0 is the M4 code, KF = 1 any
// other family (the warp-uniform id in pt.kern)
template <int KF, bool HESS>
__device__ __forceinline__ void whess(const TreeView<double>& pt, const double dl[3], double r, double ir, double h,
                                      double invh, double& W, double g[3], double H[6]) {
    if constexpr (KF == 0) m4_whess<HESS>(dl, r, ir, h, invh, W, g, H);
    else kern_whess<HESS>(pt.kern, (double)pt.sig, dl, r, ir, h, invh, W, g, H);
}

__device__ __forceinline__ void hmul(const double H[6], const double v[3], double o[3]) {
    o[0] = H[0] * v[0] + H[3] * v[1] + H[4] * v[2];
    o[1] = H[3] * v[0] + H[1] * v[1] + H[5] * v[2];
    o[2] = H[4] * v[0] + H[5] * v[1] + H[2] * v[2];
}

// Per-particle sums of the pair terms; the particle's factors 1/rho_b,
// m_b/rho_b and m_b are applied once after its last pair:
// dL/dm_b = sW / rho_b + sD, dL/dA_c,b = m_b/rho_b sA_c,
// dL/dx_b = -(m_b/rho_b vS + m_b vD)
template <int KC> struct AdjAcc {
    static constexpr int NF = 8 + KC;  // fields, in the order of f()
    double sW, sD, vS[3], vD[3], sA[KC];
    __device__ __forceinline__ void zero() {
        sW = 0.0; sD = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) { vS[d] = 0.0; vD[d] = 0.0; }
#pragma unroll
        for (int c = 0; c < KC; ++c) sA[c] = 0.0;
    }
    // field i: sW, sD, vS (3), vD (3), sA (KC)
    __device__ __forceinline__ double& f(int i) {
        return i == 0 ? sW : (i == 1 ? sD : (i < 5 ? vS[i - 2] : (i < 8 ? vD[i - 5] : sA[i - 8])));
    }
};

// The sum cotangents of a pair's sample, by meaning: S1, G (3), Dm, Dg (3),
// Sw_c, Sg_c (3 per column); a scalar catalog (SCAL) has S1 and Sw_c only.
// RowsStrided reads compact row r at ls[r * rs] (rows S1, G, Dm, Dg, Sw_c,
// Sg_c in that order, kc columns; SCAL: S1, Sw_c): the staged rows of
// k_adj_points or the global cotangent rows.
struct RowsStrided {
    const double* ls;
    int64_t rs;
    int kc;
    template <bool SCAL> __device__ __forceinline__ double S1() const { return ls[0]; }
    __device__ __forceinline__ double G(int d) const { return ls[(1 + d) * rs]; }
    __device__ __forceinline__ double Dm() const { return ls[4 * rs]; }
    __device__ __forceinline__ double Dg(int d) const { return ls[(5 + d) * rs]; }
    template <bool SCAL> __device__ __forceinline__ double Sw(int c) const { return ls[((SCAL ? 1 : 8) + c) * rs]; }
    __device__ __forceinline__ double Sg(int c, int d) const { return ls[(8 + kc + 3 * c + d) * rs]; }
};
// Per-sample records of k_adj_bodies: x, y, z, h_a, 1/h_a, 0, then the sum
// cotangents with the columns at fixed places for KC columns (those past the
// catalog's kc are 0), padded to whole 16-byte pairs: one record is read with
// 128-bit loads, where separate arrays would take a 32-byte sector per value.
template <int KC, bool SCAL> struct AdjRec {
    static constexpr int NQ = SCAL ? 1 + KC : 8 + 4 * KC;
    static constexpr int N = 6 + ((NQ + 1) & ~1);  // doubles per record
};
template <int KC, bool SCAL> struct RowsRec {
    double q[AdjRec<KC, SCAL>::N - 6];
    template <bool S> __device__ __forceinline__ double S1() const { return q[0]; }
    __device__ __forceinline__ double G(int d) const { return q[1 + d]; }
    __device__ __forceinline__ double Dm() const { return q[4]; }
    __device__ __forceinline__ double Dg(int d) const { return q[5 + d]; }
    template <bool S> __device__ __forceinline__ double Sw(int c) const { return q[(S ? 1 : 8) + c]; }
    __device__ __forceinline__ double Sg(int c, int d) const { return q[8 + KC + 3 * c + d]; }
};

// The terms of one pair (sample at (sxv, syv, szv) with h_a = ha, 1/ha = iha;
// particle xb, hb, ihb = 1/hb, columns Ab) with the sample's sum cotangents R.
template <int ST, int KC, bool SCAL, int KF, class Rows>
__device__ __forceinline__ void adj_pair(const TreeView<double>& pt, const double xb[3], double hb, double ihb,
                                         const double (&Ab)[KC], int kc, double sxv, double syv, double szv, double ha,
                                         double iha, const Rows& R, AdjAcc<KC>& S) {
    const double dl[3] = {sxv - xb[0], syv - xb[1], szv - xb[2]};
    const double r2 = dl[0] * dl[0] + dl[1] * dl[1] + dl[2] * dl[2];
    const double ir = (r2 > 0.0) ? rsqrt(r2) : 0.0;
    const double r = r2 * ir;
    double W, g[3], H[6];
    if (ST == ST_GATHER) {
        whess<KF, !SCAL>(pt, dl, r, ir, ha, iha, W, g, H);
    } else if (ST == ST_SCATTER) {
        whess<KF, !SCAL>(pt, dl, r, ir, hb, ihb, W, g, H);
    } else {
        double Wa, ga3[3], Ha[6], Wb, gb3[3], Hb[6];
        whess<KF, !SCAL>(pt, dl, r, ir, ha, iha, Wa, ga3, Ha);
        whess<KF, !SCAL>(pt, dl, r, ir, hb, ihb, Wb, gb3, Hb);
        W = 0.5 * (Wa + Wb);
        for (int d = 0; d < 3; ++d) g[d] = 0.5 * (ga3[d] + gb3[d]);
        if (!SCAL)
            for (int d = 0; d < 6; ++d) H[d] = 0.5 * (Ha[d] + Hb[d]);
    }
    if constexpr (SCAL) {
        double aS = R.template S1<SCAL>();
#pragma unroll
        for (int c = 0; c < KC; ++c) {
            if (c < kc) {
                const double lsw = R.template Sw<SCAL>(c);
                aS += lsw * Ab[c];
                S.sA[c] += lsw * W;
            }
        }
        S.sW += aS * W;
        for (int d = 0; d < 3; ++d) S.vS[d] += aS * g[d];
        return;
    }
    const double lS1 = R.template S1<SCAL>();
    const double lG[3] = {R.G(0), R.G(1), R.G(2)};
    const double lDm = R.Dm();
    const double lDg[3] = {R.Dg(0), R.Dg(1), R.Dg(2)};
    double aS = lS1, aG[3] = {lG[0], lG[1], lG[2]};
#pragma unroll
    for (int c = 0; c < KC; ++c) {
        if (c < kc) {
            const double lsw = R.template Sw<SCAL>(c);
            const double lsg[3] = {R.Sg(c, 0), R.Sg(c, 1), R.Sg(c, 2)};
            aS += lsw * Ab[c];
            aG[0] += Ab[c] * lsg[0]; aG[1] += Ab[c] * lsg[1]; aG[2] += Ab[c] * lsg[2];
            S.sA[c] += lsw * W + lsg[0] * g[0] + lsg[1] * g[1] + lsg[2] * g[2];
        }
    }
    S.sW += aS * W + aG[0] * g[0] + aG[1] * g[1] + aG[2] * g[2];
    S.sD += lDm * W + lDg[0] * g[0] + lDg[1] * g[1] + lDg[2] * g[2];
    double Ha[3], Hd[3];
    hmul(H, aG, Ha);
    hmul(H, lDg, Hd);
    for (int d = 0; d < 3; ++d) {
        S.vS[d] += aS * g[d] + Ha[d];
        S.vD[d] += lDm * g[d] + Hd[d];
    }
}

// the gradients of particle b (Morton position) from its sums
template <int KC>
__device__ __forceinline__ void adj_write(const AdjArgs& A, int64_t b, const AdjAcc<KC>& S, double mb, double rhob,
                                          int kc) {
    const double mr = mb / rhob;
    const int64_t o = A.porder[b];
    A.gm[o] = S.sW / rhob + S.sD;
    A.gx[o] = -(mr * S.vS[0] + mb * S.vD[0]);
    A.gy[o] = -(mr * S.vS[1] + mb * S.vD[1]);
    A.gz[o] = -(mr * S.vS[2] + mb * S.vD[2]);
#pragma unroll
    for (int c = 0; c < KC; ++c)
        if (c < kc && A.gcol[c]) A.gcol[c][o] = mr * S.sA[c];
}

struct AStage {
    double sx[SPAN], sy[SPAN], sz[SPAN], sh[SPAN];  // samples of the span, h_a
    double sih[SPAN];                               // 1 / h_a
    float4 Q[SPAN];   // the samples relative to the warp anchor, float h_a
    float2 AB[SPAN];  // their squared radius thresholds (surely in, maybe in)
    float4 PP[SPAN];  // the warp's particles relative to the warp anchor
    float2 PAB[SPAN]; // their squared radius thresholds
};

// SCAL: every output of the catalog is a (plain or Shepard) scalar, so only
// lambda_S1 and lambda_Sw_c can be non-zero: the pair terms drop the Hessian
// and the gradient cotangents (the same values as the general form, which
// adds exact zeros).
// A pair reads 8 + 4 kc sum cotangents of its sample (1 + kc for scalar
// catalogs: lambda_S1 and lambda_Sw_c).  Every particle of the warp that pairs
// with a sample reads the same ones, so they are staged in shared memory once
// per span, one coalesced load per row.  The general form stages up to 4
// columns (24 rows of 32 doubles per warp); with 8 it would pass the 48 KB of
// static shared memory of a block and reads them from global memory instead.
template <int KC, bool SCAL> struct ALam {
    double q[(SCAL ? 1 + KC : 8 + 4 * KC) * SPAN];  // staged row r of span sample j at r * SPAN + j
};
// the cotangent row (in A.lam) of staged row r
template <bool SCAL> __device__ __forceinline__ int lam_row(int r) { return SCAL ? (r == 0 ? 0 : 7 + r) : r; }

// COL: the pair-list pass of the two-kernel path (the list form): the same
// walk and pair decisions, with each lane's accepted samples of a span
// written to its tile's chain of list blocks instead of summed.
template <int ST, int KC, bool SCAL, int KF, bool COL = false>
__global__ void __launch_bounds__(128, (COL || SCAL) ? 8 : 4) k_adj_points(const AdjArgs A) {
    __shared__ AStage stage_all[4];
    constexpr bool STAGE = !COL && (SCAL || KC <= 4);
    __shared__ ALam<STAGE ? KC : 1, SCAL> lam_all[STAGE ? 4 : 1];
    const TreeView<double>& pt = A.pt;
    const TreeView<double>& sv = A.sv;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    AStage& st = stage_all[wib];
    int64_t tile = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    if (A.tile_list) {  // the tiles the two-kernel path handed back
        if (tile >= (int64_t)*A.tile_count) return;
        tile = A.tile_list[tile];
    }
    if (tile * 32 >= pt.n) return;  // warp-uniform
    const int64_t b = tile * 32 + lane;
    const bool valid = b < pt.n;
    double xb[3] = {0.0, 0.0, 0.0}, hb = 0.0, mb = 0.0, rhob = 1.0, Ab[KC];
#pragma unroll
    for (int c = 0; c < KC; ++c) Ab[c] = 0.0;
    if (valid) {
        xb[0] = pt.x[b]; xb[1] = pt.y[b]; xb[2] = pt.z[b];
        hb = pt.h[b]; mb = pt.m[b]; rhob = pt.rho[b];
#pragma unroll
        for (int c = 0; c < KC; ++c)
            if (c < A.kc) Ab[c] = A.colT[c][b];
    }
    // the support K (2 for M4) in double and float, and the float margin of
    // K h: 2 h is exact in float, K h in general one rounding away
    const double Kd = (KF == 0) ? 2.0 : pt.Kd;
    const float Kf = (KF == 0) ? 2.f : pt.Kf;
    const float km = (KF == 0) ? 2.f * U1 : 3.f * U1;
    // this particle's own support radius^2, with the forward's operation order
    const double rb = X<double>::mul(Kd, hb);
    const double rb2 = X<double>::mul(rb, rb);
    // float pair tests against a band (as in the forward's float walk): the
    // particle relative to the warp anchor (the first valid particle) with its
    // rounding error, its radius bounds and the warp-wide maxima of both
    const unsigned vmask = __ballot_sync(PSB_FULL, valid);
    const int first = vmask ? __ffs(vmask) - 1 : 0;
    const double cw[3] = {__shfl_sync(PSB_FULL, xb[0], first), __shfl_sync(PSB_FULL, xb[1], first),
                          __shfl_sync(PSB_FULL, xb[2], first)};
    const float P[3] = {(float)(xb[0] - cw[0]), (float)(xb[1] - cw[1]), (float)(xb[2] - cw[2])};
    float esmax = U1 * (fabsf(P[0]) + fabsf(P[1]) + fabsf(P[2])) + 1e-30f;
    float rblo = 0.f, rbmax = 0.f;
    if (ST != ST_GATHER) {
        rblo = __double2float_rd(rb) * (1.f - 2.f * U1);
        rbmax = __double2float_ru(rb) * (1.f + 2.f * U1);
    }
    const float rbhi = rbmax;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        esmax = fmaxf(esmax, __shfl_xor_sync(PSB_FULL, esmax, o));
        rbmax = fmaxf(rbmax, __shfl_xor_sync(PSB_FULL, rbmax, o));
    }
    const double ihb = 1.0 / hb;
    AdjAcc<KC> S;
    S.zero();
    const int kc = A.kc;
    const int64_t L = A.lam_stride;
    unsigned long long n_pairs = 0, n_spans = 0, n_parts = 0, n_leaves = 0;  // work counters (warp-uniform)
    int64_t steps = 0;

    const double* lst = lam_all[STAGE ? wib : 0].q;  // the span's staged cotangents
    // li: the sample; jj: its slot in the span
    auto pair = [&](int64_t li, int jj, double sxv, double syv, double szv, double ha, double iha) {
        ++n_pairs;
        // row r of this sample: staged, or from global memory
        const RowsStrided R{STAGE ? lst + jj : A.lam + li, STAGE ? (int64_t)SPAN : L, kc};
        adj_pair<ST, KC, SCAL, KF>(pt, xb, hb, ihb, Ab, kc, sxv, syv, szv, ha, iha, R, S);
    };

    // COL: this tile's chain of list blocks (block, this lane's entries in it)
    int64_t blk = -1;
    int pos = 0;
    bool dead = false;  // the pool ran out: the tile is listed for k_adj_points
    auto emit = [&](int64_t lo, unsigned acc) {
        const bool want = acc != 0;
        if (dead || !__any_sync(PSB_FULL, want)) return;
        if (blk < 0 || __any_sync(PSB_FULL, want && pos == ADJ_CH)) {  // a new block for the warp
            unsigned long long nb = 0;
            if (lane == 0) nb = atomicAdd(A.al.top, 1u);
            nb = __shfl_sync(PSB_FULL, nb, 0);
            if ((int64_t)nb >= A.al.nblocks) {
                dead = true;
                return;
            }
            if (blk >= 0) {
                A.al.bcnt[blk * 32 + lane] = (uint8_t)pos;
                if (lane == 0) A.al.bnext[blk] = (int32_t)nb;
            } else if (lane == 0) {
                A.al.head[tile] = (int32_t)nb;
            }
            if (lane == 0) A.al.btile[nb] = (int32_t)tile;
            blk = (int64_t)nb;
            pos = 0;
        }
        if (want) {
            A.al.ent[((size_t)blk * ADJ_CH + pos) * 32 + lane] = make_uint2((unsigned)lo, acc);
            ++pos;
        }
    };

    // node test seen from the particle, on the float node records (box
    // rounded outwards, scale = max h_a rounded up): the largest sample radius
    // in the node for gather, the particle's own for scatter, the larger for
    // symmetric.  A lower bound of the distance against an upper bound of
    // the radius never prunes a node holding a pair (the pair test itself
    // stays exact).
    const float pf[3] = {(float)xb[0], (float)xb[1], (float)xb[2]};
    const float pem = U1 * fmaxf(fmaxf(fabsf(pf[0]), fabsf(pf[1])), fabsf(pf[2])) + 1e-30f;
    const float rb2_hi = __double2float_ru(rb2) * (1.f + RELM);
    constexpr int SN = (ST == ST_GATHER) ? ST_SCATTER : ((ST == ST_SCATTER) ? ST_GATHER : ST_SYMMETRIC);
    auto node_fn = [&](int ni) -> bool {
        const float4 lo = __ldg(&sv.node_lo[ni]), hi = __ldg(&sv.node_hi[ni]);
        return !(lb_d2_pbox(pf, pem, lo, hi) > hi_r2_node<SN>(rb2_hi, lo.w, Kf));
    };
    auto span_fn = [&](int64_t lo, int cnt, bool part) {
        const unsigned parts = __ballot_sync(PSB_FULL, part);
        if (!parts) return;
        ++n_spans;
        n_parts += __popc(parts);
        n_leaves += cnt;
        // one error bound E for every float distance of the span (the
        // samples are stored relative to the span's first sample)
        const float o0 = (float)(__ldg(&sv.x[lo]) - cw[0]);
        const float o1 = (float)(__ldg(&sv.y[lo]) - cw[1]);
        const float o2 = (float)(__ldg(&sv.z[lo]) - cw[2]);
        const float2 sb = __ldg(&sv.spanb[lo]);
        const float eqm = U1 * (2.f * sb.x + 2.f * (fabsf(o0) + fabsf(o1) + fabsf(o2))) * (1.f + 4.f * U1);
        float rmax = rbmax;
        if (ST != ST_SCATTER) rmax = fmaxf(rmax, Kf * sb.y * (1.f + km));
        const float E = 1.7320508f * (esmax + eqm) + 4.f * U1 * rmax + 1e-30f;
        // squared radius thresholds of this lane's particle and of sample
        // `lane` (surely in: d2 < A; maybe in: d2 <= B)
        float As = 0.f, Bs = 0.f, Aj = 0.f, Bj = 0.f;
        if (ST != ST_GATHER) {  // the particle's own radius K h_b
            const float il = fmaxf((rblo - E) * (1.f - 4.f * U1), 0.f), ih = (rbhi + E) * (1.f + 4.f * U1);
            As = il * il;
            Bs = ih * ih;
        }
        float4 Qme = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncwarp();
        if (lane < cnt) {
            st.sx[lane] = __ldg(&sv.x[lo + lane]); st.sy[lane] = __ldg(&sv.y[lo + lane]);
            st.sz[lane] = __ldg(&sv.z[lo + lane]); st.sh[lane] = __ldg(&sv.h[lo + lane]);
            if (!COL) st.sih[lane] = 1.0 / st.sh[lane];
            const float4 Lq = __ldg(&sv.leaf4[lo + lane]);
            Qme = make_float4(Lq.x + o0, Lq.y + o1, Lq.z + o2, Lq.w);
            st.Q[lane] = Qme;
            if (ST != ST_SCATTER) {  // the sample's radius K h_a
                const float rahi = Kf * Lq.w * (1.f + km), ralo = Kf * Lq.w * (1.f - km);
                const float il = fmaxf((ralo - E) * (1.f - 4.f * U1), 0.f), ih = (rahi + E) * (1.f + 4.f * U1);
                Aj = il * il;
                Bj = ih * ih;
                st.AB[lane] = make_float2(Aj, Bj);
            }
        }
        const int np = __popc(parts);
        const bool by_particle = 3 * np >= 2 * cnt;  // warp-uniform
        if (!by_particle) {
            st.PP[lane] = make_float4(P[0], P[1], P[2], 0.f);
            st.PAB[lane] = make_float2(As, Bs);
        }
        __syncwarp();
        unsigned acc = 0, maybe = 0;
        if (!by_particle) {
            // few particles take part: sample `lane` against each of them
            for (unsigned pp = parts; pp; pp &= pp - 1) {
                const int s = __ffs(pp) - 1;
                const float4 Pp = st.PP[s];
                const float2 ab = st.PAB[s];
                const float dx = Pp.x - Qme.x, dy = Pp.y - Qme.y, dz = Pp.z - Qme.z;
                const float d2 = dx * dx + dy * dy + dz * dz;
                const float At = (ST == ST_GATHER) ? Aj : ((ST == ST_SCATTER) ? ab.x : fmaxf(ab.x, Aj));
                const float Bt = (ST == ST_GATHER) ? Bj : ((ST == ST_SCATTER) ? ab.y : fmaxf(ab.y, Bj));
                const unsigned bi = __ballot_sync(PSB_FULL, lane < cnt && d2 < At);
                const unsigned bm = __ballot_sync(PSB_FULL, lane < cnt && d2 <= Bt);
                if (lane == s) { acc = bi; maybe = bm; }
            }
        } else if (part) {
            // this lane's particle against every sample of the span
#pragma unroll 4
            for (int j = 0; j < cnt; ++j) {
                const float4 Q = st.Q[j];
                const float dx = P[0] - Q.x, dy = P[1] - Q.y, dz = P[2] - Q.z;
                const float d2 = dx * dx + dy * dy + dz * dz;
                float At = As, Bt = Bs;
                if (ST != ST_SCATTER) {
                    const float2 ab = st.AB[j];
                    At = (ST == ST_GATHER) ? ab.x : fmaxf(As, ab.x);
                    Bt = (ST == ST_GATHER) ? ab.y : fmaxf(Bs, ab.y);
                }
                acc |= (unsigned)(d2 < At) << j;
                maybe |= (unsigned)(d2 <= Bt) << j;
            }
        }
        // undecided pairs: the forward's exact test
        for (unsigned u = maybe & ~acc; u; u &= u - 1) {
            const int jj = __ffs(u) - 1;
            const double ps[3] = {st.sx[jj], st.sy[jj], st.sz[jj]};
            const double ra = X<double>::mul(Kd, st.sh[jj]);
            const double ra2 = X<double>::mul(ra, ra);
            const double e2 = ex_d2_pp<double>(ps, xb[0], xb[1], xb[2]);
            if (e2 <= ex_r2<ST, double>(ra2, hb, Kd)) acc |= 1u << jj;
        }
        if constexpr (COL) {
            emit(lo, acc);
        } else {
            if constexpr (STAGE) {  // stage the span's cotangent rows (a warp-uniform decision)
                if (__any_sync(PSB_FULL, acc != 0)) {
                    double* lw = lam_all[wib].q;
                    const int nq = SCAL ? 1 + kc : 8 + 4 * kc;
                    if (lane < cnt)
                        for (int r = 0; r < nq; ++r)
                            lw[r * SPAN + lane] = __ldg(&A.lam[lam_row<SCAL>(r) * L + lo + lane]);
                    __syncwarp();
                }
            }
            for (; acc; acc &= acc - 1) {
                const int jj = __ffs(acc) - 1;
                pair(lo + jj, jj, st.sx[jj], st.sy[jj], st.sz[jj], st.sh[jj], st.sih[jj]);
            }
            if constexpr (STAGE) __syncwarp();  // the rows are read before the next span's
        }
    };
    const int32_t start = (sv.root == 0) ? (int32_t)sv.n : sv.root;
    const bool ok = warp_traverse_spans(start, sv.n, sv.links, sv.escape, valid, node_fn, span_fn, steps);

    if constexpr (COL) {
        if (dead) {
            if (lane == 0) {
                A.al.head[tile] = -2;
                A.al.ovf_tiles[atomicAdd(A.al.ovf_count, 1u)] = (int32_t)tile;
            }
        } else if (blk >= 0) {
            A.al.bcnt[blk * 32 + lane] = (uint8_t)pos;
            if (lane == 0) A.al.bnext[blk] = -1;
        } else if (lane == 0) {
            A.al.head[tile] = -1;
        }
    } else if (valid) {
        adj_write<KC>(A, b, S, mb, rhob, kc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n_pairs += __shfl_xor_sync(PSB_FULL, n_pairs, o);
    if (lane == 0 && A.stats) {
        atomicAdd(&A.stats[0], n_pairs);
        atomicAdd(&A.stats[2], (unsigned long long)steps);
        atomicAdd(&A.stats[3], n_spans);
        atomicAdd(&A.stats[4], n_parts);
        atomicAdd(&A.stats[5], n_leaves);
    }

    if (!ok && lane == 0) atomicOr(A.err, PSB_DERR_TRAVERSAL);
}

// The pair terms of the two-kernel path, one list block per warp: lane j
// sums the pairs of the block's entries of particle j of the block's tile
// (its own partial sums, from zero) and stores them with the block.  A block
// holds at most ADJ_CH entries per lane, so the work items are of like size
// however long a particle's list is: a tile of large-h particles in the
// outskirts (pair lists 60 times the mean tile's) spreads over as many warps
// as it has blocks, where one warp per tile left it running long after the
// others.  Each pair reads its sample as one record (AdjRec) with 128-bit
// loads.
template <int ST, int KC, bool SCAL, int KF>
__global__ void __launch_bounds__(128, 4) k_adj_bodies(const AdjArgs A) {
    const TreeView<double>& pt = A.pt;
    const int lane = threadIdx.x & 31;
    const int64_t blk = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int64_t used = (int64_t)*A.al.top;
    if (blk >= (used < A.al.nblocks ? used : A.al.nblocks)) return;  // warp-uniform
    const int64_t tile = A.al.btile[blk];
    // A tile the pool ran out on is k_adj_points' (its last block's counts
    // were never written): skip its blocks.
    if (A.al.head[tile] == -2) return;  // warp-uniform
    const int64_t b = tile * 32 + lane;
    const bool valid = b < pt.n;
    const int kc = A.kc;
    double xb[3] = {0.0, 0.0, 0.0}, hb = 1.0, Ab[KC];
#pragma unroll
    for (int c = 0; c < KC; ++c) Ab[c] = 0.0;
    if (valid) {
        xb[0] = pt.x[b]; xb[1] = pt.y[b]; xb[2] = pt.z[b];
        hb = pt.h[b];
#pragma unroll
        for (int c = 0; c < KC; ++c)
            if (c < kc) Ab[c] = A.colT[c][b];
    }
    const double ihb = 1.0 / hb;
    AdjAcc<KC> P;
    P.zero();
    const int ne = valid ? A.al.bcnt[blk * 32 + lane] : 0;
    int e = 0;
    unsigned m = 0;
    int64_t lo = 0;
    auto next = [&]() -> bool {  // the next pair: sample lo + ffs(m) - 1
        while (m == 0) {
            if (e >= ne) return false;
            const uint2 q = A.al.ent[((size_t)blk * ADJ_CH + e) * 32 + lane];
            lo = (int64_t)q.x;
            m = q.y;
            ++e;
        }
        return true;
    };
    unsigned long long n_pairs = 0;
    bool has = next();
    while (__any_sync(PSB_FULL, has)) {
        if (has) {
            const int64_t s = lo + __ffs(m) - 1;
            m &= m - 1;
            ++n_pairs;
            using RC = AdjRec<KC, SCAL>;
            const double2* rp = reinterpret_cast<const double2*>(A.lamT + s * RC::N);
            const double2 h0 = __ldg(rp), h1 = __ldg(rp + 1), h2 = __ldg(rp + 2);
            RowsRec<KC, SCAL> R;
#pragma unroll
            for (int k = 0; k < (RC::N - 6) / 2; ++k) {
                const double2 v = __ldg(rp + 3 + k);
                R.q[2 * k] = v.x;
                R.q[2 * k + 1] = v.y;
            }
            adj_pair<ST, KC, SCAL, KF>(pt, xb, hb, ihb, Ab, kc, h0.x, h0.y, h1.x, h1.y, h2.x, R, P);
            has = next();
        }
    }
    if (A.al.head[tile] == blk && A.al.bnext[blk] < 0) {
        // the tile's only block: its sums are the particles' (k_adj_combine
        // starts from the first block's sums, so both give the same bits)
        if (valid) adj_write<KC>(A, b, P, pt.m[b], pt.rho[b], kc);
    } else {
        double* o = A.al.part + (size_t)blk * AdjAcc<KC>::NF * 32 + lane;
#pragma unroll
        for (int f = 0; f < AdjAcc<KC>::NF; ++f) o[(size_t)f * 32] = P.f(f);
    }
#pragma unroll
    for (int q = 16; q > 0; q >>= 1) n_pairs += __shfl_xor_sync(PSB_FULL, n_pairs, q);
    if (lane == 0 && A.stats) atomicAdd(&A.stats[6], n_pairs);
}

// The gradients of each particle of a tile of several blocks (and zeros for
// a tile without pairs): its blocks' partial sums added in the order of its
// tile's chain (the order the walk met the spans), then the particle's
// factors (adj_write).  The blocks' boundaries follow from the
// walk, so the result does not depend on the pool or on which block landed
// where in it.
template <int KC>
__global__ void __launch_bounds__(128) k_adj_combine(const AdjArgs A) {
    const TreeView<double>& pt = A.pt;
    const int lane = threadIdx.x & 31;
    const int64_t tile = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (tile * 32 >= pt.n) return;
    const int64_t b = tile * 32 + lane;
    if (b >= pt.n) return;
    int64_t blk = A.al.head[tile];
    if (blk == -2) return;  // overflowed: k_adj_points owns the tile
    AdjAcc<KC> T;
    T.zero();
    if (blk >= 0) {
        int64_t nxt = A.al.bnext[blk];
        if (nxt < 0) return;  // one block: k_adj_bodies wrote the gradients
        const double* o = A.al.part + (size_t)blk * AdjAcc<KC>::NF * 32 + lane;
#pragma unroll
        for (int f = 0; f < AdjAcc<KC>::NF; ++f) T.f(f) = o[(size_t)f * 32];
        for (blk = nxt; blk >= 0; blk = A.al.bnext[blk]) {
            o = A.al.part + (size_t)blk * AdjAcc<KC>::NF * 32 + lane;
#pragma unroll
            for (int f = 0; f < AdjAcc<KC>::NF; ++f) T.f(f) += o[(size_t)f * 32];
        }
    }
    adj_write<KC>(A, b, T, pt.m[b], pt.rho[b], A.kc);
}

// The records of k_adj_bodies (AdjRec), one per sample of the sample tree:
// position, h_a, 1/h_a and the sum cotangents (lam: rows [q][sample] in the
// tree's order) at the record's fixed places.
template <int KC, bool SCAL>
__global__ void k_adj_rows(const double* lam, int64_t ns, int kc, const TreeView<double> sv, double* rec) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    using RC = AdjRec<KC, SCAL>;
    double* o = rec + i * RC::N;
    const double h = sv.h[i];
    o[0] = sv.x[i]; o[1] = sv.y[i]; o[2] = sv.z[i]; o[3] = h; o[4] = 1.0 / h;
    for (int r = 5; r < RC::N; ++r) o[r] = 0.0;
    double* q = o + 6;
    auto row = [&](int r) { return lam[(int64_t)r * ns + i]; };  // compact row r (kc columns)
    if (SCAL) {
        q[0] = row(0);
        for (int c = 0; c < kc; ++c) q[1 + c] = row(8 + c);  // lambda_Sw_c
    } else {
        for (int r = 0; r < 8; ++r) q[r] = row(r);
        for (int c = 0; c < kc; ++c) {
            q[8 + c] = row(8 + c);
            for (int d = 0; d < 3; ++d) q[8 + KC + 3 * c + d] = row(8 + kc + 3 * c + d);
        }
    }
}

// line-integrated kernel and its r-derivative: the slope of the table segment
// that line_W interpolates on (LUT_N entries over [0, K], K the support)
__device__ __forceinline__ void line_Wd(double r, double h, const double* lut, double K, double& W, double& dW) {
    const double invh = 1.0 / h;
    const double q = r * invh;
    if (q >= K) { W = 0.0; dW = 0.0; return; }
    const double dq = K / (double)(LUT_N - 1);
    const double idxf = q / dq + 1.0;
    int i = (int)idxf;
    i = i < 1 ? 1 : (i > LUT_N - 1 ? LUT_N - 1 : i);
    const double t = idxf - (double)i;
    W = invh * (lut[i - 1] * (1.0 - t) + lut[i] * t);
    dW = invh * invh * (lut[i] - lut[i - 1]) / dq;
}

template <int ST, int KC>
__global__ void __launch_bounds__(128) k_adj_beam(const AdjArgs A) {
    const TreeView<double>& pt = A.pt;
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= pt.n) return;
    const double xb[3] = {pt.x[b], pt.y[b], pt.z[b]};
    const double hb = pt.h[b], mb = pt.m[b], rhob = pt.rho[b], mr = mb / rhob;
    const int kc = A.kc;
    double Ab[KC];
#pragma unroll
    for (int c = 0; c < KC; ++c) Ab[c] = (c < kc) ? A.colT[c][b] : 0.0;
    const SampleSrc<double>& B = A.beam;
    const double* f = B.frame;
    // the particle on the frame plane (frame axes orthonormal)
    const double v[3] = {xb[0] - f[0], xb[1] - f[1], xb[2] - f[2]};
    const double xi = v[0] * f[3] + v[1] * f[4] + v[2] * f[5];
    const double eta = v[0] * f[6] + v[1] * f[7] + v[2] * f[8];
    const double K = pt.Kd;  // the support (2 for M4)
    const double R = K * fmax(hb, A.ha_max) * (1.0 + 1e-9) + 1e-300;
    const double dxi = (B.params[1] - B.params[0]) / (double)(B.nx - 1);
    const double deta = (B.params[3] - B.params[2]) / (double)(B.ny - 1);
    auto range = [](double c, double R, double lo0, double d, int64_t n, int64_t& a, int64_t& z) {
        double u0 = (c - R - lo0) / d, u1 = (c + R - lo0) / d;
        if (u0 > u1) { double t = u0; u0 = u1; u1 = t; }
        u0 = floor(u0) - 1.0;
        u1 = ceil(u1) + 1.0;
        a = u0 < 0.0 ? 0 : (u0 > (double)(n - 1) ? n : (int64_t)u0);
        z = u1 > (double)(n - 1) ? n - 1 : (u1 < 0.0 ? -1 : (int64_t)u1);
    };
    int64_t i0, i1, j0, j1;
    range(xi, R, B.params[0], dxi, B.nx, i0, i1);
    range(eta, R, B.params[2], deta, B.ny, j0, j1);
    double gm = 0.0, gx[3] = {0.0, 0.0, 0.0}, ga[KC];
#pragma unroll
    for (int c = 0; c < KC; ++c) ga[c] = 0.0;
    const int64_t L = A.lam_stride;
    unsigned long long n_pairs = 0;
    for (int64_t j = j0; j <= j1; ++j) {
        for (int64_t i = i0; i <= i1; ++i) {
            const int64_t k = i + B.nx * j;
            double o[3], m[3];
            sample_coords(B, k, o, m);
            double ha = 0.0;
            if (ST != ST_SCATTER) ha = (A.hmode == PSB_H_PER_SAMPLE) ? A.hs[k] : A.hs[0];
            const double ra = X<double>::mul(K, ha);
            const double ra2 = X<double>::mul(ra, ra);
            const double e2 = ex_d2_line<double>(o, m, xb[0], xb[1], xb[2]);
            if (!(e2 <= ex_r2<ST, double>(ra2, hb, K))) continue;
            ++n_pairs;
            const double dr = sqrt(e2 < 0.0 ? 0.0 : e2);
            double W, dW;
            if (ST == ST_GATHER) {
                line_Wd(dr, ha, A.lut, K, W, dW);
            } else if (ST == ST_SCATTER) {
                line_Wd(dr, hb, A.lut, K, W, dW);
            } else {
                double Wa, da, Wb, db;
                line_Wd(dr, ha, A.lut, K, Wa, da);
                line_Wd(dr, hb, A.lut, K, Wb, db);
                W = 0.5 * (Wa + Wb);
                dW = 0.5 * (da + db);
            }
            double aS = __ldg(&A.lam[k]);
#pragma unroll
            for (int c = 0; c < KC; ++c) {
                if (c < kc) {
                    const double lsw = __ldg(&A.lam[(1 + c) * L + k]);
                    aS += lsw * Ab[c];
                    ga[c] += mr * lsw * W;
                }
            }
            gm += aS * W / rhob;
            if (dr > 0.0) {
                // d r_perp / d x_b = (D - (D.m) m) / r_perp, D = x_b - o
                const double D[3] = {xb[0] - o[0], xb[1] - o[1], xb[2] - o[2]};
                const double Dm = D[0] * m[0] + D[1] * m[1] + D[2] * m[2];
                const double s = mr * aS * dW / dr;
                for (int d = 0; d < 3; ++d) gx[d] += s * (D[d] - Dm * m[d]);
            }
        }
    }
    const int64_t ob = A.porder[b];
    A.gm[ob] = gm;
    A.gx[ob] = gx[0]; A.gy[ob] = gx[1]; A.gz[ob] = gx[2];
#pragma unroll
    for (int c = 0; c < KC; ++c)
        if (c < kc && A.gcol[c]) A.gcol[c][ob] = ga[c];
    if (A.stats && n_pairs) atomicAdd(&A.stats[0], n_pairs);
}

// sample coordinates of every sample of a source (grid, box) as arrays
__global__ void k_sample_xyz(const SampleSrc<double> S, int64_t ns, double* x, double* y, double* z) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ns) return;
    double p[3], d[3];
    sample_coords(S, k, p, d);
    x[k] = p[0]; y[k] = p[1]; z[k] = p[2];
}

// lam_out[q][i] = lam_in[q][order[i]]: sum cotangents in the sample tree's order
__global__ void k_gather_rows(const double* in, const int64_t* order, int64_t n, int nq, double* out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t s = order[i];
    for (int q = 0; q < nq; ++q) out[q * n + i] = in[q * n + s];
}

}  // namespace psb
