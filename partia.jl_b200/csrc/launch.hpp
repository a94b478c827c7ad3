// launch.hpp -- template dispatch of the interpolation kernels.  The
// instantiations are split over inst_*.cu so that they compile in parallel.
#pragma once

#include "k_split.cuh"

namespace psb {

// KF: 0 = the M4 kernel's own code, 1 = the other kernel families (digests
// evaluate no kernel)
template <class T, int P, int S, int W, int KF>
static void dispatch_points_kf(const Args<T>& a, int kc, unsigned g, cudaStream_t s) {
    if constexpr (W != WHAT_INTERP) {
        k_points<T, P, S, 1, W, KF><<<g, 128, 0, s>>>(a);
    } else {
        if (kc <= 1) k_points<T, P, S, 1, W, KF><<<g, 128, 0, s>>>(a);
        else if (kc <= 2) k_points<T, P, S, 2, W, KF><<<g, 128, 0, s>>>(a);
        else if (kc <= 4) k_points<T, P, S, 4, W, KF><<<g, 128, 0, s>>>(a);
        else k_points<T, P, S, 8, W, KF><<<g, 128, 0, s>>>(a);
    }
}
template <class T, int P, int S, int W>
static void dispatch_points_k(const Args<T>& a, int kc, unsigned g, cudaStream_t s) {
    if (W == WHAT_DIGEST || a.tv.kern == KERN_M4) dispatch_points_kf<T, P, S, W, 0>(a, kc, g, s);
    else if constexpr (W != WHAT_DIGEST) dispatch_points_kf<T, P, S, W, 1>(a, kc, g, s);
}

template <class T, int P, int W>
static void dispatch_points_s(const Args<T>& a, int st, int kc, unsigned g, cudaStream_t s) {
    if (st == ST_GATHER) dispatch_points_k<T, P, ST_GATHER, W>(a, kc, g, s);
    else if (st == ST_SCATTER) dispatch_points_k<T, P, ST_SCATTER, W>(a, kc, g, s);
    else dispatch_points_k<T, P, ST_SYMMETRIC, W>(a, kc, g, s);
}

template <class T, int P>
static cudaError_t dispatch_points_p(const Args<T>& a, int st, int kc, int what, cudaStream_t s) {
    unsigned g = (unsigned)((a.src.ntiles + 3) / 4);
    if (g == 0) return cudaSuccess;
    if (what == WHAT_INTERP) dispatch_points_s<T, P, WHAT_INTERP>(a, st, kc, g, s);
    else if (what == WHAT_DENSITY) dispatch_points_s<T, P, WHAT_DENSITY>(a, st, kc, g, s);
    else dispatch_points_s<T, P, WHAT_DIGEST>(a, st, kc, g, s);
    return cudaGetLastError();
}

template <class T, int P, int S, int W>
static void dispatch_lines_k(const Args<T>& a, int kc, unsigned g, size_t smem, cudaStream_t s) {
    if constexpr (W != WHAT_INTERP) {
        k_lines<T, P, S, 1, W><<<g, 128, smem, s>>>(a);
    } else {
        if (kc <= 1) k_lines<T, P, S, 1, W><<<g, 128, smem, s>>>(a);
        else k_lines<T, P, S, 4, W><<<g, 128, smem, s>>>(a);
    }
}

template <class T, int P, int W>
static void dispatch_lines_s(const Args<T>& a, int st, int kc, unsigned g, size_t smem, cudaStream_t s) {
    if (st == ST_GATHER) dispatch_lines_k<T, P, ST_GATHER, W>(a, kc, g, smem, s);
    else if (st == ST_SCATTER) dispatch_lines_k<T, P, ST_SCATTER, W>(a, kc, g, smem, s);
    else dispatch_lines_k<T, P, ST_SYMMETRIC, W>(a, kc, g, smem, s);
}

template <class T, int P>
static cudaError_t dispatch_lines_p(const Args<T>& a, int st, int kc, int what, cudaStream_t s) {
    unsigned g = (unsigned)((a.src.ntiles + 3) / 4);
    if (g == 0) return cudaSuccess;
    // shared memory only for the FP64 sums over the short float table (k_lines)
    size_t smem = (P == PREC_FP64 && a.lut_n == LUT_SHORT_N) ? (size_t)LUT_SHORT_N * sizeof(double) : 0;
    if (what == WHAT_INTERP) dispatch_lines_s<T, P, WHAT_INTERP>(a, st, kc, g, smem, s);
    else dispatch_lines_s<T, P, WHAT_DIGEST>(a, st, kc, g, smem, s);
    return cudaGetLastError();
}

// two-kernel point path: k_collect (bodies = false) or k_bodies (bodies = true)
// over the batch a.sp
template <class T, int P, int S, int KF, bool DG>
static void dispatch_bodies_kfd(const Args<T>& a, int kc, unsigned g, cudaStream_t s) {
    if (kc <= 1) k_bodies<T, P, S, 1, KF, DG><<<g, 128, 0, s>>>(a);
    else if (kc <= 2) k_bodies<T, P, S, 2, KF, DG><<<g, 128, 0, s>>>(a);
    else if (kc <= 4) k_bodies<T, P, S, 4, KF, DG><<<g, 128, 0, s>>>(a);
    else k_bodies<T, P, S, 8, KF, DG><<<g, 128, 0, s>>>(a);
}
// DG: the catalog has a density gradient (its sums and the masses in
// registers only where they are used)
template <class T, int P, int S, int KF>
static void dispatch_bodies_kf(const Args<T>& a, int kc, unsigned g, cudaStream_t s) {
    if (a.rec.need_dg) dispatch_bodies_kfd<T, P, S, KF, true>(a, kc, g, s);
    else dispatch_bodies_kfd<T, P, S, KF, false>(a, kc, g, s);
}
template <class T, int P, int S>
static void dispatch_bodies_k(const Args<T>& a, int kc, unsigned g, cudaStream_t s) {
    if (a.tv.kern == KERN_M4) dispatch_bodies_kf<T, P, S, 0>(a, kc, g, s);
    else dispatch_bodies_kf<T, P, S, 1>(a, kc, g, s);
}

template <class T, int P>
static cudaError_t dispatch_split_p(const Args<T>& a, int st, int kc, bool bodies, cudaStream_t s) {
    unsigned g = (unsigned)((a.sp.ntiles + 3) / 4);
    if (g == 0) return cudaSuccess;
    if (!bodies) {
        if (st == ST_GATHER) k_collect<T, P, ST_GATHER><<<g, 128, 0, s>>>(a);
        else if (st == ST_SCATTER) k_collect<T, P, ST_SCATTER><<<g, 128, 0, s>>>(a);
        else k_collect<T, P, ST_SYMMETRIC><<<g, 128, 0, s>>>(a);
    } else {
        if (st == ST_GATHER) dispatch_bodies_k<T, P, ST_GATHER>(a, kc, g, s);
        else if (st == ST_SCATTER) dispatch_bodies_k<T, P, ST_SCATTER>(a, kc, g, s);
        else dispatch_bodies_k<T, P, ST_SYMMETRIC>(a, kc, g, s);
    }
    return cudaGetLastError();
}

// defined in inst_*.cu
template <class T> cudaError_t launch_points(const Args<T>& a, int prec, int st, int kc, int what, cudaStream_t s);
cudaError_t launch_split_d0(const Args<double>& a, int st, int kc, bool bodies, cudaStream_t s);
cudaError_t launch_split_d1(const Args<double>& a, int st, int kc, bool bodies, cudaStream_t s);
cudaError_t launch_split_f0(const Args<float>& a, int st, int kc, bool bodies, cudaStream_t s);
cudaError_t launch_split_f1(const Args<float>& a, int st, int kc, bool bodies, cudaStream_t s);
inline cudaError_t launch_split(const Args<double>& a, int prec, int st, int kc, bool bodies, cudaStream_t s) {
    return prec == PREC_FP64 ? launch_split_d0(a, st, kc, bodies, s) : launch_split_d1(a, st, kc, bodies, s);
}
inline cudaError_t launch_split(const Args<float>& a, int prec, int st, int kc, bool bodies, cudaStream_t s) {
    return prec == PREC_FP64 ? launch_split_f0(a, st, kc, bodies, s) : launch_split_f1(a, st, kc, bodies, s);
}
template <class T> cudaError_t launch_lines(const Args<T>& a, int prec, int st, int kc, int what, cudaStream_t s);

}  // namespace psb
