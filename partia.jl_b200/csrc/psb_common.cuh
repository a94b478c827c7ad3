// psb_common.cuh -- shared device helpers of the B200 SPH interpolation library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "partia_b200.h"
#include "kernels.cuh"

#define PSB_WARP 32
#define PSB_FULL 0xffffffffu

// Device error word bits (set with atomicOr, read back by the host).
#define PSB_DERR_TRAVERSAL 1u   // a traversal or refit loop hit its bound
#define PSB_DERR_REFIT 2u       // a refit node was not combined exactly once
#define PSB_DERR_INPUT 4u       // non-finite particle coordinate
#define PSB_DERR_SORT 8u        // a radix-sort look-back wait ran out of iterations

namespace psb {

// A subtree of at most SPAN_LEAVES leaves is handled as one unit ("span") by
// the traversals; its root is the highest node with at most that many leaves.
constexpr int SPAN_LEAVES = 32;
// The traversal kernels size the per-warp stage arrays of a tile's samples
// (one per lane) and of a span's leaves (one per lane in the leaf-per-lane
// tests) by the same constant: a span is exactly one warp wide.
static_assert(SPAN_LEAVES == 32, "a span is one warp wide: stage arrays are indexed by lane");

// ---------------------------------------------------------------------------
// Exactly rounded arithmetic.  Parity-critical steps (Morton quantisation,
// squared distances, radii, the neighbour inclusion test, the nearest-particle
// argmin) restate the reference's uncontracted IEEE operations, so they use
// the _rn intrinsics, which the compiler never fuses into an FMA.
// ---------------------------------------------------------------------------
template <class T> struct X;
template <> struct X<double> {
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double sqrt(double a) { return __dsqrt_rn(a); }
};
template <> struct X<float> {
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float sqrt(float a) { return __fsqrt_rn(a); }
};

// Julia's max(a, b) / min(a, b) on non-NaN values, as used by the traversal
// macros (LinearBVHTraversalMacros.jl:325,342,358,908-909).
template <class T> __device__ __forceinline__ T jmax(T a, T b) { return (a < b) ? b : a; }
template <class T> __device__ __forceinline__ T jmin(T a, T b) { return (b < a) ? b : a; }

template <class T> __device__ __forceinline__ T qnan();
template <> __device__ __forceinline__ double qnan<double>() { return __longlong_as_double(0x7ff8000000000000ll); }
template <> __device__ __forceinline__ float qnan<float>() { return __int_as_float(0x7fc00000); }

// SplitMix64 finaliser: the neighbour-digest hash of a 1-based leaf index.
__device__ __forceinline__ uint64_t mix64(uint64_t v) {
    v += 0x9E3779B97F4A7C15ull;
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
    return v ^ (v >> 31);
}

// 3D Morton bit spread: bit b of a 21-bit value moves to bit 3b.
__device__ __forceinline__ uint64_t spread3(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

// ---------------------------------------------------------------------------
// Device-side LBVH view.  Node ids are the reference's unified 1-based ids;
// per-id arrays are indexed id-1.  Internal node i (1..n-1) is record i-1 of
// the node arrays.  Particles are stored in Morton order.
// ---------------------------------------------------------------------------
template <class T> struct TreeView {
    int64_t n;
    int32_t root;
    const int32_t* left;     // 2n-1
    const int32_t* escape;   // 2n-1
    const int4* links;       // n-1: (left, escape, range_lo, range_hi) of internal nodes
    const uint64_t* codes;   // n sorted, de-duplicated Morton codes
    double qlo[3];           // particle bounding-box minimum (Morton quantisation)
    double qscale[3];        // (2^21 - 1) / extent per axis, 0 for a flat axis
    const int32_t* range_lo; // n-1, first leaf (1-based) of internal node
    const int32_t* range_hi; // n-1, last leaf (1-based)
    const T* nmin[3];        // n-1 each
    const T* nmax[3];
    const T* nscale;
    // exact particle data (Morton order)
    const T* x; const T* y; const T* z; const T* h; const T* m; const T* rho;
    const T* const* cols;    // device array of ncol column pointers
    int32_t ncol;
    // float traversal records (used by the FP32C path of double inputs)
    const float4* node_lo;   // (minx, miny, minz, node_scale) rounded outward / up
    const float4* node_hi;   // (maxx, maxy, maxz, 0) rounded outward
    // (x - ax, y - ay, z - az, h): position relative to the first leaf of the
    // leaf's span (the leaf's highest ancestor with <= SPAN_LEAVES leaves)
    const float4* leaf4;
    const float* mrho;       // m / rho (float)
    const float* mf;         // m (float)
    const float4* leafK;     // (1/h, sigma/h^3, sigma/h^4, m/rho) in float
    // at the first leaf of every span: (max over the span of |leaf4.x| +
    // |leaf4.y| + |leaf4.z|, max h), both rounded up (float error bounds)
    const float2* spanb;
    float coord_err;         // bound on |float coordinate - exact| for node tests
    // kernel family (psb_kernel): support K in units of h (exact in float),
    // the 3D norm, and the first q of the piece that reaches the support edge
    int kern;
    float Kf;
    double Kd;
    double sig;
    float qedge;
};

// Host-side helpers -----------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace psb
