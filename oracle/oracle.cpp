// oracle.cpp -- CPU restatement of Partia.jl's SPH interpolation hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library and
// the timed CPU baseline ("port" of the reference's multithreaded CPU path).
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs load
// it; the product library never links it.
//
// It restates the reference's arithmetic literally, in the same operation
// order and without FMA contraction (build with -ffp-contract=off, no
// fast-math), so that Morton codes, tree topology and neighbour sets are
// bit-identical to the reference's CPU path and fields follow the same
// roundings.  Every function names the reference file:line it follows; paths
// are relative to the Partia.jl source tree (src/julia/...).
//
// Parity pins: the reference's own known-answer tests for this path
// (test/kernel_function_tests.jl, test/neighbor_search_tests.jl,
// test/interpolation_tests.jl, test/point_samples_interpolation_tests.jl and
// the M4 line-integral table of table/line_integrated_kernel_tables.jl) are
// restated in tests/test_oracle_*.py and run against this file.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <new>
#include <numeric>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// ---------------------------------------------------------------------------
// Kernel functions: M4 cubic spline.
// kernel_function/kernels/M4_spline.jl:13-36 (f, f'), :66 (support 2),
// :101 (3D norm 1/pi); kernel_function/kernel.jl:141-146 (W),
// :273-286 (dimensionless gradient), :360-365 (dimensional gradient).
// Julia literal powers x^3 / x^2 are x*x*x / x*x (Base.literal_pow).
// ---------------------------------------------------------------------------
template <class T> static inline T m4_f(T q) {
    if (q < T(0)) return std::numeric_limits<T>::quiet_NaN();
    if (T(0) <= q && q < T(1)) {
        T a = T(2) - q, b = T(1) - q;
        return T(0.25) * (a * a * a) - (b * b * b);
    } else if (T(1) <= q && q < T(2)) {
        T a = T(2) - q;
        return T(0.25) * (a * a * a);
    }
    return T(0);
}

template <class T> static inline T m4_df(T q) {
    if (q < T(0)) return std::numeric_limits<T>::quiet_NaN();
    if (T(0) <= q && q < T(1)) {
        T a = T(2) - q, b = T(1) - q;
        return T(-0.75) * (a * a) + T(3) * (b * b);
    } else if (T(1) <= q && q < T(2)) {
        T a = T(2) - q;
        return T(-0.75) * (a * a);
    }
    return T(0);
}

template <class T> static inline T m4_norm3() { return T(1) / T(3.141592653589793238462643383279502884L); }

// ---------------------------------------------------------------------------
// The other kernel families, as the reference writes them:
// kernels/M5_spline.jl (support 2.5, 3D norm 0.05/pi), kernels/M6_spline.jl
// (support 3, 1/(120 pi)), kernels/C2_Wendland.jl (2, 21/(16 pi)),
// kernels/C4_Wendland.jl (2, 495/(256 pi)), kernels/C6_Wendland.jl
// (2, 1365/(512 pi)), each with f and f' per piece.  g_kern is the kernel of
// the current call (orc_set_kernel; calls are made one at a time).
// ---------------------------------------------------------------------------
enum { KERN_M4 = 0, KERN_M5 = 1, KERN_M6 = 2, KERN_C2 = 3, KERN_C4 = 4, KERN_C6 = 5, KERN_COUNT = 6 };
static int g_kern = KERN_M4;

template <class T> static inline T pw2(T x) { return x * x; }
template <class T> static inline T pw3(T x) { return x * x * x; }
template <class T> static inline T pw4(T x) { T y = x * x; return y * y; }
template <class T> static inline T pw5(T x) { T y = x * x; return y * y * x; }

template <class T> static inline T kern_support() {
    switch (g_kern) {
    case KERN_M5: return T(2.5);
    case KERN_M6: return T(3.0);
    default: return T(2.0);
    }
}

template <class T> static inline T kern_norm3() {
    const T pi = T(3.141592653589793238462643383279502884L);
    switch (g_kern) {
    case KERN_M5: return T(0.05) / pi;
    case KERN_M6: return T(1) / (T(120) * pi);
    case KERN_C2: return T(21) / (T(16) * pi);
    case KERN_C4: return T(495) / (T(256) * pi);
    case KERN_C6: return T(1365) / (T(512) * pi);
    default: return m4_norm3<T>();
    }
}

template <class T> static inline T kern_f(T q) {
    if (q < T(0)) return std::numeric_limits<T>::quiet_NaN();
    switch (g_kern) {
    case KERN_M5:
        if (q < T(0.5)) return pw4(T(2.5) - q) - T(5) * pw4(T(1.5) - q) + T(10) * pw4(T(0.5) - q);
        if (q < T(1.5)) return pw4(T(2.5) - q) - T(5) * pw4(T(1.5) - q);
        if (q < T(2.5)) return pw4(T(2.5) - q);
        return T(0);
    case KERN_M6:
        if (q < T(1)) return pw5(T(3) - q) - T(6) * pw5(T(2) - q) + T(15) * pw5(T(1) - q);
        if (q < T(2)) return pw5(T(3) - q) - T(6) * pw5(T(2) - q);
        if (q < T(3)) return pw5(T(3) - q);
        return T(0);
    case KERN_C2:
        if (q < T(2)) return pw4(T(1) - T(0.5) * q) * (T(2) * q + T(1));
        return T(0);
    case KERN_C4:
        if (q < T(2)) { T a = T(1) - T(0.5) * q; return pw3(a) * pw3(a) * ((T(35) / T(12)) * pw2(q) + T(3) * q + T(1)); }
        return T(0);
    case KERN_C6:
        if (q < T(2)) { T a = T(1) - T(0.5) * q; return pw4(a) * pw4(a) * (T(4) * pw3(q) + T(6.25) * pw2(q) + T(4) * q + T(1)); }
        return T(0);
    default: return m4_f(q);
    }
}

template <class T> static inline T kern_df(T q) {
    if (q < T(0)) return std::numeric_limits<T>::quiet_NaN();
    switch (g_kern) {
    case KERN_M5:
        if (q < T(0.5)) return T(-4) * pw3(T(2.5) - q) + T(20) * pw3(T(1.5) - q) - T(40) * pw3(T(0.5) - q);
        if (q < T(1.5)) return T(-4) * pw3(T(2.5) - q) + T(20) * pw3(T(1.5) - q);
        if (q < T(2.5)) return T(-4) * pw3(T(2.5) - q);
        return T(0);
    case KERN_M6:
        if (q < T(1)) return T(-5) * pw4(T(3) - q) + T(30) * pw4(T(2) - q) - T(75) * pw4(T(1) - q);
        if (q < T(2)) return T(-5) * pw4(T(3) - q) + T(30) * pw4(T(2) - q);
        if (q < T(3)) return T(-5) * pw4(T(3) - q);
        return T(0);
    case KERN_C2:
        if (q < T(2)) { T a = T(1) - T(0.5) * q; return pw4(a) * T(2) - pw3(a) * (T(4) * q + T(2)); }
        return T(0);
    case KERN_C4:
        if (q < T(2)) {
            T a = T(1) - T(0.5) * q;
            return pw3(a) * pw3(a) * ((T(35) / T(6)) * q + T(3)) -
                   pw5(a) * ((T(35) / T(4)) * pw2(q) + T(9) * q + T(3));
        }
        return T(0);
    case KERN_C6:
        if (q < T(2)) {
            T a = T(1) - T(0.5) * q;
            return pw4(a) * pw4(a) * (T(12) * pw2(q) + T(12.5) * q + T(4)) -
                   pw4(a) * pw3(a) * (T(16) * pw3(q) + T(25) * pw2(q) + T(16) * q + T(4));
        }
        return T(0);
    default: return m4_df(q);
    }
}

// Smoothed_kernel_function(K, r, h, Val(3)), kernel.jl:141-146
template <class T> static inline T kernel_W(T r, T h) {
    T invh = T(1) / h;
    T inv_hD = invh * invh * invh;
    T q = r * invh;
    return inv_hD * (kern_norm3<T>() * kern_f(q));
}

// Smoothed_gradient_kernel_function(K, dx, dy, dz, h), kernel.jl:273-286,360-365
template <class T> static inline void kernel_gradW(T dx, T dy, T dz, T h, T& gx, T& gy, T& gz) {
    T invh = T(1) / h;
    T inv_hDp1 = invh * invh * invh * invh;
    T r2 = dx * dx + dy * dy + dz * dz;
    T wx, wy, wz;
    if (r2 == T(0)) {
        wx = wy = wz = T(0);
    } else {
        T r = std::sqrt(r2);
        T invr = T(1) / r;
        T q = r / h;
        T coeff = kern_df(q) * kern_norm3<T>() * invr;
        wx = dx * coeff; wy = dy * coeff; wz = dz * coeff;
    }
    gx = inv_hDp1 * wx; gy = inv_hDp1 * wy; gz = inv_hDp1 * wz;
}

// ---------------------------------------------------------------------------
// Line-integrated kernel.  kernel_function/line_integrated_kernel.jl:13-19
// (_lin_lut), :90-94 (q >= q_max -> 0), :132-137 (1/h scaling).
// The table is regenerated from the M4 integral I(q) = int f(sqrt(q^2+s^2)) ds
// (times the 3D norm) on the reference's grid Q_k = (k-1) * 2/4095,
// k = 1..4096 (table/line_integrated_kernel_tables.jl:1,1029), by 64-point
// Gauss-Legendre quadrature on each smooth segment (split at the kinks
// s = sqrt(1-q^2), sqrt(4-q^2)).
// ---------------------------------------------------------------------------
static const int LUT_N = 4096;

static void gauss_legendre(int n, std::vector<long double>& x, std::vector<long double>& w) {
    x.resize(n); w.resize(n);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int i = 0; i < n; ++i) {
        long double z = std::cos(pi * (i + 0.75L) / (n + 0.5L)), pp = 0;
        for (int it = 0; it < 100; ++it) {
            long double p1 = 1, p2 = 0;
            for (int j = 1; j <= n; ++j) {
                long double p3 = p2; p2 = p1;
                p1 = ((2 * j - 1) * z * p2 - (j - 1) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1);
            long double dz = p1 / pp;
            z -= dz;
            if (std::fabs(dz) < 1e-19L) break;
        }
        x[i] = z;
        w[i] = 2 / ((1 - z * z) * pp * pp);
    }
}

// kernel shape f(q) of kernel kid in long double, and its break points (the
// last one is the support)
static long double shape_ld(int kid, long double q) {
    switch (kid) {
    case KERN_M5: {
        long double a = 2.5L - q, b = 1.5L - q, c = 0.5L - q;
        if (q < 0.5L) return a * a * a * a - 5 * b * b * b * b + 10 * c * c * c * c;
        if (q < 1.5L) return a * a * a * a - 5 * b * b * b * b;
        if (q < 2.5L) return a * a * a * a;
        return 0;
    }
    case KERN_M6: {
        long double a = 3 - q, b = 2 - q, c = 1 - q;
        if (q < 1) return a * a * a * a * a - 6 * b * b * b * b * b + 15 * c * c * c * c * c;
        if (q < 2) return a * a * a * a * a - 6 * b * b * b * b * b;
        if (q < 3) return a * a * a * a * a;
        return 0;
    }
    case KERN_C2: { if (q >= 2) return 0; long double a = 1 - 0.5L * q; return a * a * a * a * (2 * q + 1); }
    case KERN_C4: {
        if (q >= 2) return 0;
        long double a = 1 - 0.5L * q, a2 = a * a;
        return a2 * a2 * a2 * (35.0L / 12 * q * q + 3 * q + 1);
    }
    case KERN_C6: {
        if (q >= 2) return 0;
        long double a = 1 - 0.5L * q, a4 = a * a * a * a;
        return a4 * a4 * (4 * q * q * q + 6.25L * q * q + 4 * q + 1);
    }
    default:
        if (q < 1) { long double a = 2 - q, b = 1 - q; return 0.25L * a * a * a - b * b * b; }
        if (q < 2) { long double a = 2 - q; return 0.25L * a * a * a; }
        return 0;
    }
}
static int breaks_ld(int kid, long double* t) {
    switch (kid) {
    case KERN_M5: t[0] = 0.5L; t[1] = 1.5L; t[2] = 2.5L; return 3;
    case KERN_M6: t[0] = 1; t[1] = 2; t[2] = 3; return 3;
    case KERN_C2: case KERN_C4: case KERN_C6: t[0] = 2; return 1;
    default: t[0] = 1; t[1] = 2; return 2;
    }
}

// I(b) = norm3 * 2 * int_0^sqrt(K^2-b^2) f(sqrt(b^2+s^2)) ds on the reference's
// grid Q_k = (k-1) K/4095, k = 1..4096, by 64-point Gauss-Legendre on each
// smooth segment (split where sqrt(b^2+s^2) crosses a break point).
static void build_line_table(int kid, double* Q, double* Inorm) {
    std::vector<long double> gx, gw;
    gauss_legendre(64, gx, gw);
    const long double pi = 3.141592653589793238462643383279502884L;
    long double t[3];
    const int nb = breaks_ld(kid, t);
    const long double K = t[nb - 1];
    long double norm;
    switch (kid) {
    case KERN_M5: norm = 0.05L / pi; break;
    case KERN_M6: norm = 1 / (120 * pi); break;
    case KERN_C2: norm = 21 / (16 * pi); break;
    case KERN_C4: norm = 495 / (256 * pi); break;
    case KERN_C6: norm = 1365 / (512 * pi); break;
    default: norm = 1 / pi;
    }
    const double Kd = (double)K;
    for (int k = 0; k < LUT_N; ++k) {
        long double b = K / (LUT_N - 1) * k;
        Q[k] = Kd / 4095.0 * (double)k;
        long double tot = 0;
        if (b < K) {
            long double segs[4] = {0, 0, 0, 0};
            int ns = 0;
            for (int i = 0; i < nb; ++i)
                if (t[i] > b) segs[++ns] = std::sqrt(t[i] * t[i] - b * b);
            for (int sgi = 0; sgi < ns; ++sgi) {
                long double a = segs[sgi], c = segs[sgi + 1];
                for (int i = 0; i < 64; ++i) {
                    long double s = 0.5L * (c - a) * gx[i] + 0.5L * (c + a);
                    tot += 0.5L * (c - a) * gw[i] * shape_ld(kid, std::sqrt(b * b + s * s));
                }
            }
            tot *= 2;
        }
        Inorm[k] = (double)(tot * norm);
    }
    Q[0] = 0.0;
}

struct LineTable {
    double Q[LUT_N], I[LUT_N];
    float Qf[LUT_N], If[LUT_N];
    explicit LineTable(int kid) {
        build_line_table(kid, Q, I);
        for (int k = 0; k < LUT_N; ++k) { Qf[k] = (float)Q[k]; If[k] = (float)I[k]; }
    }
};
template <int KID> static const LineTable& line_table_k() { static LineTable t(KID); return t; }
static const LineTable& line_table() {
    switch (g_kern) {
    case KERN_M5: return line_table_k<KERN_M5>();
    case KERN_M6: return line_table_k<KERN_M6>();
    case KERN_C2: return line_table_k<KERN_C2>();
    case KERN_C4: return line_table_k<KERN_C4>();
    case KERN_C6: return line_table_k<KERN_C6>();
    default: return line_table_k<KERN_M4>();
    }
}

template <class T> static inline const T* lut_Q();
template <class T> static inline const T* lut_I();
template <> inline const double* lut_Q<double>() { return line_table().Q; }
template <> inline const double* lut_I<double>() { return line_table().I; }
template <> inline const float* lut_Q<float>() { return line_table().Qf; }
template <> inline const float* lut_I<float>() { return line_table().If; }

// _lin_lut, line_integrated_kernel.jl:13-19 (1-based i restated 0-based)
template <class T> static inline T lin_lut(T q) {
    const T* Q = lut_Q<T>();
    const T* I = lut_I<T>();
    T dq = Q[1] - Q[0];
    T idxf = q / dq + T(1);
    // Base.unsafe_trunc(Int32, idxf), then clamp to 1..N-1
    int32_t i;
    if (!(idxf == idxf) || idxf >= T(2147483647.0) || idxf <= T(-2147483648.0)) i = 1;
    else i = (int32_t)idxf;
    if (i < 1) i = 1;
    if (i > LUT_N - 1) i = LUT_N - 1;
    T t = idxf - T(i);
    return I[i - 1] * (T(1) - t) + I[i] * t;
}

// line_integrated_kernel_function(K, r, h), line_integrated_kernel.jl:90-94,132-137
template <class T> static inline T line_kernel(T r, T h) {
    T invh = T(1) / h;
    T q = r * invh;
    T Idl = (q >= kern_support<T>()) ? T(0) : lin_lut(q);
    return invh * Idl;
}

// ---------------------------------------------------------------------------
// Morton encoding.  LinearBoundingVolumeHierarchy/MortonEncoding/toolbox.jl:
// 131-144 (sort + strictly-increasing dedup), 158-166 (3D bit spread),
// 224-229 (x<<2 | y<<1 | z), 375-383 (21 bits, scale 2^21-1),
// 392-405 (min/max normalise, all-equal axis -> 0.5), 422-447 (floor).
// ---------------------------------------------------------------------------
static inline uint64_t spread3(uint64_t v) {
    // bit b of v goes to bit 3b (b = 0..20)
    uint64_t out = 0;
    for (int b = 0; b < 21; ++b) out |= ((v >> b) & 1ull) << (3 * b);
    return out;
}

template <class T> static void normalize_axis(const T* v, int64_t n, std::vector<T>& out) {
    out.resize(n);
    T vmin = v[0], vmax = v[0];
    for (int64_t i = 1; i < n; ++i) {
        vmin = (v[i] < vmin) ? v[i] : vmin;
        vmax = (v[i] > vmax) ? v[i] : vmax;
    }
    T dv = vmax - vmin;
    if (dv == T(0)) { std::fill(out.begin(), out.end(), T(0.5)); return; }
    T inv = T(1) / dv;
    for (int64_t i = 0; i < n; ++i) out[i] = (v[i] - vmin) * inv;
}

template <class T>
static void morton_codes(const T* x, const T* y, const T* z, int64_t n, std::vector<uint64_t>& codes) {
    std::vector<T> fx, fy, fz;
    normalize_axis(x, n, fx); normalize_axis(y, n, fy); normalize_axis(z, n, fz);
    const T scale = T(2097151);  // exp2(21) - 1
    codes.resize(n);
    for (int64_t i = 0; i < n; ++i) {
        uint64_t ix = (uint64_t)std::floor(scale * fx[i]);
        uint64_t iy = (uint64_t)std::floor(scale * fy[i]);
        uint64_t iz = (uint64_t)std::floor(scale * fz[i]);
        codes[i] = (spread3(ix) << 2) | (spread3(iy) << 1) | spread3(iz);
    }
}

// ---------------------------------------------------------------------------
// LBVH.  BinaryRadixTree/BinaryRadixTree.jl:82-133, BinaryRadixTree/toolbox.jl
// (all of it), LinearBVH/LinearBVH.jl:56-94, LinearBVH/toolbox.jl:36-94.
// Node ids are the reference's unified 1-based ids; arrays hold id at [id-1].
// ---------------------------------------------------------------------------
template <class T> struct Tree {
    int64_t n = 0;
    int32_t root = 0;
    std::vector<uint64_t> codes;   // sorted, deduplicated
    std::vector<int64_t> order;    // 0-based original index per Morton position
    std::vector<int32_t> left, right, escape, parent, range_hi;
    std::vector<T> lx, ly, lz, lh; // leaf coordinates and scale (Morton order)
    std::vector<T> nmin[3], nmax[3], nscale;
};

static inline int64_t clz64(uint64_t v) { return v == 0 ? 64 : __builtin_clzll(v); }

// _longest_common_prefix_length(codes, i, j), MortonEncoding/toolbox.jl:329-336 (1-based)
static inline int64_t delta(const std::vector<uint64_t>& c, int64_t i, int64_t j) {
    uint64_t a = c[i - 1], b = c[j - 1];
    if (a == b) return clz64((uint64_t)i ^ (uint64_t)j);
    return clz64(a ^ b);
}

// _range_direction / _find_range, BinaryRadixTree/toolbox.jl:14-53
static inline void find_range(const std::vector<uint64_t>& c, int64_t i, int64_t& lo, int64_t& hi) {
    int64_t n = (int64_t)c.size();
    int64_t dL = (i > 1) ? delta(c, i, i - 1) : -1;
    int64_t dR = (i < n) ? delta(c, i, i + 1) : -1;
    int64_t s = dR - dL;
    int64_t d = (s > 0) ? 1 : ((s < 0) ? -1 : 1);
    int64_t dmin = (1 <= i - d && i - d <= n) ? delta(c, i, i - d) : -1;
    int64_t lmax = 2;
    while (true) {
        int64_t j = i + lmax * d;
        if (j < 1 || j > n) break;
        if (delta(c, i, j) <= dmin) break;
        lmax *= 2;
    }
    int64_t l = 0;
    int64_t t = lmax >> 1;
    while (t > 0) {
        int64_t j = i + (l + t) * d;
        if (j >= 1 && j <= n && delta(c, i, j) > dmin) l += t;
        t >>= 1;
    }
    int64_t j = i + l * d;
    lo = std::min(i, j); hi = std::max(i, j);
}

// _split_position, BinaryRadixTree/toolbox.jl:55-76
static inline int64_t split_position(const std::vector<uint64_t>& c, int64_t first, int64_t last) {
    if (c[first - 1] == c[last - 1]) {
        int64_t m = (first + last) >> 1;
        return std::min(std::max(m, first), last - 1);
    }
    int64_t pfl = delta(c, first, last);
    int64_t split = first, step = last - first;
    while (step > 1) {
        step = (step + 1) >> 1;
        int64_t ns = split + step;
        if (ns < last) {
            if (delta(c, first, ns) > pfl) split = ns;
        }
    }
    return split;
}

template <class T>
static void build_tree(Tree<T>& tr, const T* x, const T* y, const T* z, const T* h, int64_t n) {
    tr.n = n;
    // MortonEncoding(x, y, z), MortonEncoding.jl:36-43
    std::vector<uint64_t> raw;
    morton_codes(x, y, z, n, raw);
    tr.order.resize(n);
    std::iota(tr.order.begin(), tr.order.end(), (int64_t)0);
    // sortperm(codes; alg=QuickSort) with Perm ordering: ties broken by index
    std::stable_sort(tr.order.begin(), tr.order.end(),
                     [&](int64_t a, int64_t b) { return raw[a] < raw[b]; });
    tr.codes.resize(n);
    for (int64_t i = 0; i < n; ++i) tr.codes[i] = raw[tr.order[i]];
    for (int64_t i = 1; i < n; ++i)
        if (tr.codes[i] <= tr.codes[i - 1]) tr.codes[i] = tr.codes[i - 1] + 1;
    tr.lx.resize(n); tr.ly.resize(n); tr.lz.resize(n); tr.lh.resize(n);
    for (int64_t i = 0; i < n; ++i) {
        int64_t o = tr.order[i];
        tr.lx[i] = x[o]; tr.ly[i] = y[o]; tr.lz[i] = z[o]; tr.lh[i] = h[o];
    }
    // BinaryRadixTree(enc), BinaryRadixTree.jl:82-133
    int64_t total = 2 * n - 1, nint = n - 1;
    tr.root = (n >= 2) ? 1 : 0;
    tr.left.assign(total, 0); tr.right.assign(total, 0);
    tr.escape.assign(total, 0); tr.parent.assign(total, 0);
    tr.range_hi.assign(std::max<int64_t>(nint, 0), 0);
    if (nint > 0) {
        const auto& c = tr.codes;
        #pragma omp parallel for schedule(static)
        for (int64_t i = 1; i <= nint; ++i) {
            int64_t lo, hi;
            find_range(c, i, lo, hi);
            tr.range_hi[i - 1] = (int32_t)hi;
            int64_t s = split_position(c, lo, hi);
            int64_t li = (s == lo) ? lo + (n - 1) : s;
            tr.left[i - 1] = (int32_t)li;
            tr.parent[li - 1] = (int32_t)i;
            int64_t ri = (s + 1 == hi) ? hi + (n - 1) : s + 1;
            tr.right[i - 1] = (int32_t)ri;
            tr.parent[ri - 1] = (int32_t)i;
        }
        std::vector<int32_t> adj(n);
        for (int64_t i = 1; i <= n - 1; ++i) adj[i - 1] = (int32_t)delta(c, i, i + 1);
        adj[n - 1] = std::numeric_limits<int32_t>::max();
        for (int64_t i = 1; i <= nint; ++i) {   // _build_escape! (internal), toolbox.jl:119-134
            int64_t hi = tr.range_hi[i - 1];
            int32_t e;
            if (hi == n) e = 0;
            else if (hi == n - 1) e = (int32_t)((n - 1) + n);
            else {
                int64_t next = hi + 1;
                e = (adj[next - 1] < adj[next - 2]) ? (int32_t)((n - 1) + next) : (int32_t)next;
            }
            tr.escape[i - 1] = e;
        }
        for (int64_t id = n; id <= total; ++id) {   // _build_escape! (leaf), toolbox.jl:136-156
            int32_t p = tr.parent[id - 1];
            if (p == 0) { tr.escape[id - 1] = 0; continue; }
            if (tr.left[p - 1] == (int32_t)id) tr.escape[id - 1] = tr.right[p - 1];
            else tr.escape[id - 1] = tr.escape[p - 1];
        }
    }
    // LinearBVH(enc, brt, BoxScale(h, true)), LinearBVH.jl:56-94; refit
    // _build_internal_aabb!, LinearBVH/toolbox.jl:36-94 ("second arrival").
    for (int d = 0; d < 3; ++d) { tr.nmin[d].assign(std::max<int64_t>(nint, 0), T(0)); tr.nmax[d].assign(std::max<int64_t>(nint, 0), T(0)); }
    tr.nscale.assign(std::max<int64_t>(nint, 0), T(0));
    std::vector<uint32_t> visited(std::max<int64_t>(nint, 0), 0);
    const std::vector<T>* leafc[3] = {&tr.lx, &tr.ly, &tr.lz};
    for (int64_t startid = n; startid <= total && nint > 0; ++startid) {
        int32_t p = tr.parent[startid - 1];
        while (p != 0) {
            uint32_t nv = ++visited[p - 1];
            if (nv != 2) break;
            int32_t l = tr.left[p - 1], r = tr.right[p - 1];
            bool ll = l >= (int32_t)n, rl = r >= (int32_t)n;
            T hl = ll ? tr.lh[l - n] : tr.nscale[l - 1];
            T hr = rl ? tr.lh[r - n] : tr.nscale[r - 1];
            tr.nscale[p - 1] = (hl > hr) ? hl : hr;
            for (int d = 0; d < 3; ++d) {
                T lmin = ll ? (*leafc[d])[l - n] : tr.nmin[d][l - 1];
                T rmin = rl ? (*leafc[d])[r - n] : tr.nmin[d][r - 1];
                T lmax = ll ? (*leafc[d])[l - n] : tr.nmax[d][l - 1];
                T rmax = rl ? (*leafc[d])[r - n] : tr.nmax[d][r - 1];
                tr.nmin[d][p - 1] = (lmin < rmin) ? lmin : rmin;
                tr.nmax[d][p - 1] = (lmax > rmax) ? lmax : rmax;
            }
            p = tr.parent[p - 1];
        }
    }
}

// ---------------------------------------------------------------------------
// Distances.  LinearBVH/LinearBVHTraversalMacros.jl:800-814 (point-point),
// :816-835 (point-AABB), :837-857 (point-line), :859-876 (line-point),
// :878-916 (line-AABB slab test), :918-953 (line-AABB lower bound).
// ---------------------------------------------------------------------------
template <class T> static inline T d2_point_leaf(const Tree<T>& tr, const T p[3], int64_t li) {
    T s = T(0);
    T d0 = p[0] - tr.lx[li]; s += d0 * d0;
    T d1 = p[1] - tr.ly[li]; s += d1 * d1;
    T d2 = p[2] - tr.lz[li]; s += d2 * d2;
    return s;
}

template <class T> static inline T d2_point_aabb(const Tree<T>& tr, const T p[3], int64_t ni) {
    T s = T(0);
    for (int d = 0; d < 3; ++d) {
        T a = tr.nmin[d][ni], b = tr.nmax[d][ni], pd = p[d];
        T t = pd < a ? (a - pd) : (pd > b ? (pd - b) : T(0));
        s += t * t;
    }
    return s;
}

template <class T> static inline T d2_line_point(const T o[3], const T m[3], T px, T py, T pz) {
    T D2 = T(0), Dm = T(0);
    T c[3] = {px, py, pz};
    for (int d = 0; d < 3; ++d) {
        T D = c[d] - o[d];
        D2 += D * D;
        Dm += D * m[d];
    }
    return D2 - Dm * Dm;
}

template <class T> static inline T d2_point_line(const T p[3], const T o[3], const T m[3]) {
    T D2 = T(0), Dm = T(0);
    for (int d = 0; d < 3; ++d) {
        T D = p[d] - o[d];
        D2 += D * D;
        Dm += D * m[d];
    }
    return D2 - Dm * Dm;
}

template <class T> static inline T jmax(T a, T b) { return (a < b) ? b : a; }
template <class T> static inline T jmin(T a, T b) { return (b < a) ? b : a; }

template <class T> static inline bool line_hits_aabb(const Tree<T>& tr, const T o[3], const T m[3], int64_t ni) {
    T tmin = -std::numeric_limits<T>::infinity();
    T tmax = std::numeric_limits<T>::infinity();
    for (int d = 0; d < 3; ++d) {
        T a = tr.nmin[d][ni], b = tr.nmax[d][ni];
        if (m[d] == T(0)) {
            if (o[d] < a || o[d] > b) return false;
        } else {
            T t0 = (a - o[d]) / m[d];
            T t1 = (b - o[d]) / m[d];
            if (t0 > t1) std::swap(t0, t1);
            tmin = jmax(tmin, t0);
            tmax = jmin(tmax, t1);
            if (tmin > tmax) return false;
        }
    }
    return true;
}

template <class T> static inline T d2_line_aabb_lb(const Tree<T>& tr, const T o[3], const T m[3], int64_t ni) {
    const T half = T(1) / T(2);
    if (line_hits_aabb(tr, o, m, ni)) return T(0);
    T c[3];
    for (int d = 0; d < 3; ++d) c[d] = (tr.nmin[d][ni] + tr.nmax[d][ni]) * half;
    T r2 = T(0);
    for (int d = 0; d < 3; ++d) {
        T hh = (tr.nmax[d][ni] - tr.nmin[d][ni]) * half;
        r2 += hh * hh;
    }
    T dc2 = d2_point_line(c, o, m);
    if (dc2 <= r2) return T(0);
    T dc = std::sqrt(dc2);
    T r = std::sqrt(r2);
    T dl = dc - r;
    return dl * dl;
}

// ---------------------------------------------------------------------------
// Stackless DFS traversals, LinearBVHTraversalMacros.jl:26-108 (point gather),
// :135-236 (point scatter), :268-371 (point symmetric), :408-494 (line gather),
// :539-644 (line scatter), :691-796 (line symmetric).  `mode` selects the
// radius rule; r2_of() is re-read at every test so the nearest search can
// shrink it (LinearBVHQueries.jl:118-140).  The visit count is bounded by
// 4n+4 steps; exceeding it returns false (corrupt escape links).
// ---------------------------------------------------------------------------
enum Mode { GATHER = 0, SCATTER = 1, SYMMETRIC = 2 };

template <class T, bool LINE, class R2, class HIT>
static bool traverse(const Tree<T>& tr, const T a[3], const T m[3], int mode, T K, R2 r2_of, HIT hit) {
    const int64_t n = tr.n;
    auto leaf_d2 = [&](int64_t li) -> T {
        if (LINE) return d2_line_point(a, m, tr.lx[li], tr.ly[li], tr.lz[li]);
        return d2_point_leaf(tr, a, li);
    };
    auto leaf_r2 = [&](int64_t li) -> T {
        if (mode == GATHER) return r2_of();
        T hb = tr.lh[li];
        T r = K * hb;
        if (mode == SCATTER) return r * r;
        return jmax(r2_of(), r * r);
    };
    if (tr.root == 0) {
        for (int64_t li = 0; li < n; ++li) {
            T d2 = leaf_d2(li);
            if (d2 <= leaf_r2(li)) hit(li, d2, tr.lh[li]);
        }
        return true;
    }
    int32_t node = tr.root;
    int64_t steps = 0, bound = 4 * n + 4;
    while (node != 0) {
        if (++steps > bound) return false;
        if (node >= (int32_t)n) {
            int64_t li = node - n;  // leaf_index - 1
            T d2 = leaf_d2(li);
            if (d2 <= leaf_r2(li)) hit(li, d2, tr.lh[li]);
            node = tr.escape[node - 1];
            continue;
        }
        int64_t ni = node - 1;
        T r2;
        if (mode == GATHER) r2 = r2_of();
        else {
            T hb = tr.nscale[ni];
            T r = K * hb;
            r2 = (mode == SCATTER) ? r * r : jmax(r2_of(), r * r);
        }
        T d2n = LINE ? d2_line_aabb_lb(tr, a, m, ni) : d2_point_aabb(tr, a, ni);
        if (d2n > r2) { node = tr.escape[node - 1]; continue; }
        node = tr.left[ni];
    }
    return true;
}

// LBVH_find_nearest_h, LinearBVHQueries.jl:118-140
template <class T> static T nearest_h(const Tree<T>& tr, const T p[3], bool& ok) {
    int64_t best = -1;
    T best2 = std::numeric_limits<T>::infinity();
    ok = traverse<T, false>(tr, p, p, GATHER, T(0), [&]() { return best2; },
        [&](int64_t li, T d2, T) { if (d2 < best2) { best2 = d2; best = li; } });
    if (best < 0) return std::numeric_limits<T>::quiet_NaN();
    return tr.lh[best];
}

// ---------------------------------------------------------------------------
// Catalog and fused per-sample interpolation.
// single_point_interpolation/kernels/general_interpolation.jl:1-223 (gather),
// :225-444 (scatter), :446-669 (symmetric); accumulation helpers in
// single_point_interpolation/accumulations/*.jl.
// ---------------------------------------------------------------------------
struct Catalog {
    int ns = 0, ng = 0, nd = 0, nc = 0;
    const int32_t* sslot = nullptr; const uint8_t* shep = nullptr;
    const int32_t* gslot = nullptr; const int32_t* dslot = nullptr; const int32_t* cslot = nullptr;
    int L() const { return ns + 3 * ng + nd + 3 * nc; }
};

template <class T> struct Particles {
    int64_t n = 0;
    std::vector<T> x, y, z, m, h, rho;   // Morton order after build
    std::vector<std::vector<T>> cols;
};

struct Mix { static inline uint64_t mix64(uint64_t v) {
    v += 0x9E3779B97F4A7C15ull;
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
    return v ^ (v >> 31);
} };

template <class T>
static bool interp_point(const Particles<T>& P, const Tree<T>& tr, const Catalog& cat, const T pa[3], T ha, int mode, T* out) {
    const T K = kern_support<T>();
    const T radius = K * ha;
    const T radius2 = radius * radius;
    const int NS = cat.ns, NG = cat.ng, ND = cat.nd, NC = cat.nc;
    T S1 = 0;
    std::vector<T> sc(NS, 0), gf(3 * NG, 0), gb(3 * NG, 0), gs(NG, 0);
    std::vector<T> df(ND, 0), db(3 * ND, 0), ds(3 * ND, 0), cf(3 * NC, 0), cb(3 * NC, 0), cs(3 * NC, 0);
    auto Wof = [&](T dr, T hb) -> T {
        if (mode == GATHER) return kernel_W(dr, ha);
        if (mode == SCATTER) return kernel_W(dr, hb);
        return T(0.5) * (kernel_W(dr, ha) + kernel_W(dr, hb));
    };
    auto gWof = [&](T dx, T dy, T dz, T hb, T& gx, T& gy, T& gz) {
        if (mode == GATHER) { kernel_gradW(dx, dy, dz, ha, gx, gy, gz); return; }
        if (mode == SCATTER) { kernel_gradW(dx, dy, dz, hb, gx, gy, gz); return; }
        T ax, ay, az, bx, by, bz;
        kernel_gradW(dx, dy, dz, ha, ax, ay, az);
        kernel_gradW(dx, dy, dz, hb, bx, by, bz);
        gx = T(0.5) * (ax + bx); gy = T(0.5) * (ay + by); gz = T(0.5) * (az + bz);
    };
    bool ok = traverse<T, false>(tr, pa, pa, mode, K, [&]() { return radius2; },
        [&](int64_t li, T d2, T hb) {
            T dx = pa[0] - P.x[li], dy = pa[1] - P.y[li], dz = pa[2] - P.z[li];
            T dr = std::sqrt(d2);
            T mb = P.m[li], rb = P.rho[li];
            T W = Wof(dr, hb);
            T mbWlrb = mb * W / rb;          // _ShepardNormalization_accumulation
            S1 += mbWlrb;
            for (int j = 0; j < NS; ++j) sc[j] += P.cols[cat.sslot[j]][li] * mbWlrb;
            bool need_grad = (NG + ND + NC) > 0;
            T gx = 0, gy = 0, gz = 0;
            if (need_grad) gWof(dx, dy, dz, hb, gx, gy, gz);
            T invrb = T(1) / rb;
            for (int j = 0; j < NG; ++j) {
                int s = cat.gslot[j];
                if (s < 0) {  // _gradient_density_accumulation + _density_accumulation
                    T ax = mb * gx, ay = mb * gy, az = mb * gz;
                    gf[3*j] += ax; gf[3*j+1] += ay; gf[3*j+2] += az;
                    gb[3*j] += ax * invrb; gb[3*j+1] += ay * invrb; gb[3*j+2] += az * invrb;
                    gs[j] += mb * W;
                } else {       // _gradient_quantity_accumulation
                    T Ab = P.cols[s][li];
                    T ax = mb * invrb * gx, ay = mb * invrb * gy, az = mb * invrb * gz;
                    gf[3*j] += ax * Ab; gf[3*j+1] += ay * Ab; gf[3*j+2] += az * Ab;
                    gb[3*j] += ax; gb[3*j+1] += ay; gb[3*j+2] += az;
                    gs[j] += Ab * mbWlrb;
                }
            }
            for (int j = 0; j < ND; ++j) {   // _divergence_quantity_accumulation
                T Ax = P.cols[cat.dslot[3*j]][li], Ay = P.cols[cat.dslot[3*j+1]][li], Az = P.cols[cat.dslot[3*j+2]][li];
                T ax = mb * invrb * gx, ay = mb * invrb * gy, az = mb * invrb * gz;
                df[j] += ax * Ax + ay * Ay + az * Az;
                db[3*j] += ax; db[3*j+1] += ay; db[3*j+2] += az;
                ds[3*j] += Ax * mbWlrb; ds[3*j+1] += Ay * mbWlrb; ds[3*j+2] += Az * mbWlrb;
            }
            for (int j = 0; j < NC; ++j) {   // _curl_quantity_accumulation
                T Ax = P.cols[cat.cslot[3*j]][li], Ay = P.cols[cat.cslot[3*j+1]][li], Az = P.cols[cat.cslot[3*j+2]][li];
                T ax = mb * invrb * gx, ay = mb * invrb * gy, az = mb * invrb * gz;
                cf[3*j] += Ay * az - Az * ay;
                cf[3*j+1] += Az * ax - Ax * az;
                cf[3*j+2] += Ax * ay - Ay * ax;
                cb[3*j] += ax; cb[3*j+1] += ay; cb[3*j+2] += az;
                cs[3*j] += Ax * mbWlrb; cs[3*j+1] += Ay * mbWlrb; cs[3*j+2] += Az * mbWlrb;
            }
        });
    const int L = cat.L();
    if (S1 == T(0)) {   // general_interpolation.jl:128-131
        for (int k = 0; k < L; ++k) out[k] = std::numeric_limits<T>::quiet_NaN();
        return ok;
    }
    T invS1 = T(1) / S1;
    int o = 0;
    for (int j = 0; j < NS; ++j) out[o++] = cat.shep[j] ? sc[j] * invS1 : sc[j];
    for (int j = 0; j < NG; ++j) {
        T A = gs[j] * invS1;
        for (int d = 0; d < 3; ++d) out[o++] = gf[3*j+d] - gb[3*j+d] * A;
    }
    for (int j = 0; j < ND; ++j) {
        T Ax = ds[3*j] * invS1, Ay = ds[3*j+1] * invS1, Az = ds[3*j+2] * invS1;
        T Ab = Ax * db[3*j] + Ay * db[3*j+1] + Az * db[3*j+2];
        out[o++] = df[j] - Ab;
    }
    for (int j = 0; j < NC; ++j) {
        T Ax = cs[3*j] * invS1, Ay = cs[3*j+1] * invS1, Az = cs[3*j+2] * invS1;
        T bx = cb[3*j], by = cb[3*j+1], bz = cb[3*j+2];
        T Bx = Ay * bz - Az * by, By = Az * bx - Ax * bz, Bz = Ax * by - Ay * bx;
        out[o++] = -(cf[3*j] - Bx);
        out[o++] = -(cf[3*j+1] - By);
        out[o++] = -(cf[3*j+2] - Bz);
    }
    return ok;
}

// _line_integrated_quantities_interpolate_kernel,
// line_integrated_interpolation/kernels/line_integrated_scalar_interpolation.jl:76-214,
// accumulations/line_integrated_scalar_accumulation.jl:6-46.  A negative
// point-line d2 (rounding) is clamped to 0 before sqrt.
template <class T>
static bool interp_line(const Particles<T>& P, const Tree<T>& tr, const Catalog& cat, const T o[3], const T dir[3], T ha, int mode, T* out) {
    const T K = kern_support<T>();
    const T radius = K * ha;
    const T radius2 = radius * radius;
    T S1 = 0;
    std::vector<T> acc(cat.ns, 0);
    bool ok = traverse<T, true>(tr, o, dir, mode, K, [&]() { return radius2; },
        [&](int64_t li, T d2, T hb) {
            T dr = std::sqrt(d2 < T(0) ? T(0) : d2);
            T mb = P.m[li], rb = P.rho[li];
            T W;
            if (mode == GATHER) W = line_kernel(dr, ha);
            else if (mode == SCATTER) W = line_kernel(dr, hb);
            else W = T(0.5) * (line_kernel(dr, ha) + line_kernel(dr, hb));
            T mbWlr = mb * W / rb;
            S1 += mbWlr;
            for (int j = 0; j < cat.ns; ++j) acc[j] += P.cols[cat.sslot[j]][li] * mbWlr;
        });
    if (S1 == T(0)) {
        for (int j = 0; j < cat.ns; ++j) out[j] = std::numeric_limits<T>::quiet_NaN();
        return ok;
    }
    T invS1 = T(1) / S1;
    for (int j = 0; j < cat.ns; ++j) out[j] = cat.shep[j] ? acc[j] * invS1 : acc[j];
    return ok;
}

// _density_kernel, single_point_interpolation/kernels/scalar_interpolation.jl:1-75
// (mb * W per pair, accumulations/scalar_accumulation.jl:6-28); with number
// set, _number_density_kernel (:86-166), W per pair (scalar_accumulation.jl:31-52).
template <class T>
static bool density_point(const Particles<T>& P, const Tree<T>& tr, const T pa[3], T ha, int mode, T& out,
                          bool number = false) {
    const T K = kern_support<T>();
    const T radius = K * ha;
    const T radius2 = radius * radius;
    T rho = 0;
    bool ok = traverse<T, false>(tr, pa, pa, mode, K, [&]() { return radius2; },
        [&](int64_t li, T d2, T hb) {
            T dr = std::sqrt(d2);
            T mb = P.m[li];
            T W;
            if (mode == GATHER) W = kernel_W(dr, ha);
            else if (mode == SCATTER) W = kernel_W(dr, hb);
            else W = T(0.5) * (kernel_W(dr, ha) + kernel_W(dr, hb));
            rho += number ? W : mb * W;
        });
    out = rho;
    return ok;
}

// _gradient_density_kernel, single_point_interpolation/kernels/gradient_interpolation.jl:1-170:
// f = sum mb gradW, b = sum (mb gradW) / rho_b (accumulations/gradient_accumulation.jl:7-100),
// rho = sum mb W; NaN if rho == 0, else f - b rho.
template <class T>
static bool gradient_density_point(const Particles<T>& P, const Tree<T>& tr, const T pa[3], T ha, int mode, T out[3]) {
    const T K = kern_support<T>();
    const T radius = K * ha;
    const T radius2 = radius * radius;
    T f[3] = {0, 0, 0}, b[3] = {0, 0, 0}, rho = 0;
    bool ok = traverse<T, false>(tr, pa, pa, mode, K, [&]() { return radius2; },
        [&](int64_t li, T d2, T hb) {
            T dx = pa[0] - P.x[li], dy = pa[1] - P.y[li], dz = pa[2] - P.z[li];
            T dr = std::sqrt(d2);
            T mb = P.m[li], invrb = T(1) / P.rho[li];
            T g[3], W;
            if (mode == GATHER) {
                kernel_gradW(dx, dy, dz, ha, g[0], g[1], g[2]);
                W = kernel_W(dr, ha);
            } else if (mode == SCATTER) {
                kernel_gradW(dx, dy, dz, hb, g[0], g[1], g[2]);
                W = kernel_W(dr, hb);
            } else {
                T a[3], c[3];
                kernel_gradW(dx, dy, dz, ha, a[0], a[1], a[2]);
                kernel_gradW(dx, dy, dz, hb, c[0], c[1], c[2]);
                for (int d = 0; d < 3; ++d) g[d] = T(0.5) * (a[d] + c[d]);
                W = T(0.5) * (kernel_W(dr, ha) + kernel_W(dr, hb));
            }
            for (int d = 0; d < 3; ++d) {
                T mg = mb * g[d];
                f[d] += mg;
                b[d] += mg * invrb;
            }
            rho += mb * W;
        });
    for (int d = 0; d < 3; ++d) out[d] = rho == T(0) ? std::numeric_limits<T>::quiet_NaN() : f[d] - b[d] * rho;
    return ok;
}

// ---------------------------------------------------------------------------
// Adjoint (vector-Jacobian product) of the point and line interpolation for a
// loss L = sum_s sum_k gout_k(s) out_k(s), with respect to particle masses,
// columns and positions.  Densities and smoothing lengths are held fixed, and
// so is h_a: the nearest-particle h is piecewise constant in the positions.
// Written with the per-sample sums S1 = sum w, G = sum g, Sw_c = sum A_c w,
// Sg_c = sum A_c g, Dm = sum m W, Dg = sum m gradW (w = m/rho W,
// g = m/rho gradW), whose finalisation is the algebra of
// general_interpolation.jl:128-214 (and
// line_integrated_scalar_interpolation.jl:154-166 for lines).  The reference
// has no adjoint; this is the checker of the GPU adjoint and is itself checked
// against central finite differences of the forward restatement.
// ---------------------------------------------------------------------------

// M4 in terms of delta = p - x, r = |delta|, q = r/h (kernels/M4_spline.jl:13-36):
// gradW = sigma/h^5 g1(q) delta and Hessian = sigma/h^5 (g1 I + g2 q n n^T),
// with g1 = f'(q)/q, g2 = d g1/dq and n = delta/r.
template <class T> static inline void m4_g12(T q, T& g1, T& g2) {
    if (q < T(1)) {
        g1 = T(2.25) * q - T(3);
        g2 = T(2.25);
    } else if (q < T(2)) {
        T a = T(2) - q;
        g1 = T(-0.75) * a * a / q;
        g2 = T(0.75) * a * (q + T(2)) / (q * q);
    } else {
        g1 = T(0);
        g2 = T(0);
    }
}

// g1 = f'(q)/q and g2 = d g1/dq of the current kernel (g_kern), from the f'
// of kern_df and f'' of each piece: g2 = (f'' - g1)/q.  The pieces that
// contain q = 0 are written without the division: M5 on q < 1/2 and M6 on
// q < 1 are even polynomials there (f = 14.375 - 15 q^2 + 6 q^4 and
// 66 - 60 q^2 + 30 q^4 - 10 q^5), and the Wendland f' = q P(q) a^n factor
// exactly (a = 1 - q/2).
template <class T> static inline void kern_g12(T q, T& g1, T& g2) {
    g1 = T(0);
    g2 = T(0);
    T d1 = T(0), d2 = T(0);
    switch (g_kern) {
    case KERN_M5:
        if (q < T(0.5)) { g1 = T(-30) + T(24) * q * q; g2 = T(48) * q; return; }
        if (q < T(1.5)) {
            d1 = T(-4) * pw3(T(2.5) - q) + T(20) * pw3(T(1.5) - q);
            d2 = T(12) * pw2(T(2.5) - q) - T(60) * pw2(T(1.5) - q);
        } else if (q < T(2.5)) {
            d1 = T(-4) * pw3(T(2.5) - q);
            d2 = T(12) * pw2(T(2.5) - q);
        } else {
            return;
        }
        break;
    case KERN_M6:
        if (q < T(1)) { g1 = T(-120) + q * q * (T(120) - T(50) * q); g2 = q * (T(240) - T(150) * q); return; }
        if (q < T(2)) {
            d1 = T(-5) * pw4(T(3) - q) + T(30) * pw4(T(2) - q);
            d2 = T(20) * pw3(T(3) - q) - T(120) * pw3(T(2) - q);
        } else if (q < T(3)) {
            d1 = T(-5) * pw4(T(3) - q);
            d2 = T(20) * pw3(T(3) - q);
        } else {
            return;
        }
        break;
    case KERN_C2: case KERN_C4: case KERN_C6: {
        if (!(q < T(2))) return;
        const T a = T(1) - T(0.5) * q;
        if (g_kern == KERN_C2) {         // f' = -5 q a^3
            g1 = T(-5) * pw3(a);
            g2 = T(7.5) * pw2(a);
        } else if (g_kern == KERN_C4) {  // f' = -14/3 q (1 + 5q/2) a^5
            g1 = (T(-14) / T(3)) * (T(1) + T(2.5) * q) * pw5(a);
            g2 = T(35) * q * pw4(a);
        } else {                         // f' = -11/2 q (1 + 7q/2 + 4q^2) a^7
            g1 = T(-5.5) * (T(1) + T(3.5) * q + T(4) * q * q) * pw4(a) * pw3(a);
            g2 = T(33) * q * (T(1) + T(3) * q) * pw3(a) * pw3(a);
        }
        return;
    }
    default:
        m4_g12(q, g1, g2);
        return;
    }
    g1 = d1 / q;
    g2 = (d2 - g1) / q;
}

// W, gradW and the Hessian (xx, yy, zz, xy, xz, yz) with respect to delta
template <class T> static inline void kernel_whess(T dx, T dy, T dz, T h, T& W, T g[3], T H[6]) {
    T r2 = dx * dx + dy * dy + dz * dz;
    T r = std::sqrt(r2);
    W = kernel_W(r, h);
    kernel_gradW(dx, dy, dz, h, g[0], g[1], g[2]);
    T g1, g2;
    kern_g12(r / h, g1, g2);
    T s5 = kern_norm3<T>() / (h * h * h * h * h);
    T c = s5 * g1;
    T e = (r2 > T(0)) ? s5 * g2 * (r / h) / r2 : T(0);
    H[0] = c + e * dx * dx; H[1] = c + e * dy * dy; H[2] = c + e * dz * dz;
    H[3] = e * dx * dy; H[4] = e * dx * dz; H[5] = e * dy * dz;
}

template <class T> static inline void hess_mul(const T H[6], const T v[3], T out[3]) {
    out[0] = H[0] * v[0] + H[3] * v[1] + H[4] * v[2];
    out[1] = H[3] * v[0] + H[1] * v[1] + H[5] * v[2];
    out[2] = H[4] * v[0] + H[5] * v[1] + H[2] * v[2];
}

// Per-particle accumulator layout (Morton index li): [m, x, y, z, col 0, ...]
template <class T>
static bool adjoint_point(const Particles<T>& P, const Tree<T>& tr, const Catalog& cat, const T pa[3], T ha, int mode,
                          const T* gout, T* acc) {
    const T K = kern_support<T>();
    const T radius = K * ha;
    const T radius2 = radius * radius;
    const int nc = (int)P.cols.size();
    const int stride = 4 + nc;
    struct Nb { int64_t li; T hb; };
    std::vector<Nb> nb;
    bool ok = traverse<T, false>(tr, pa, pa, mode, K, [&]() { return radius2; },
                                 [&](int64_t li, T, T hb) { nb.push_back({li, hb}); });
    auto eval = [&](const Nb& b, T& W, T g[3], T H[6]) {
        T dx = pa[0] - P.x[b.li], dy = pa[1] - P.y[b.li], dz = pa[2] - P.z[b.li];
        if (mode == GATHER) { kernel_whess(dx, dy, dz, ha, W, g, H); return; }
        if (mode == SCATTER) { kernel_whess(dx, dy, dz, b.hb, W, g, H); return; }
        T Wa, ga[3], Ha[6], Wb, gb[3], Hb[6];
        kernel_whess(dx, dy, dz, ha, Wa, ga, Ha);
        kernel_whess(dx, dy, dz, b.hb, Wb, gb, Hb);
        W = T(0.5) * (Wa + Wb);
        for (int d = 0; d < 3; ++d) g[d] = T(0.5) * (ga[d] + gb[d]);
        for (int d = 0; d < 6; ++d) H[d] = T(0.5) * (Ha[d] + Hb[d]);
    };
    // sums
    T S1 = 0, G[3] = {0, 0, 0}, Dm = 0, Dg[3] = {0, 0, 0};
    std::vector<T> Sw(nc, T(0)), Sg(3 * nc, T(0));
    for (const Nb& b : nb) {
        T W, g[3], H[6];
        eval(b, W, g, H);
        const T m = P.m[b.li], mr = m / P.rho[b.li];
        S1 += mr * W;
        Dm += m * W;
        for (int d = 0; d < 3; ++d) { G[d] += mr * g[d]; Dg[d] += m * g[d]; }
        for (int c = 0; c < nc; ++c) {
            const T A = P.cols[c][b.li];
            Sw[c] += A * mr * W;
            for (int d = 0; d < 3; ++d) Sg[3 * c + d] += A * mr * g[d];
        }
    }
    if (S1 == T(0)) return ok;  // every output NaN, nothing flows back
    // cotangents of the sums
    const T inv = T(1) / S1, inv2 = inv * inv;
    T lS1 = 0, lG[3] = {0, 0, 0}, lDm = 0, lDg[3] = {0, 0, 0};
    std::vector<T> lSw(nc, T(0)), lSg(3 * nc, T(0));
    int o = 0;
    for (int j = 0; j < cat.ns; ++j) {
        const int c = cat.sslot[j];
        const T go = gout[o++];
        if (cat.shep[j]) { lSw[c] += go * inv; lS1 -= go * Sw[c] * inv2; }
        else lSw[c] += go;
    }
    for (int j = 0; j < cat.ng; ++j) {
        const int c = cat.gslot[j];
        for (int d = 0; d < 3; ++d) {
            const T go = gout[o++];
            if (c < 0) {  // Dg - G Dm / S1
                lDg[d] += go; lG[d] -= go * Dm * inv; lDm -= go * G[d] * inv; lS1 += go * G[d] * Dm * inv2;
            } else {      // Sg_c - G Sw_c / S1
                lSg[3 * c + d] += go; lG[d] -= go * Sw[c] * inv; lSw[c] -= go * G[d] * inv;
                lS1 += go * G[d] * Sw[c] * inv2;
            }
        }
    }
    for (int j = 0; j < cat.nd; ++j) {  // sum_d Sg_{c_d}[d] - sum_d Sw_{c_d}/S1 G[d]
        const T go = gout[o++];
        for (int d = 0; d < 3; ++d) {
            const int c = cat.dslot[3 * j + d];
            lSg[3 * c + d] += go; lG[d] -= go * Sw[c] * inv; lSw[c] -= go * G[d] * inv;
            lS1 += go * Sw[c] * G[d] * inv2;
        }
    }
    for (int j = 0; j < cat.nc; ++j) {
        const int cx = cat.cslot[3 * j], cy = cat.cslot[3 * j + 1], cz = cat.cslot[3 * j + 2];
        // component = -Sg_a[ka] + Sg_b[kb] + Sw_a/S1 G[ka] - Sw_b/S1 G[kb]
        const int a_[3] = {cy, cz, cx}, ka_[3] = {2, 0, 1}, b_[3] = {cz, cx, cy}, kb_[3] = {1, 2, 0};
        for (int d = 0; d < 3; ++d) {
            const T go = gout[o++];
            const int a = a_[d], ka = ka_[d], b = b_[d], kb = kb_[d];
            lSg[3 * a + ka] -= go; lSg[3 * b + kb] += go;
            lG[ka] += go * Sw[a] * inv; lG[kb] -= go * Sw[b] * inv;
            lSw[a] += go * G[ka] * inv; lSw[b] -= go * G[kb] * inv;
            lS1 -= go * (Sw[a] * G[ka] - Sw[b] * G[kb]) * inv2;
        }
    }
    // pair terms
    for (const Nb& b : nb) {
        T W, g[3], H[6];
        eval(b, W, g, H);
        const T m = P.m[b.li], rho = P.rho[b.li], mr = m / rho;
        T aS = lS1, aG[3] = {lG[0], lG[1], lG[2]};
        for (int c = 0; c < nc; ++c) {
            const T A = P.cols[c][b.li];
            aS += lSw[c] * A;
            for (int d = 0; d < 3; ++d) aG[d] += A * lSg[3 * c + d];
        }
        T* a = acc + b.li * stride;
        a[0] += (aS * W + aG[0] * g[0] + aG[1] * g[1] + aG[2] * g[2]) / rho + lDm * W +
                lDg[0] * g[0] + lDg[1] * g[1] + lDg[2] * g[2];
        for (int c = 0; c < nc; ++c)
            a[4 + c] += mr * (lSw[c] * W + lSg[3 * c] * g[0] + lSg[3 * c + 1] * g[1] + lSg[3 * c + 2] * g[2]);
        T Ha[3], Hd[3];
        hess_mul(H, aG, Ha);
        hess_mul(H, lDg, Hd);
        for (int d = 0; d < 3; ++d)  // delta = p - x_b
            a[1 + d] -= mr * (aS * g[d] + Ha[d]) + m * (lDm * g[d] + Hd[d]);
    }
    return ok;
}

// line_integrated_kernel_function and its derivative in r: the slope of the
// table segment that lin_lut interpolates on (line_integrated_kernel.jl:13-19)
template <class T> static inline void line_kernel_d(T r, T h, T& W, T& dW) {
    const T invh = T(1) / h;
    const T q = r * invh;
    if (q >= kern_support<T>()) { W = T(0); dW = T(0); return; }
    const T* Q = lut_Q<T>();
    const T* I = lut_I<T>();
    const T dq = Q[1] - Q[0];
    const T idxf = q / dq + T(1);
    int32_t i = (int32_t)idxf;
    if (i < 1) i = 1;
    if (i > LUT_N - 1) i = LUT_N - 1;
    const T t = idxf - T(i);
    W = invh * (I[i - 1] * (T(1) - t) + I[i] * t);
    dW = invh * invh * (I[i] - I[i - 1]) / dq;
}

template <class T>
static bool adjoint_line(const Particles<T>& P, const Tree<T>& tr, const Catalog& cat, const T o[3], const T dir[3],
                         T ha, int mode, const T* gout, T* acc) {
    const T K = kern_support<T>();
    const T radius = K * ha;
    const T radius2 = radius * radius;
    const int nc = (int)P.cols.size();
    const int stride = 4 + nc;
    struct Nb { int64_t li; T d2, hb; };
    std::vector<Nb> nb;
    bool ok = traverse<T, true>(tr, o, dir, mode, K, [&]() { return radius2; },
                                [&](int64_t li, T d2, T hb) { nb.push_back({li, d2, hb}); });
    auto eval = [&](const Nb& b, T& W, T& dW) {
        const T dr = std::sqrt(b.d2 < T(0) ? T(0) : b.d2);
        if (mode == GATHER) { line_kernel_d(dr, ha, W, dW); return; }
        if (mode == SCATTER) { line_kernel_d(dr, b.hb, W, dW); return; }
        T Wa, da, Wb, db;
        line_kernel_d(dr, ha, Wa, da);
        line_kernel_d(dr, b.hb, Wb, db);
        W = T(0.5) * (Wa + Wb);
        dW = T(0.5) * (da + db);
    };
    T S1 = 0;
    std::vector<T> Sw(nc, T(0));
    for (const Nb& b : nb) {
        T W, dW;
        eval(b, W, dW);
        const T mr = P.m[b.li] / P.rho[b.li];
        S1 += mr * W;
        for (int c = 0; c < nc; ++c) Sw[c] += P.cols[c][b.li] * mr * W;
    }
    if (S1 == T(0)) return ok;
    const T inv = T(1) / S1;
    T lS1 = 0;
    std::vector<T> lSw(nc, T(0));
    for (int j = 0; j < cat.ns; ++j) {
        const int c = cat.sslot[j];
        const T go = gout[j];
        if (cat.shep[j]) { lSw[c] += go * inv; lS1 -= go * Sw[c] * inv * inv; }
        else lSw[c] += go;
    }
    for (const Nb& b : nb) {
        T W, dW;
        eval(b, W, dW);
        const T rho = P.rho[b.li], mr = P.m[b.li] / rho;
        T aS = lS1;
        for (int c = 0; c < nc; ++c) aS += lSw[c] * P.cols[c][b.li];
        T* a = acc + b.li * stride;
        a[0] += aS * W / rho;
        for (int c = 0; c < nc; ++c) a[4 + c] += mr * lSw[c] * W;
        // d r_perp / d x_b = (D - (D.m) m) / r_perp with D = x_b - o
        const T D[3] = {P.x[b.li] - o[0], P.y[b.li] - o[1], P.z[b.li] - o[2]};
        const T Dm = D[0] * dir[0] + D[1] * dir[1] + D[2] * dir[2];
        const T dr = std::sqrt(b.d2 < T(0) ? T(0) : b.d2);
        if (dr > T(0))
            for (int d = 0; d < 3; ++d) a[1 + d] += mr * aS * dW * (D[d] - Dm * dir[d]) / dr;
    }
    return ok;
}

}  // namespace orc

// ===========================================================================
// extern "C" API used by the Python test harness (ctypes).
// ===========================================================================
using namespace orc;

struct orc_ctx {
    int dtype = 0;  // 0 = double, 1 = float
    Particles<double> Pd; Particles<float> Pf;
    Tree<double> Td; Tree<float> Tf;
    bool built = false;
};

template <class T> static Particles<T>& parts(orc_ctx* c);
template <> Particles<double>& parts<double>(orc_ctx* c) { return c->Pd; }
template <> Particles<float>& parts<float>(orc_ctx* c) { return c->Pf; }
template <class T> static Tree<T>& tree(orc_ctx* c);
template <> Tree<double>& tree<double>(orc_ctx* c) { return c->Td; }
template <> Tree<float>& tree<float>(orc_ctx* c) { return c->Tf; }

#define ORC_API extern "C" __attribute__((visibility("default")))

ORC_API int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n; return 1;
#endif
}

ORC_API double orc_W(double r, double h) { return kernel_W<double>(r, h); }
ORC_API float orc_Wf(float r, float h) { return kernel_W<float>(r, h); }
ORC_API double orc_f(double q) { return kern_f<double>(q); }
ORC_API double orc_df(double q) { return kern_df<double>(q); }
ORC_API double orc_support(void) { return kern_support<double>(); }
ORC_API double orc_norm3(void) { return kern_norm3<double>(); }
// The kernel family of the following calls (0 M4, 1 M5, 2 M6, 3 C2, 4 C4, 5 C6).
ORC_API int orc_set_kernel(int k) {
    if (k < 0 || k >= KERN_COUNT) return -1;
    g_kern = k;
    return 0;
}
ORC_API void orc_gradW(double dx, double dy, double dz, double h, double* g) { kernel_gradW<double>(dx, dy, dz, h, g[0], g[1], g[2]); }
ORC_API double orc_line_kernel(double r, double h) { return line_kernel<double>(r, h); }
ORC_API float orc_line_kernelf(float r, float h) { return line_kernel<float>(r, h); }
ORC_API void orc_line_table(double* Q, double* I) {
    std::memcpy(Q, line_table().Q, sizeof(double) * LUT_N);
    std::memcpy(I, line_table().I, sizeof(double) * LUT_N);
}

ORC_API orc_ctx* orc_create(int64_t n, int dtype, const void* x, const void* y, const void* z,
                    const void* m, const void* h, const void* rho, int ncol, const void* const* cols) {
    orc_ctx* c = new (std::nothrow) orc_ctx();
    if (!c) return nullptr;
    c->dtype = dtype;
    auto fill = [&](auto& P, auto tag) {
        using T = decltype(tag);
        P.n = n;
        auto cp = [&](std::vector<T>& v, const void* p) { v.assign((const T*)p, (const T*)p + n); };
        cp(P.x, x); cp(P.y, y); cp(P.z, z); cp(P.m, m); cp(P.h, h); cp(P.rho, rho);
        P.cols.resize(ncol);
        for (int k = 0; k < ncol; ++k) cp(P.cols[k], cols[k]);
    };
    if (dtype == 0) fill(c->Pd, double()); else fill(c->Pf, float());
    return c;
}

ORC_API void orc_destroy(orc_ctx* c) { delete c; }

template <class T> static int build_impl(orc_ctx* c, int64_t* perm, uint64_t* codes) {
    Particles<T>& P = parts<T>(c);
    Tree<T>& tr = tree<T>(c);
    if (P.n < 1) return -1;
    if (P.n > (int64_t)1073741824) return -1;
    build_tree<T>(tr, P.x.data(), P.y.data(), P.z.data(), P.h.data(), P.n);
    // LinearBVH!(input): permute every particle array into Morton order
    auto perm_vec = [&](std::vector<T>& v) {
        std::vector<T> t(P.n);
        for (int64_t i = 0; i < P.n; ++i) t[i] = v[tr.order[i]];
        v.swap(t);
    };
    perm_vec(P.x); perm_vec(P.y); perm_vec(P.z); perm_vec(P.m); perm_vec(P.h); perm_vec(P.rho);
    for (auto& col : P.cols) perm_vec(col);
    if (perm) for (int64_t i = 0; i < P.n; ++i) perm[i] = tr.order[i];
    if (codes) for (int64_t i = 0; i < P.n; ++i) codes[i] = tr.codes[i];
    c->built = true;
    return 0;
}

ORC_API int orc_build(orc_ctx* c, int64_t* perm, uint64_t* codes) {
    return c->dtype == 0 ? build_impl<double>(c, perm, codes) : build_impl<float>(c, perm, codes);
}

// Failure injection for the tests: every escape link that ends a walk (0:
// the right spine and the last leaf) is pointed at the root, so every
// traversal cycles until its step bound and the call reports it (-5).
// orc_build restores the tree.
template <class T> static int loop_escapes_impl(orc_ctx* c) {
    Tree<T>& tr = tree<T>(c);
    if (tr.root == 0) return -1;
    for (auto& e : tr.escape)
        if (e == 0) e = tr.root;
    return 0;
}

ORC_API int orc_test_loop_escapes(orc_ctx* c) {
    if (!c->built) return -7;
    return c->dtype == 0 ? loop_escapes_impl<double>(c) : loop_escapes_impl<float>(c);
}

template <class T> static void get_tree_impl(orc_ctx* c, int32_t* root, int32_t* l, int32_t* r, int32_t* e, int32_t* p,
                                             double* nmin, double* nmax, double* nscale) {
    Tree<T>& tr = tree<T>(c);
    int64_t total = 2 * tr.n - 1, nint = tr.n - 1;
    if (root) *root = tr.root;
    for (int64_t i = 0; i < total; ++i) {
        if (l) l[i] = tr.left[i];
        if (r) r[i] = tr.right[i];
        if (e) e[i] = tr.escape[i];
        if (p) p[i] = tr.parent[i];
    }
    for (int64_t i = 0; i < nint; ++i) {
        for (int d = 0; d < 3; ++d) {
            if (nmin) nmin[d * nint + i] = (double)tr.nmin[d][i];
            if (nmax) nmax[d * nint + i] = (double)tr.nmax[d][i];
        }
        if (nscale) nscale[i] = (double)tr.nscale[i];
    }
}

ORC_API int orc_get_tree(orc_ctx* c, int32_t* root, int32_t* l, int32_t* r, int32_t* e, int32_t* p,
                 double* nmin, double* nmax, double* nscale) {
    if (!c->built) return -7;
    if (c->dtype == 0) get_tree_impl<double>(c, root, l, r, e, p, nmin, nmax, nscale);
    else get_tree_impl<float>(c, root, l, r, e, p, nmin, nmax, nscale);
    return 0;
}

// hmode: 0 nearest, 1 per-sample, 2 constant; mode: 0 gather, 1 scatter, 2 symmetric
template <class T> static T sample_h(const Tree<T>& tr, const T p[3], int hmode, const T* hs, int64_t i, bool& ok) {
    ok = true;
    if (hmode == 0) return nearest_h(tr, p, ok);
    if (hmode == 1) return hs[i];
    return hs[0];
}

template <class T> static int interp_points_impl(orc_ctx* c, int64_t ns, const T* sx, const T* sy, const T* sz,
                                                 int hmode, const T* hs, int mode, const Catalog& cat, T* const* out) {
    Particles<T>& P = parts<T>(c);
    Tree<T>& tr = tree<T>(c);
    std::atomic<int> bad(0);
    const int L = cat.L();
    #pragma omp parallel
    {
        std::vector<T> buf(L > 0 ? L : 1);
        #pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < ns; ++i) {
            T p[3] = {sx[i], sy[i], sz[i]};
            bool ok1 = true, ok2;
            T ha = (mode == SCATTER) ? T(0) : sample_h(tr, p, hmode, hs, i, ok1);
            ok2 = interp_point(P, tr, cat, p, ha, mode, buf.data());
            if (!ok1 || !ok2) bad = 1;
            for (int k = 0; k < L; ++k) out[k][i] = buf[k];
        }
    }
    return bad ? -5 : 0;
}

static Catalog make_cat(int ns, const int32_t* ss, const uint8_t* sh, int ng, const int32_t* gs,
                        int nd, const int32_t* ds, int nc, const int32_t* cs) {
    Catalog cat;
    cat.ns = ns; cat.sslot = ss; cat.shep = sh; cat.ng = ng; cat.gslot = gs;
    cat.nd = nd; cat.dslot = ds; cat.nc = nc; cat.cslot = cs;
    return cat;
}

ORC_API int orc_interp_points(orc_ctx* c, int64_t ns, const void* sx, const void* sy, const void* sz,
                      int hmode, const void* hs, int mode,
                      int nsc, const int32_t* ss, const uint8_t* sh, int ng, const int32_t* gs,
                      int nd, const int32_t* ds, int nc, const int32_t* cs, void* const* out) {
    if (!c->built) return -7;
    Catalog cat = make_cat(nsc, ss, sh, ng, gs, nd, ds, nc, cs);
    if (c->dtype == 0)
        return interp_points_impl<double>(c, ns, (const double*)sx, (const double*)sy, (const double*)sz, hmode,
                                          (const double*)hs, mode, cat, (double* const*)out);
    return interp_points_impl<float>(c, ns, (const float*)sx, (const float*)sy, (const float*)sz, hmode,
                                     (const float*)hs, mode, cat, (float* const*)out);
}

template <class T> static int interp_lines_impl(orc_ctx* c, int64_t nl, const T* const* od, int hmode, const T* hs,
                                                int mode, const Catalog& cat, T* const* out) {
    Particles<T>& P = parts<T>(c);
    Tree<T>& tr = tree<T>(c);
    std::atomic<int> bad(0);
    #pragma omp parallel
    {
        std::vector<T> buf(cat.ns > 0 ? cat.ns : 1);
        #pragma omp for schedule(dynamic, 16)
        for (int64_t i = 0; i < nl; ++i) {
            T o[3] = {od[0][i], od[1][i], od[2][i]};
            T d[3] = {od[3][i], od[4][i], od[5][i]};
            T ha = T(0);
            if (mode != SCATTER) ha = (hmode == 1) ? hs[i] : hs[0];
            if (!interp_line(P, tr, cat, o, d, ha, mode, buf.data())) bad = 1;
            for (int k = 0; k < cat.ns; ++k) out[k][i] = buf[k];
        }
    }
    return bad ? -5 : 0;
}

ORC_API int orc_interp_lines(orc_ctx* c, int64_t nl, const void* const* od, int hmode, const void* hs, int mode,
                     int nsc, const int32_t* ss, const uint8_t* sh, void* const* out) {
    if (!c->built) return -7;
    if (mode != SCATTER && hmode == 0) return -1;
    Catalog cat = make_cat(nsc, ss, sh, 0, nullptr, 0, nullptr, 0, nullptr);
    if (c->dtype == 0)
        return interp_lines_impl<double>(c, nl, (const double* const*)od, hmode, (const double*)hs, mode, cat, (double* const*)out);
    return interp_lines_impl<float>(c, nl, (const float* const*)od, hmode, (const float*)hs, mode, cat, (float* const*)out);
}

template <class T> static int density_impl(orc_ctx* c, int64_t ns, const T* sx, const T* sy, const T* sz,
                                           int hmode, const T* hs, int mode, T* out, int what) {
    Particles<T>& P = parts<T>(c);
    Tree<T>& tr = tree<T>(c);
    std::atomic<int> bad(0);
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < ns; ++i) {
        T p[3] = {sx[i], sy[i], sz[i]};
        bool ok1 = true;
        T ha = (mode == SCATTER) ? T(0) : sample_h(tr, p, hmode, hs, i, ok1);
        bool ok2;
        if (what == 2) {  // gradient of the density: out holds 3 ns values, component-major
            T g[3];
            ok2 = gradient_density_point(P, tr, p, ha, mode, g);
            for (int d = 0; d < 3; ++d) out[d * ns + i] = g[d];
        } else {
            T v;
            ok2 = density_point(P, tr, p, ha, mode, v, what == 1);
            out[i] = v;
        }
        if (!ok1 || !ok2) bad = 1;
    }
    return bad ? -5 : 0;
}

// what: 0 _density_kernel, 1 _number_density_kernel, 2 _gradient_density_kernel
ORC_API int orc_density(orc_ctx* c, int64_t ns, const void* sx, const void* sy, const void* sz,
                int hmode, const void* hs, int mode, void* out, int what) {
    if (!c->built) return -7;
    if (what < 0 || what > 2) return -1;
    if (c->dtype == 0)
        return density_impl<double>(c, ns, (const double*)sx, (const double*)sy, (const double*)sz, hmode,
                                    (const double*)hs, mode, (double*)out, what);
    return density_impl<float>(c, ns, (const float*)sx, (const float*)sy, (const float*)sz, hmode,
                               (const float*)hs, mode, (float*)out, what);
}

// Neighbour digest through the stackless traversal (kind 0 points, 1 lines).
template <class T> static int digest_impl(orc_ctx* c, int kind, int64_t ns, const T* const* a, int hmode, const T* hs,
                                          int mode, int64_t* cnt, uint64_t* hsh, T* ha_out) {
    Tree<T>& tr = tree<T>(c);
    std::atomic<int> bad(0);
    const T K = kern_support<T>();
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < ns; ++i) {
        T p[3] = {a[0][i], a[1][i], a[2][i]};
        T d[3] = {T(0), T(0), T(0)};
        if (kind == 1) { d[0] = a[3][i]; d[1] = a[4][i]; d[2] = a[5][i]; }
        bool ok1 = true;
        T ha = T(0);
        if (mode != SCATTER) {
            if (kind == 0) ha = sample_h(tr, p, hmode, hs, i, ok1);
            else ha = (hmode == 1) ? hs[i] : hs[0];
        }
        T radius = K * ha;
        T r2 = radius * radius;
        int64_t count = 0; uint64_t hash = 0;
        auto hit = [&](int64_t li, T, T) { ++count; hash += Mix::mix64((uint64_t)(li + 1)); };
        bool ok2 = (kind == 0) ? traverse<T, false>(tr, p, d, mode, K, [&]() { return r2; }, hit)
                               : traverse<T, true>(tr, p, d, mode, K, [&]() { return r2; }, hit);
        if (!ok1 || !ok2) bad = 1;
        cnt[i] = count; hsh[i] = hash;
        if (ha_out) ha_out[i] = ha;
    }
    return bad ? -5 : 0;
}

ORC_API int orc_neighbor_digest(orc_ctx* c, int kind, int64_t ns, const void* const* a, int hmode, const void* hs, int mode,
                        int64_t* cnt, uint64_t* hsh, void* ha_out) {
    if (!c->built) return -7;
    if (kind == 1 && mode != SCATTER && hmode == 0) return -1;
    if (c->dtype == 0)
        return digest_impl<double>(c, kind, ns, (const double* const*)a, hmode, (const double*)hs, mode, cnt, hsh, (double*)ha_out);
    return digest_impl<float>(c, kind, ns, (const float* const*)a, hmode, (const float*)hs, mode, cnt, hsh, (float*)ha_out);
}

// Brute-force neighbour digest (no tree): the reference tests compare every
// traversal with an O(N) scan (test/neighbor_search_tests.jl:309-457).
template <class T> static void brute_impl(orc_ctx* c, int kind, int64_t ns, const T* const* a, const T* ha_in,
                                          int mode, int64_t* cnt, uint64_t* hsh) {
    Tree<T>& tr = tree<T>(c);
    const T K = kern_support<T>();
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < ns; ++i) {
        T p[3] = {a[0][i], a[1][i], a[2][i]};
        T d[3] = {T(0), T(0), T(0)};
        if (kind == 1) { d[0] = a[3][i]; d[1] = a[4][i]; d[2] = a[5][i]; }
        T ha = (mode == SCATTER) ? T(0) : ha_in[i];
        T r = K * ha; T r2a = r * r;
        int64_t count = 0; uint64_t hash = 0;
        for (int64_t li = 0; li < tr.n; ++li) {
            T d2 = (kind == 0) ? d2_point_leaf(tr, p, li) : d2_line_point(p, d, tr.lx[li], tr.ly[li], tr.lz[li]);
            T rb = K * tr.lh[li];
            T r2 = (mode == GATHER) ? r2a : (mode == SCATTER ? rb * rb : jmax(r2a, rb * rb));
            if (d2 <= r2) { ++count; hash += Mix::mix64((uint64_t)(li + 1)); }
        }
        cnt[i] = count; hsh[i] = hash;
    }
}

ORC_API int orc_brute_digest(orc_ctx* c, int kind, int64_t ns, const void* const* a, const void* ha, int mode,
                     int64_t* cnt, uint64_t* hsh) {
    if (!c->built) return -7;
    if (c->dtype == 0) brute_impl<double>(c, kind, ns, (const double* const*)a, (const double*)ha, mode, cnt, hsh);
    else brute_impl<float>(c, kind, ns, (const float* const*)a, (const float*)ha, mode, cnt, hsh);
    return 0;
}

// Brute-force nearest particle (argmin d2, ties to the smallest Morton index).
ORC_API int orc_brute_nearest(orc_ctx* c, int64_t ns, const double* sx, const double* sy, const double* sz, int64_t* idx) {
    if (!c->built || c->dtype != 0) return -7;
    Tree<double>& tr = c->Td;
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < ns; ++i) {
        double p[3] = {sx[i], sy[i], sz[i]};
        int64_t best = -1; double b2 = std::numeric_limits<double>::infinity();
        for (int64_t li = 0; li < tr.n; ++li) {
            double d2 = d2_point_leaf(tr, p, li);
            if (d2 < b2) { b2 = d2; best = li; }
        }
        idx[i] = best;
    }
    return 0;
}

// Morton codes alone (unsorted), for the quantisation known-answer tests.
ORC_API int orc_morton_codes(int64_t n, int dtype, const void* x, const void* y, const void* z, uint64_t* codes) {
    std::vector<uint64_t> c;
    if (dtype == 0) morton_codes((const double*)x, (const double*)y, (const double*)z, n, c);
    else morton_codes((const float*)x, (const float*)y, (const float*)z, n, c);
    std::memcpy(codes, c.data(), sizeof(uint64_t) * n);
    return 0;
}


// Adjoint of orc_interp_points / orc_interp_lines (double particles only):
// gout[k] holds the cotangent of output field k per sample; gm, gcols[c], gx,
// gy, gz receive dL/dm, dL/dA_c, dL/dx.. per particle in the order the
// particles were given to orc_create.
template <class F>
static int adjoint_impl(orc_ctx* c, int64_t ns, F per_sample, void* gm, void* const* gcols, void* gx, void* gy, void* gz) {
    Particles<double>& P = c->Pd;
    Tree<double>& tr = c->Td;
    const int nc = (int)P.cols.size();
    const int stride = 4 + nc;
    std::vector<double> acc((size_t)P.n * stride, 0.0);
    std::atomic<int> bad(0);
    #pragma omp parallel
    {
        std::vector<double> mine((size_t)P.n * stride, 0.0);
        #pragma omp for schedule(dynamic, 16)
        for (int64_t i = 0; i < ns; ++i)
            if (!per_sample(i, mine.data())) bad = 1;
        #pragma omp critical
        for (size_t k = 0; k < mine.size(); ++k) acc[k] += mine[k];
    }
    for (int64_t i = 0; i < P.n; ++i) {
        const int64_t j = tr.order[i];  // original index of Morton position i
        const double* a = acc.data() + (size_t)i * stride;
        if (gm) ((double*)gm)[j] = a[0];
        if (gx) ((double*)gx)[j] = a[1];
        if (gy) ((double*)gy)[j] = a[2];
        if (gz) ((double*)gz)[j] = a[3];
        for (int k = 0; k < nc; ++k)
            if (gcols && gcols[k]) ((double*)gcols[k])[j] = a[4 + k];
    }
    return bad ? -5 : 0;
}

ORC_API int orc_adjoint_points(orc_ctx* c, int64_t ns, const void* sx, const void* sy, const void* sz,
                               int hmode, const void* hs, int mode,
                               int nsc, const int32_t* ss, const uint8_t* sh, int ng, const int32_t* gs,
                               int nd, const int32_t* ds, int nc, const int32_t* cs, const void* const* gout,
                               void* gm, void* const* gcols, void* gx, void* gy, void* gz) {
    if (!c->built) return -7;
    if (c->dtype != 0) return -6;
    Catalog cat = make_cat(nsc, ss, sh, ng, gs, nd, ds, nc, cs);
    const int L = cat.L();
    const double* X = (const double*)sx; const double* Y = (const double*)sy; const double* Z = (const double*)sz;
    const double* const* GO = (const double* const*)gout;
    return adjoint_impl(c, ns, [&](int64_t i, double* acc) {
        double p[3] = {X[i], Y[i], Z[i]};
        bool ok1 = true;
        double ha = (mode == SCATTER) ? 0.0 : sample_h(c->Td, p, hmode, (const double*)hs, i, ok1);
        std::vector<double> go(L > 0 ? L : 1);
        for (int k = 0; k < L; ++k) go[k] = GO[k][i];
        return adjoint_point(c->Pd, c->Td, cat, p, ha, mode, go.data(), acc) && ok1;
    }, gm, gcols, gx, gy, gz);
}

ORC_API int orc_adjoint_lines(orc_ctx* c, int64_t nl, const void* const* od, int hmode, const void* hs, int mode,
                              int nsc, const int32_t* ss, const uint8_t* sh, const void* const* gout,
                              void* gm, void* const* gcols, void* gx, void* gy, void* gz) {
    if (!c->built) return -7;
    if (c->dtype != 0) return -6;
    if (mode != SCATTER && hmode == 0) return -1;
    Catalog cat = make_cat(nsc, ss, sh, 0, nullptr, 0, nullptr, 0, nullptr);
    const double* const* A = (const double* const*)od;
    const double* const* GO = (const double* const*)gout;
    return adjoint_impl(c, nl, [&](int64_t i, double* acc) {
        double o[3] = {A[0][i], A[1][i], A[2][i]}, d[3] = {A[3][i], A[4][i], A[5][i]};
        double ha = 0.0;
        if (mode != SCATTER) ha = (hmode == 1) ? ((const double*)hs)[i] : ((const double*)hs)[0];
        std::vector<double> go(cat.ns > 0 ? cat.ns : 1);
        for (int k = 0; k < cat.ns; ++k) go[k] = GO[k][i];
        return adjoint_line(c->Pd, c->Td, cat, o, d, ha, mode, go.data(), acc);
    }, gm, gcols, gx, gy, gz);
}
