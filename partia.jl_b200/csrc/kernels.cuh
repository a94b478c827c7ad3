// kernels.cuh -- the SPH kernel families other than M4
// (kernel_function/kernels/M5_spline.jl, M6_spline.jl, C2_Wendland.jl,
// C4_Wendland.jl, C6_Wendland.jl): support K in units of h
// (KernelFunctionValid), the 3D norm (KernelFunctionnorm(K, Val(3), T)) and
// f, f' of the dimensionless kernel (and f'/q with its q-derivative for the
// adjoint).  Ids follow psb_kernel.  M4 keeps its own functions (m4_fdf,
// m4_fdf_edge in interp.cuh, m4_whess in k_adjoint.cuh).
#pragma once

namespace psb {

enum { KERN_M4 = 0, KERN_M5 = 1, KERN_M6 = 2, KERN_C2 = 3, KERN_C4 = 4, KERN_C6 = 5, KERN_COUNT = 6 };

__host__ __device__ inline double kern_support(int k) {
    return k == KERN_M5 ? 2.5 : (k == KERN_M6 ? 3.0 : 2.0);
}

__host__ __device__ inline double kern_norm3(int k) {
    const double pi = 3.141592653589793;
    switch (k) {
    case KERN_M5: return 0.05 / pi;
    case KERN_M6: return 1.0 / (120.0 * pi);
    case KERN_C2: return 21.0 / (16.0 * pi);
    case KERN_C4: return 495.0 / (256.0 * pi);
    case KERN_C6: return 1365.0 / (512.0 * pi);
    default: return 0.31830988618379067154;
    }
}

// First q of the piece that reaches the support edge: from there on the float
// pair sums of M4, M5 and M6 take K - q from K^2 h^2 - d^2 formed in double
// (see kern_fdf_f32).  The Wendland families take q and 1 - q/2 from the
// exact separation for every q (f32c_wendland_weights in interp.cuh).
__host__ __device__ inline float kern_qedge(int k) {
    return k == KERN_M5 ? 1.5f : (k == KERN_M6 ? 2.f : 1.f);
}

// f and f' for k != M4 at q >= 0, in the reference's piecewise forms; the
// Wendland derivatives are written in their factored form
// (C2: f' = -5 q a^3, C4: -14/3 q (1 + 5q/2) a^5, C6: -11/2 q (1 + 7q/2 + 4q^2) a^7,
// a = 1 - q/2), the same polynomials without the cancellation at small q.
template <class C> __device__ __forceinline__ void kern_fdf(int k, C q, C& f, C& df) {
    f = C(0);
    df = C(0);
    switch (k) {
    case KERN_M5: {
        const C a = C(2.5) - q, b = C(1.5) - q, c = C(0.5) - q;
        const C a3 = a * a * a, b3 = b * b * b, c3 = c * c * c;
        if (q < C(0.5)) {
            f = a3 * a - C(5) * (b3 * b) + C(10) * (c3 * c);
            df = C(-4) * a3 + C(20) * b3 - C(40) * c3;
        } else if (q < C(1.5)) {
            f = a3 * a - C(5) * (b3 * b);
            df = C(-4) * a3 + C(20) * b3;
        } else if (q < C(2.5)) {
            f = a3 * a;
            df = C(-4) * a3;
        }
        break;
    }
    case KERN_M6: {
        const C a = C(3) - q, b = C(2) - q, c = C(1) - q;
        const C a4 = (a * a) * (a * a), b4 = (b * b) * (b * b), c4 = (c * c) * (c * c);
        if (q < C(1)) {
            f = a4 * a - C(6) * (b4 * b) + C(15) * (c4 * c);
            df = C(-5) * a4 + C(30) * b4 - C(75) * c4;
        } else if (q < C(2)) {
            f = a4 * a - C(6) * (b4 * b);
            df = C(-5) * a4 + C(30) * b4;
        } else if (q < C(3)) {
            f = a4 * a;
            df = C(-5) * a4;
        }
        break;
    }
    case KERN_C2:
        if (q < C(2)) {
            const C a = C(1) - C(0.5) * q, a3 = a * a * a;
            f = a3 * a * (C(2) * q + C(1));
            df = C(-5) * q * a3;
        }
        break;
    case KERN_C4:
        if (q < C(2)) {
            const C a = C(1) - C(0.5) * q, a2 = a * a, a5 = a2 * a2 * a;
            f = a5 * a * ((C(35) / C(12)) * (q * q) + C(3) * q + C(1));
            df = (C(-14) / C(3)) * q * (C(1) + C(2.5) * q) * a5;
        }
        break;
    case KERN_C6:
        if (q < C(2)) {
            const C a = C(1) - C(0.5) * q, a2 = a * a, a7 = a2 * a2 * a2 * a;
            f = a7 * a * (C(4) * (q * q * q) + C(6.25) * (q * q) + C(4) * q + C(1));
            df = C(-5.5) * q * (C(1) + C(3.5) * q + C(4) * (q * q)) * a7;
        }
        break;
    default:
        break;
    }
}

// f and f' for M5 and M6 in the float pair sums of double inputs (the
// Wendland families have wendland_fdf_f32 below).  The
// innermost spline pieces are expanded (M5 on q < 1/2: 14.375 - 15 q^2 + 6 q^4,
// M6 on q < 1: 66 - 60 q^2 + 30 q^4 - 10 q^5), so f' carries its factor q
// exactly instead of a difference of terms of size ~70.  On the piece that
// reaches the support edge, K - q is taken as num / (h (K h + r)) with
// num = K^2 h^2 - d^2 formed in double: from the float q it would carry a
// few float ulps of absolute error, a relative error that grows without bound
// towards the edge.  A pair beyond this h's support (accepted for the other h
// of a symmetric pair) has num < 0 and gets f = f' = 0.
__device__ __forceinline__ void kern_fdf_f32(int k, float q, float r, float num, float hf, float Kf, float& f,
                                             float& df) {
    // every rounding written out, as in m4_fdf_edge (interp.cuh)
    f = 0.f;
    df = 0.f;
    const float u = fmaxf(__fdividef(num, __fmul_rn(hf, __fmaf_rn(Kf, hf, r))), 0.f);  // K - q
    switch (k) {
    case KERN_M5:
        if (q < 0.5f) {
            const float q2 = __fmul_rn(q, q);
            f = __fmaf_rn(q2, __fmaf_rn(6.f, q2, -15.f), 14.375f);
            df = __fmul_rn(q, __fmaf_rn(24.f, q2, -30.f));
        } else if (q < 1.5f) {
            const float a = __fsub_rn(2.5f, q), b = __fsub_rn(1.5f, q);
            const float a3 = __fmul_rn(__fmul_rn(a, a), a), b3 = __fmul_rn(__fmul_rn(b, b), b);
            f = __fmaf_rn(-5.f, __fmul_rn(b3, b), __fmul_rn(a3, a));
            df = __fmaf_rn(20.f, b3, __fmul_rn(-4.f, a3));
        } else {
            const float u3 = __fmul_rn(__fmul_rn(u, u), u);
            f = __fmul_rn(u3, u);
            df = __fmul_rn(-4.f, u3);
        }
        break;
    case KERN_M6:
        if (q < 1.f) {
            const float q2 = __fmul_rn(q, q);
            f = __fmaf_rn(q2, __fmaf_rn(q2, __fmaf_rn(-10.f, q, 30.f), -60.f), 66.f);
            df = __fmul_rn(q, __fmaf_rn(q2, __fmaf_rn(-50.f, q, 120.f), -120.f));
        } else if (q < 2.f) {
            const float a = __fsub_rn(3.f, q), b = __fsub_rn(2.f, q);
            const float a2 = __fmul_rn(a, a), b2 = __fmul_rn(b, b);
            const float a4 = __fmul_rn(a2, a2), b4 = __fmul_rn(b2, b2);
            f = __fmaf_rn(-6.f, __fmul_rn(b4, b), __fmul_rn(a4, a));
            df = __fmaf_rn(30.f, b4, __fmul_rn(-5.f, a4));
        } else {
            const float u2 = __fmul_rn(u, u);
            const float u4 = __fmul_rn(u2, u2);
            f = __fmul_rn(u4, u);
            df = __fmul_rn(-5.f, u4);
        }
        break;
    default:
        break;
    }
}

// f and f' of a Wendland family (C2, C4, C6) in the float pair sums, from q
// and a = 1 - q/2 (formed more accurately than from q; f32c_wendland_weights),
// in the factored forms.
__device__ __forceinline__ void wendland_fdf_f32(int k, float q, float a, float& f, float& df) {
    // every rounding written out, as in m4_fdf_edge (interp.cuh)
    const float a2 = __fmul_rn(a, a);
    if (k == KERN_C2) {  // (2q + 1) a^4, f' = -5 q a^3
        const float a3 = __fmul_rn(a2, a);
        f = __fmul_rn(__fmul_rn(a3, a), __fmaf_rn(2.f, q, 1.f));
        df = __fmul_rn(__fmul_rn(-5.f, q), a3);
    } else if (k == KERN_C4) {  // (35/12 q^2 + 3 q + 1) a^6, f' = -14/3 q (1 + 5/2 q) a^5
        const float a5 = __fmul_rn(__fmul_rn(a2, a2), a);
        f = __fmul_rn(__fmul_rn(a5, a), __fmaf_rn(__fmaf_rn(35.f / 12.f, q, 3.f), q, 1.f));
        df = __fmul_rn(__fmul_rn(__fmul_rn(-14.f / 3.f, q), __fmaf_rn(2.5f, q, 1.f)), a5);
    } else {  // (4 q^3 + 25/4 q^2 + 4 q + 1) a^8, f' = -11/2 q (1 + 7/2 q + 4 q^2) a^7
        const float a7 = __fmul_rn(__fmul_rn(__fmul_rn(a2, a2), a2), a);
        const float pf = __fmaf_rn(__fmaf_rn(__fmaf_rn(4.f, q, 6.25f), q, 4.f), q, 1.f);
        const float pd = __fmaf_rn(__fmaf_rn(4.f, q, 3.5f), q, 1.f);
        f = __fmul_rn(__fmul_rn(a7, a), pf);
        df = __fmul_rn(__fmul_rn(__fmul_rn(-5.5f, q), pd), a7);
    }
}

// g1 = f'(q)/q and g2 = d g1/dq for k != M4 (the adjoint's gradient and
// Hessian factors): g2 = (f'' - g1)/q on the pieces away from q = 0; the
// pieces that contain q = 0 are written without the division (M5 on q < 1/2
// and M6 on q < 1 are even polynomials there; the Wendland f' = q P(q) a^n
// factor exactly).  iq = 1/q (unused where q = 0 is possible).
__device__ __forceinline__ void kern_g12(int k, double q, double iq, double& g1, double& g2) {
    g1 = 0.0;
    g2 = 0.0;
    double d1 = 0.0, d2 = 0.0;
    switch (k) {
    case KERN_M5: {
        if (q < 0.5) { g1 = -30.0 + 24.0 * q * q; g2 = 48.0 * q; return; }
        const double a = 2.5 - q, b = 1.5 - q;
        if (q < 1.5) {
            d1 = -4.0 * (a * a * a) + 20.0 * (b * b * b);
            d2 = 12.0 * (a * a) - 60.0 * (b * b);
        } else if (q < 2.5) {
            d1 = -4.0 * (a * a * a);
            d2 = 12.0 * (a * a);
        } else {
            return;
        }
        break;
    }
    case KERN_M6: {
        if (q < 1.0) { g1 = -120.0 + q * q * (120.0 - 50.0 * q); g2 = q * (240.0 - 150.0 * q); return; }
        const double a = 3.0 - q, b = 2.0 - q;
        const double a2 = a * a, b2 = b * b;
        if (q < 2.0) {
            d1 = -5.0 * (a2 * a2) + 30.0 * (b2 * b2);
            d2 = 20.0 * (a2 * a) - 120.0 * (b2 * b);
        } else if (q < 3.0) {
            d1 = -5.0 * (a2 * a2);
            d2 = 20.0 * (a2 * a);
        } else {
            return;
        }
        break;
    }
    case KERN_C2: case KERN_C4: case KERN_C6: {
        if (!(q < 2.0)) return;
        const double a = 1.0 - 0.5 * q, a2 = a * a, a3 = a2 * a, a4 = a2 * a2;
        if (k == KERN_C2) {         // f' = -5 q a^3
            g1 = -5.0 * a3;
            g2 = 7.5 * a2;
        } else if (k == KERN_C4) {  // f' = -14/3 q (1 + 5q/2) a^5
            g1 = (-14.0 / 3.0) * (1.0 + 2.5 * q) * (a4 * a);
            g2 = 35.0 * q * a4;
        } else {                    // f' = -11/2 q (1 + 7q/2 + 4q^2) a^7
            g1 = -5.5 * (1.0 + 3.5 * q + 4.0 * q * q) * (a4 * a3);
            g2 = 33.0 * q * (1.0 + 3.0 * q) * (a3 * a3);
        }
        return;
    }
    default:
        return;
    }
    g1 = d1 * iq;
    g2 = (d2 - g1) * iq;
}

}  // namespace psb
