// euler_math.cuh -- pointwise math of the compressible Euler RHS (device).
//
// WENO5-JS reconstruction (Jiang & Shu, J. Comput. Phys. 126, 1996) of the
// primitive variables (rho, u, v, w, p) and the Rusanov (local Lax-Friedrichs)
// flux, gamma-law gas.  The reference library only promises these operators
// (README.rst:28-31); this is an implementation of the published method.
//
// Every operation is written out explicitly: contractions are only the fma()
// calls below (the file is compiled with --fmad=false), so the CPU oracle can
// repeat the computation bit for bit.
//
// Nonlinear weights: with s_k = eps + beta_k and t_k = s_k^2 the JS weights
// alpha_k = d_k / t_k normalise to omega_k = d_k*prod_{j!=k} t_j / D with
// D = sum_k d_k*prod_{j!=k} t_j, so one division per reconstruction suffices:
//   v = (w0*n0 + w1*n1 + w2*n2) / (6*D),  w0 = d0*t1*t2, w1 = d1*t0*t2, w2 = d2*t0*t1,
// where n_k = 6*q_k are the candidate stencils' numerators.
#pragma once

#include <cuda_runtime.h>

namespace cn {
namespace euler {

template <typename T> struct K {
    static constexpr T c1312 = T(13.0 / 12.0);
    static constexpr T quarter = T(0.25);
    static constexpr T eps = T(1e-6);
    static constexpr T d0 = T(0.1);
    static constexpr T d1 = T(0.6);
    static constexpr T d2 = T(0.3);
    static constexpr T half = T(0.5);
    static constexpr T six = T(6);
};

__device__ __forceinline__ double dfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float dfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ float dsqrt(float a) { return sqrtf(a); }
__device__ __forceinline__ double dabs(double a) { return fabs(a); }
__device__ __forceinline__ float dabs(float a) { return fabsf(a); }
__device__ __forceinline__ double dmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float dmax(float a, float b) { return fmaxf(a, b); }

// Left-biased WENO5-JS reconstruction at i+1/2 from v0..v4 = v[i-2..i+2],
// returned as numerator and denominator: value = num / den.
template <typename T>
__device__ __forceinline__ void weno5_nd(T v0, T v1, T v2, T v3, T v4, T &num, T &den)
{
    using C = K<T>;
    // smoothness indicators
    const T a0 = dfma(T(-2), v1, v0) + v2;            // v0 - 2v1 + v2
    const T b0 = dfma(T(3), v2, dfma(T(-4), v1, v0)); // v0 - 4v1 + 3v2
    const T a1 = dfma(T(-2), v2, v1) + v3;            // v1 - 2v2 + v3
    const T b1 = v1 - v3;
    const T a2 = dfma(T(-2), v3, v2) + v4;            // v2 - 2v3 + v4
    const T b2 = dfma(T(3), v2, dfma(T(-4), v3, v4)); // 3v2 - 4v3 + v4
    const T s0 = C::eps + dfma(C::c1312 * a0, a0, C::quarter * (b0 * b0));
    const T s1 = C::eps + dfma(C::c1312 * a1, a1, C::quarter * (b1 * b1));
    const T s2 = C::eps + dfma(C::c1312 * a2, a2, C::quarter * (b2 * b2));
    const T t0 = s0 * s0, t1 = s1 * s1, t2 = s2 * s2;
    const T w0 = C::d0 * (t1 * t2);
    const T w1 = C::d1 * (t0 * t2);
    const T w2 = C::d2 * (t0 * t1);
    // candidate numerators 6*q_k
    const T n0 = dfma(T(2), v0, dfma(T(-7), v1, T(11) * v2)); // 2v0 - 7v1 + 11v2
    const T n1 = dfma(T(5), v2, dfma(T(2), v3, -v1));         // -v1 + 5v2 + 2v3
    const T n2 = dfma(T(2), v2, dfma(T(5), v3, -v4));         // 2v2 + 5v3 - v4
    num = dfma(w0, n0, dfma(w1, n1, w2 * n2));
    den = C::six * ((w0 + w1) + w2);
}

// Left and right states at the face between v2 and v3 from v0..v5 =
// v[i-2..i+3].  FP64 shares one division between the two:
//   inv = 1/(denL*denR), vL = (numL*denR)*inv, vR = (numR*denL)*inv
// (den >= 6e-25 since eps = 1e-6, so the product cannot underflow in FP64);
// FP32 divides twice, as the product could leave the FP32 range.
__device__ __forceinline__ void weno5_pair(double v0, double v1, double v2, double v3, double v4, double v5,
                                           double &vl, double &vr)
{
    double nl, dl, nr, dr;
    weno5_nd<double>(v0, v1, v2, v3, v4, nl, dl);
    weno5_nd<double>(v5, v4, v3, v2, v1, nr, dr);
    const double inv = 1.0 / (dl * dr);
    vl = (nl * dr) * inv;
    vr = (nr * dl) * inv;
}

__device__ __forceinline__ void weno5_pair(float v0, float v1, float v2, float v3, float v4, float v5, float &vl,
                                           float &vr)
{
    float nl, dl, nr, dr;
    weno5_nd<float>(v0, v1, v2, v3, v4, nl, dl);
    weno5_nd<float>(v5, v4, v3, v2, v1, nr, dr);
    vl = nl / dl;
    vr = nr / dr;
}

// Rusanov flux through a face with normal direction `d` (0,1,2) from the
// reconstructed primitive states WL, WR = (rho, u, v, w, p).
template <typename T>
__device__ __forceinline__ void rusanov(const T (&WL)[5], const T (&WR)[5], int d, T gamma,
                                        T igm1, T (&F)[5])
{
    using C = K<T>;
    const T rl = WL[0], rr = WR[0];
    // normal velocities (selects, not an index: d is a runtime value)
    const T unl = d == 0 ? WL[1] : (d == 1 ? WL[2] : WL[3]);
    const T unr = d == 0 ? WR[1] : (d == 1 ? WR[2] : WR[3]);
    const T pl = WL[4], pr = WR[4];
    // conservative states
    const T mul0 = rl * WL[1], mul1 = rl * WL[2], mul2 = rl * WL[3];
    const T mur0 = rr * WR[1], mur1 = rr * WR[2], mur2 = rr * WR[3];
    const T kel = dfma(WL[1], WL[1], dfma(WL[2], WL[2], WL[3] * WL[3]));
    const T ker = dfma(WR[1], WR[1], dfma(WR[2], WR[2], WR[3] * WR[3]));
    const T El = dfma(C::half * rl, kel, pl * igm1);
    const T Er = dfma(C::half * rr, ker, pr * igm1);
    // wave speeds
    const T cl = dsqrt((gamma * pl) / rl);
    const T cr = dsqrt((gamma * pr) / rr);
    const T a = dmax(dabs(unl) + cl, dabs(unr) + cr);
    // physical fluxes
    const T fl0 = rl * unl, fr0 = rr * unr;
    T fl1 = mul0 * unl, fr1 = mur0 * unr;
    T fl2 = mul1 * unl, fr2 = mur1 * unr;
    T fl3 = mul2 * unl, fr3 = mur2 * unr;
    if (d == 0) {
        fl1 = fl1 + pl;
        fr1 = fr1 + pr;
    } else if (d == 1) {
        fl2 = fl2 + pl;
        fr2 = fr2 + pr;
    } else {
        fl3 = fl3 + pl;
        fr3 = fr3 + pr;
    }
    const T fl4 = (El + pl) * unl, fr4 = (Er + pr) * unr;
    F[0] = C::half * dfma(-a, rr - rl, fl0 + fr0);
    F[1] = C::half * dfma(-a, mur0 - mul0, fl1 + fr1);
    F[2] = C::half * dfma(-a, mur1 - mul1, fl2 + fr2);
    F[3] = C::half * dfma(-a, mur2 - mul2, fl3 + fr3);
    F[4] = C::half * dfma(-a, Er - El, fl4 + fr4);
}

// Conservative -> primitive (rho, u, v, w, p).
template <typename T>
__device__ __forceinline__ void to_primitive(T r, T m0, T m1, T m2, T E, T gm1, T (&W)[5])
{
    const T inv = T(1) / r;
    const T u = m0 * inv, v = m1 * inv, w = m2 * inv;
    const T ke = K<T>::half * dfma(m0, u, dfma(m1, v, m2 * w));
    W[0] = r;
    W[1] = u;
    W[2] = v;
    W[3] = w;
    W[4] = gm1 * (E - ke);
}

} // namespace euler
} // namespace cn
