// euler_math.cuh -- pointwise math of the compressible Euler RHS (device).
//
// WENO5-JS reconstruction (Jiang & Shu, J. Comput. Phys. 126, 1996) of the
// primitive variables (rho, u, v, w, p) and the Rusanov (local Lax-Friedrichs)
// flux, gamma-law gas.  The reference library only promises these operators
// (README.rst:28-31); this is an implementation of the published method.
//
// Floating-point contract.  The file is compiled with FMA contraction on
// (nvcc's default --fmad=true): beyond the fma() calls written out below, the
// compiler fuses any multiply feeding an add.  Reciprocals and square roots
// are not IEEE-rounded: FP64 uses the hardware approximations refined by one
// third-order step (rcp_pos / rsqrt_pos below, within a few ulp), FP32 calls
// CUDA's fast intrinsics (__fdividef, rsqrtf: about 2 ulp).  The CPU oracle
// computes the same formulas with IEEE division and square root and no
// contraction; FP64 results agree with it within 1e-13 relative, FP32 results
// are judged by their error against FP64.
//
// Nonlinear weights: with s_k = eps + beta_k and t_k = s_k^2 the JS weights
// alpha_k = d_k / t_k normalise to omega_k = d_k*prod_{j!=k} t_j / D with
// D = sum_k d_k*prod_{j!=k} t_j, so one division per reconstruction suffices:
//   v = (w0*n0 + w1*n1 + w2*n2) / (6*D),  w0 = d0*t1*t2, w1 = d1*t0*t2, w2 = d2*t0*t1,
// where n_k = 6*q_k are the candidate stencils' numerators, written as
// 6*u_j plus differences so that v = u_j + (sum w_k e_k) / (6*D).  The indicators
// beta_k and the products t_i t_j belong to the cell, not to the face: a
// cell's left-biased state (at its upper face) and right-biased state (at its
// lower face) share them.
//
// Range.  A jump J in the data gives s ~ 3 J^2 and t_i t_j ~ 20 J^8, which
// leaves the FP32 range above J ~ 4e4 (a pressure jump of one bar in SI
// units).  So in FP32 t_k is formed from s_k * 2^-e, with e the mean of the
// binary exponents of the largest and the middle s_k (rounded down).  Scaling
// by a power of two is exact and cancels in every ratio below.  With it the
// dominant product t_max t_mid lies in [1, 64) and every FP32 denominator in
// [0.6, 384]; the only products that can underflow are those of negligible
// weights.  FP64 needs no scaling: its denominators lie in [6e-25, ~70 J^8].
// Since the factor is an exact power of two, the scaled and unscaled forms
// give the same values wherever the unscaled one stays in range; a tile whose
// primitives are all within kUnscaledMax in magnitude (then t_i t_j < 1.3e30
// and the numerators < 2e34, eps keeps them above 1e-24) skips the scaling
// (`scaled` false).
#pragma once

#include <cuda_runtime.h>

namespace cn {
namespace euler {

// largest primitive magnitude of a tile for the unscaled FP32 WENO5 weights
constexpr float kUnscaledMax = 1000.0f;

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

// 1/x for a positive normal x (denominators of the face states, densities).
// FP64: the PTX approximation rcp.approx.ftz.f64 refined by one step of the
// third-order iteration that truncates the series 1/x = r / (1 - e) =
// r (1 + e + e^2 + ...), e = 1 - x r:  r' = r + r (e + e^2), relative error
// e^3 plus rounding.  FP32: CUDA's __fdividef (valid for x < 2^126).
__device__ __forceinline__ double rcp_pos(double x)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    const double e = fma(-x, r, 1.0);
    return fma(r, fma(e, e, e), r);
}
__device__ __forceinline__ float rcp_pos(float x) { return __fdividef(1.0f, x); }

// 1/sqrt(x) for a positive normal x.  FP64: rsqrt.approx.ftz.f64 refined by one
// step of the third-order iteration from the series (1 - h)^(-1/2) =
// 1 + h/2 + 3h^2/8 + ..., h = 1 - x y^2:  y' = y + y h (1/2 + 3/8 h).
// FP32: CUDA's rsqrtf.
__device__ __forceinline__ double rsqrt_pos(double x)
{
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double h = fma(-x * y, y, 1.0);
    return fma(y * h, fma(0.375, h, 0.5), y);
}
__device__ __forceinline__ float rsqrt_pos(float x) { return rsqrtf(x); }

// The FP32 factor 2^-e of the range note above for s0, s1, s2 >= eps: e =
// floor((E_max + E_mid) / 2) - 127 from the biased exponents of the largest
// and the middle of the three (E_max + E_mid = E0 + E1 + E2 - E_min).  The
// exponents come from the bit patterns (integer instructions only).  A NaN
// or infinite s gives NaN states, and so do two sums above 2^127 (~1.7e38,
// jumps ~1e19: the factor leaves the normal range there).
__device__ __forceinline__ float weno5_scale(float s0, float s1, float s2)
{
    const int e0 = __float_as_int(s0) >> 23, e1 = __float_as_int(s1) >> 23, e2 = __float_as_int(s2) >> 23;
    const int emin = min(min(e0, e1), e2);
    return __int_as_float(int(unsigned(254 - ((e0 + e1 + e2 - emin) >> 1)) << 23));
}

// Differences of the 5-point stencil u0..u4 = v[j-2..j+2] of cell j: the
// smoothness indicators and both reconstructions are written in them, and a
// state is the cell value u2 plus a correction, so that smooth data loses no
// digits to the cancellation inside the candidate stencils.
template <typename T> struct Diff5 {
    T d01, d12, d23, d34;
};
template <typename T> __device__ __forceinline__ Diff5<T> weno5_diff(T u0, T u1, T u2, T u3, T u4)
{
    return {u1 - u0, u2 - u1, u3 - u2, u4 - u3};
}

// Smoothness of cell j: with s_k = eps + beta_k and t_k = s_k^2 for the
// stencils S0 = {j-2, j-1, j}, S1 = {j-1, j, j+1}, S2 = {j, j+1, j+2}, the
// products p12 = t1 t2, p02 = t0 t2, p01 = t0 t1.  beta_k = 13/12 a_k^2 +
// 1/4 b_k^2 with a0 = d12 - d01, a1 = d23 - d12, a2 = d34 - d23 and
// b0/2 = a0/2 + d12, b1/2 = (d12 + d23)/2 (up to sign), b2/2 = a2/2 - d23.
// They serve both states of the cell (left-biased at j+1/2, right-biased at
// j-1/2), so a cell's indicators are computed once for its two faces.
template <typename T>
__device__ __forceinline__ void weno5_beta(const Diff5<T> &d, T &p12, T &p02, T &p01, bool scaled = true)
{
    using C = K<T>;
    const T a0 = d.d12 - d.d01, a1 = d.d23 - d.d12, a2 = d.d34 - d.d23;
    const T h0 = dfma(C::half, a0, d.d12);
    const T h1 = C::half * (d.d12 + d.d23);
    const T h2 = dfma(C::half, a2, -d.d23);
    const T s0 = dfma(C::c1312 * a0, a0, dfma(h0, h0, C::eps));
    const T s1 = dfma(C::c1312 * a1, a1, dfma(h1, h1, C::eps));
    const T s2 = dfma(C::c1312 * a2, a2, dfma(h2, h2, C::eps));
    T q0 = s0, q1 = s1, q2 = s2;
    if constexpr (sizeof(T) == 4) { // FP32: exact power-of-two rescaling
        if (scaled) {
            const T sc = weno5_scale(s0, s1, s2);
            q0 = s0 * sc;
            q1 = s1 * sc;
            q2 = s2 * sc;
        }
    }
    const T t0 = q0 * q0, t1 = q1 * q1, t2 = q2 * q2;
    p12 = t1 * t2;
    p02 = t0 * t2;
    p01 = t0 * t1;
}

// Left-biased state of cell j at j+1/2 (linear weights 1/10, 6/10, 3/10 on
// S0, S1, S2): value = u2 + num / den.  The candidates' numerators 6 q_k are
// 6 u2 + e_k with e0 = 5 d12 - 2 d01, e1 = d12 + 2 d23, e2 = 4 d23 - d34.
// w1 = 0.6 p02 is the middle weight of both states of the cell.
template <typename T>
__device__ __forceinline__ void weno5_left(const Diff5<T> &d, T p12, T w1, T p01, T &num, T &den)
{
    using C = K<T>;
    const T w0 = C::d0 * p12, w2 = C::d2 * p01;
    const T e0 = dfma(T(-2), d.d01, T(5) * d.d12);
    const T e1 = dfma(T(2), d.d23, d.d12);
    const T e2 = dfma(T(4), d.d23, -d.d34);
    num = dfma(w0, e0, dfma(w1, e1, w2 * e2));
    den = C::six * ((w0 + w1) + w2);
}

// Right-biased state of cell j at j-1/2 (linear weights 3/10, 6/10, 1/10):
// value = u2 + num / den with candidates 6 u2 + f_k, f0 = d01 - 4 d12,
// f1 = -2 d12 - d23, f2 = 2 d34 - 5 d23.
template <typename T>
__device__ __forceinline__ void weno5_right(const Diff5<T> &d, T p12, T w1, T p01, T &num, T &den)
{
    using C = K<T>;
    const T r0 = C::d2 * p12, r2 = C::d0 * p01;
    const T f0 = dfma(T(-4), d.d12, d.d01);
    const T f1 = dfma(T(-2), d.d12, -d.d23);
    const T f2 = dfma(T(2), d.d34, T(-5) * d.d23);
    num = dfma(r0, f0, dfma(w1, f1, r2 * f2));
    den = C::six * ((r0 + w1) + r2);
}

// A reconstructed state u2 + num / den (den > 0: a sum of positive weights).
template <typename T> __device__ __forceinline__ T weno5_value(T u2, T num, T den)
{
    return dfma(num, rcp_pos(den), u2);
}

// ---------------------------------------------------------------------------
// FP32, two variables per instruction.  Blackwell executes FP32 add, multiply
// and fused multiply-add on a pair of values per thread (PTX add/mul/fma
// .rn.f32x2, CUDA's __fadd2_rn / __fmul2_rn / __ffma2_rn); the WENO5 formulas
// above are evaluated for two primitive variables at once, lane x holding
// one variable and lane y the other.  Same operations as the scalar forms,
// one packed instruction per pair.  (The Rusanov flux stays scalar: packing
// its left and right states measured slower, 11.9 against 12.5
// Gcell-updates/s at 1024^3, from the moves that regroup the lanes.)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.0f), a); }

struct Diff5x2 {
    float2 d01, d12, d23, d34;
};
__device__ __forceinline__ Diff5x2 weno5_diff2(float2 u0, float2 u1, float2 u2, float2 u3, float2 u4)
{
    return {sub2(u1, u0), sub2(u2, u1), sub2(u3, u2), sub2(u4, u3)};
}

// weno5_scale for both lanes of a pair at once, from the top 7 bits of each
// biased exponent (byte 3 of a positive float, E >> 1) packed as two 16-bit
// halves: m = (E_max >> 1) + (E_mid >> 1) differs from (E_max + E_mid) / 2
// by at most 1, so the dominant product t_max t_mid lies in [1/4, 256) and
// the range note's bounds widen by a factor 4 at most.  The halves never
// carry into each other (each stays below 2^9).
__device__ __forceinline__ float2 weno5_scale2(float2 s0, float2 s1, float2 s2)
{
    // bytes [x.b3, 0, y.b3, 0]: selector nibbles 3, 7 pick byte 3 of each
    // word, 0xB / 0xF replicate its sign bit (0 for s > 0)
    const unsigned e0 = __byte_perm(__float_as_uint(s0.x), __float_as_uint(s0.y), 0xF7B3);
    const unsigned e1 = __byte_perm(__float_as_uint(s1.x), __float_as_uint(s1.y), 0xF7B3);
    const unsigned e2 = __byte_perm(__float_as_uint(s2.x), __float_as_uint(s2.y), 0xF7B3);
    const unsigned mn = __vmins2(__vmins2(e0, e1), e2);
    const unsigned b = 0x00FE00FEu - (e0 + e1 + e2 - mn); // biased exponents of the factors
    return make_float2(__uint_as_float(b << 23), __uint_as_float((b >> 16) << 23));
}

// weno5_beta for a pair (rescaling factors from weno5_scale2).  h2 enters
// squared only, so its sign is dropped: h2' = d23 - a2/2.
__device__ __forceinline__ void weno5_beta2(const Diff5x2 &d, float2 &p12, float2 &p02, float2 &p01,
                                            bool scaled = true)
{
    using C = K<float>;
    const float2 a0 = sub2(d.d12, d.d01), a1 = sub2(d.d23, d.d12), a2 = sub2(d.d34, d.d23);
    const float2 h0 = fma2(f2(C::half), a0, d.d12);
    const float2 h1 = mul2(f2(C::half), add2(d.d12, d.d23));
    const float2 h2 = fma2(f2(-C::half), a2, d.d23);
    const float2 s0 = fma2(mul2(f2(C::c1312), a0), a0, fma2(h0, h0, f2(C::eps)));
    const float2 s1 = fma2(mul2(f2(C::c1312), a1), a1, fma2(h1, h1, f2(C::eps)));
    const float2 s2 = fma2(mul2(f2(C::c1312), a2), a2, fma2(h2, h2, f2(C::eps)));
    float2 q0 = s0, q1 = s1, q2 = s2;
    if (scaled) {
        const float2 sc = weno5_scale2(s0, s1, s2);
        q0 = mul2(s0, sc);
        q1 = mul2(s1, sc);
        q2 = mul2(s2, sc);
    }
    const float2 t0 = mul2(q0, q0), t1 = mul2(q1, q1), t2 = mul2(q2, q2);
    p12 = mul2(t1, t2);
    p02 = mul2(t0, t2);
    p01 = mul2(t0, t1);
}

__device__ __forceinline__ void weno5_left2(const Diff5x2 &d, float2 p12, float2 w1, float2 p01, float2 &num,
                                            float2 &den)
{
    using C = K<float>;
    const float2 w0 = mul2(f2(C::d0), p12), w2 = mul2(f2(C::d2), p01);
    const float2 e0 = fma2(f2(-2.0f), d.d01, mul2(f2(5.0f), d.d12));
    const float2 e1 = fma2(f2(2.0f), d.d23, d.d12);
    const float2 e2 = sub2(mul2(f2(4.0f), d.d23), d.d34);
    num = fma2(w0, e0, fma2(w1, e1, mul2(w2, e2)));
    den = mul2(f2(C::six), add2(add2(w0, w1), w2));
}

__device__ __forceinline__ void weno5_right2(const Diff5x2 &d, float2 p12, float2 w1, float2 p01, float2 &num,
                                             float2 &den)
{
    using C = K<float>;
    const float2 r0 = mul2(f2(C::d2), p12), r2 = mul2(f2(C::d0), p01);
    const float2 f0 = fma2(f2(-4.0f), d.d12, d.d01);
    const float2 f1 = sub2(mul2(f2(-2.0f), d.d12), d.d23);
    const float2 g2 = fma2(f2(2.0f), d.d34, mul2(f2(-5.0f), d.d23));
    num = fma2(r0, f0, fma2(w1, f1, mul2(r2, g2)));
    den = mul2(f2(C::six), add2(add2(r0, w1), r2));
}

__device__ __forceinline__ float2 weno5_value2(float2 u2, float2 num, float2 den)
{
    return fma2(num, make_float2(rcp_pos(den.x), rcp_pos(den.y)), u2);
}

// Twice the Rusanov flux through a face with normal direction `d` (0,1,2)
// from the reconstructed primitive states WL, WR = (rho, u, v, w, p):
// F = (f(UL) + f(UR)) - a (UR - UL), a = max(|u_n| + c) of both sides.  The
// factor 1/2 of the flux is exact and is taken with 1/h by the flux
// differences.
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
    // sound speeds c = sqrt(gamma p / rho) = (gamma p) / sqrt(gamma p rho)
    const T gpl = gamma * pl, gpr = gamma * pr;
    const T cl = gpl * rsqrt_pos(gpl * rl);
    const T cr = gpr * rsqrt_pos(gpr * rr);
    const T a = dmax(dabs(unl) + cl, dabs(unr) + cr);
    // mass
    const T fl0 = rl * unl, fr0 = rr * unr;
    F[0] = dfma(-a, rr - rl, fl0 + fr0);
    // momentum: flux = mass flux * velocity (+ p along the normal)
#pragma unroll
    for (int k = 1; k <= 3; ++k) {
        const T ml = rl * WL[k], mr = rr * WR[k];
        T fl = fl0 * WL[k], fr = fr0 * WR[k];
        if (k - 1 == d) {
            fl = fl + pl;
            fr = fr + pr;
        }
        F[k] = dfma(-a, mr - ml, fl + fr);
    }
    // energy
    const T kel = dfma(WL[1], WL[1], dfma(WL[2], WL[2], WL[3] * WL[3]));
    const T ker = dfma(WR[1], WR[1], dfma(WR[2], WR[2], WR[3] * WR[3]));
    const T El = dfma(C::half * rl, kel, pl * igm1);
    const T Er = dfma(C::half * rr, ker, pr * igm1);
    const T fl4 = (El + pl) * unl, fr4 = (Er + pr) * unr;
    F[4] = dfma(-a, Er - El, fl4 + fr4);
}

// Conservative -> primitive (rho, u, v, w, p).
template <typename T>
__device__ __forceinline__ void to_primitive(T r, T m0, T m1, T m2, T E, T gm1, T (&W)[5])
{
    const T inv = rcp_pos(r);
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
