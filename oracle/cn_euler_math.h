/*
 * cn_euler_math.h -- pointwise Euler math of the CPU oracle (WENO5-JS
 * reconstruction, Rusanov flux, conservative -> primitive).
 *
 * TEST INFRASTRUCTURE ONLY.  Shared by cn_euler.c (plain-C oracle) and
 * ref_shim.cpp (the same math on labs filled by the reference's FieldLab).
 * See cn_euler.c for the published methods followed.  Must be compiled
 * without floating-point contraction (-ffp-contract=off).
 */
#ifndef CN_EULER_MATH_H
#define CN_EULER_MATH_H

#include <math.h>
#include <stdint.h>
#include <string.h>

/* FP32 power-of-two factor 2^-e for the smoothness sums s0, s1, s2 (all
 * >= eps): e = floor((E_max + E_mid) / 2) - 127 from the biased exponents of
 * the largest and the middle sum (E_max + E_mid = E0 + E1 + E2 - E_min).
 * t_k = (s_k 2^-e)^2: scaling by a power of two is exact and cancels in the
 * weights, and keeps the dominant product t_max t_mid in [1, 64), so the
 * products of a jump J (~20 J^8 unscaled) stay in the FP32 range.  The
 * factor's bit pattern is formed as on the device (32-bit wrap-around); FP64
 * is not rescaled (factor 1). */
static inline int cn_imin_(int a, int b) { return a < b ? a : b; }

static inline float weno5_scale_f32(float s0, float s1, float s2)
{
    int32_t b0, b1, b2;
    memcpy(&b0, &s0, 4);
    memcpy(&b1, &s1, 4);
    memcpy(&b2, &s2, 4);
    const int e0 = b0 >> 23, e1 = b1 >> 23, e2 = b2 >> 23;
    const int emin = cn_imin_(cn_imin_(e0, e1), e2);
    const uint32_t bits = (uint32_t)(254 - ((e0 + e1 + e2 - emin) >> 1)) << 23;
    float r;
    memcpy(&r, &bits, 4);
    return r;
}

static inline double weno5_scale_f64(double s0, double s1, double s2)
{
    (void)s0;
    (void)s1;
    (void)s2;
    return 1.0;
}

#define DEFINE_EULER_MATH(SUF, T, FMA, SQRT, FABS, FMAX)                        \
    /* smoothness of cell j from the differences of u0..u4 = v[j-2..j+2]     \
     * (d01 = u1 - u0, ...): the products p12 = t1 t2, p02 = t0 t2,          \
     * p01 = t0 t1 of t_k = (eps + beta_k)^2 for the stencils S0 = {j-2..j}, \
     * S1 = {j-1..j+1}, S2 = {j..j+2}, beta_k = 13/12 a_k^2 + 1/4 b_k^2 with \
     * a0 = d12 - d01, a1 = d23 - d12, a2 = d34 - d23, b0/2 = a0/2 + d12,     \
     * b1/2 = (d12 + d23)/2 (up to sign), b2/2 = a2/2 - d23; shared by the    \
     * cell's left-biased (j+1/2) and right-biased (j-1/2) states */          \
    static inline void weno5_beta_##SUF(T d01, T d12, T d23, T d34, T *p12, T *p02, T *p01) \
    {                                                                          \
        const T c1312 = (T)(13.0 / 12.0), half = (T)0.5, eps = (T)1e-6;        \
        const T a0 = d12 - d01, a1 = d23 - d12, a2 = d34 - d23;                \
        const T h0 = FMA(half, a0, d12);                                       \
        const T h1 = half * (d12 + d23);                                       \
        const T h2 = FMA(half, a2, -d23);                                      \
        const T s0 = FMA(c1312 * a0, a0, FMA(h0, h0, eps));                    \
        const T s1 = FMA(c1312 * a1, a1, FMA(h1, h1, eps));                    \
        const T s2 = FMA(c1312 * a2, a2, FMA(h2, h2, eps));                    \
        const T sc = weno5_scale_##SUF(s0, s1, s2);                            \
        const T q0 = s0 * sc, q1 = s1 * sc, q2 = s2 * sc;                      \
        const T t0 = q0 * q0, t1 = q1 * q1, t2 = q2 * q2;                      \
        *p12 = t1 * t2;                                                        \
        *p02 = t0 * t2;                                                        \
        *p01 = t0 * t1;                                                        \
    }                                                                          \
                                                                               \
    /* left-biased state of cell j at j+1/2: linear weights 1/10, 6/10, 3/10  \
     * on S0, S1, S2; value = u2 + num / den, the candidates' numerators      \
     * 6 q_k = 6 u2 + e_k, e0 = 5 d12 - 2 d01, e1 = d12 + 2 d23,             \
     * e2 = 4 d23 - d34 */                                                     \
    static inline void weno5_left_##SUF(T u0, T u1, T u2, T u3, T u4, T *num, T *den) \
    {                                                                          \
        const T d01 = u1 - u0, d12 = u2 - u1, d23 = u3 - u2, d34 = u4 - u3;    \
        T p12, p02, p01;                                                       \
        weno5_beta_##SUF(d01, d12, d23, d34, &p12, &p02, &p01);                \
        const T w1 = (T)0.6 * p02;                                             \
        const T w0 = (T)0.1 * p12, w2 = (T)0.3 * p01;                          \
        const T e0 = FMA((T)-2, d01, (T)5 * d12);                              \
        const T e1 = FMA((T)2, d23, d12);                                      \
        const T e2 = FMA((T)4, d23, -d34);                                     \
        *num = FMA(w0, e0, FMA(w1, e1, w2 * e2));                              \
        *den = (T)6 * ((w0 + w1) + w2);                                        \
    }                                                                          \
                                                                               \
    /* right-biased state of cell j at j-1/2: linear weights 3/10, 6/10, 1/10 \
     * on S0, S1, S2; candidates 6 u2 + f_k, f0 = d01 - 4 d12,               \
     * f1 = -2 d12 - d23, f2 = 2 d34 - 5 d23 */                                \
    static inline void weno5_right_##SUF(T u0, T u1, T u2, T u3, T u4, T *num, T *den) \
    {                                                                          \
        const T d01 = u1 - u0, d12 = u2 - u1, d23 = u3 - u2, d34 = u4 - u3;    \
        T p12, p02, p01;                                                       \
        weno5_beta_##SUF(d01, d12, d23, d34, &p12, &p02, &p01);                \
        const T w1 = (T)0.6 * p02;                                             \
        const T r0 = (T)0.3 * p12, r2 = (T)0.1 * p01;                          \
        const T f0 = FMA((T)-4, d12, d01);                                     \
        const T f1 = FMA((T)-2, d12, -d23);                                    \
        const T f2 = FMA((T)2, d34, (T)-5 * d23);                              \
        *num = FMA(r0, f0, FMA(w1, f1, r2 * f2));                              \
        *den = (T)6 * ((r0 + w1) + r2);                                        \
    }                                                                          \
                                                                               \
    /* the two reconstructions at the face between v2 and v3 (v0..v5 =      \
     * v[i-2..i+3]): cell v2's left-biased and cell v3's right-biased state   \
     * as base value, numerator and denominator (state = b + n / d) */         \
    static inline void weno5_nd_face_##SUF(T v0, T v1, T v2, T v3, T v4, T v5, \
                                           T *bl, T *nl, T *dl, T *br, T *nr, T *dr) \
    {                                                                          \
        weno5_left_##SUF(v0, v1, v2, v3, v4, nl, dl);                          \
        weno5_right_##SUF(v1, v2, v3, v4, v5, nr, dr);                         \
        *bl = v2;                                                              \
        *br = v3;                                                              \
    }                                                                          \
                                                                               \
    /* face states of the 5 variables from their base values, numerators and \
     * denominators (each denominator in [0.6, 384] with the scaled          \
     * weights): variables (0,1) and (2,3) share one division for their four \
     * states, variable 4 takes one for its two */                            \
    static inline void face_states5_##SUF(const T *bl, const T *nl, const T *dl, \
                                          const T *br, const T *nr, const T *dr, \
                                          T *WL, T *WR)                        \
    {                                                                          \
        for (int c = 0; c < 4; c += 2) {                                       \
            const T Da = dl[c] * dr[c], Db = dl[c + 1] * dr[c + 1];            \
            const T inv = (T)1 / (Da * Db);                                    \
            const T qa = Db * inv, qb = Da * inv;                              \
            WL[c] = FMA(nl[c] * dr[c], qa, bl[c]);                             \
            WR[c] = FMA(nr[c] * dl[c], qa, br[c]);                             \
            WL[c + 1] = FMA(nl[c + 1] * dr[c + 1], qb, bl[c + 1]);             \
            WR[c + 1] = FMA(nr[c + 1] * dl[c + 1], qb, br[c + 1]);             \
        }                                                                      \
        const T inv = (T)1 / (dl[4] * dr[4]);                                  \
        WL[4] = FMA(nl[4] * dr[4], inv, bl[4]);                                \
        WR[4] = FMA(nr[4] * dl[4], inv, br[4]);                                \
    }                                                                          \
                                                                               \
    /* twice the Rusanov flux: (f(UL) + f(UR)) - a (UR - UL) with            \
     * a = max(|u_n| + c) of both sides; the factor 1/2 is taken with 1/h    \
     * by the flux differences (exact) */                                     \
    static inline void rusanov_##SUF(const T *WL, const T *WR, int d, T gamma,        \
                              T igm1, T *F)                                    \
    {                                                                          \
        const T half = (T)0.5;                                                 \
        const T rl = WL[0], rr = WR[0];                                        \
        const T unl = WL[1 + d], unr = WR[1 + d];                              \
        const T pl = WL[4], pr = WR[4];                                        \
        /* one division for both sound speeds */                               \
        const T irr = (T)1 / (rl * rr);                                        \
        const T cl = SQRT(((gamma * pl) * rr) * irr);                          \
        const T cr = SQRT(((gamma * pr) * rl) * irr);                          \
        const T a = FMAX(FABS(unl) + cl, FABS(unr) + cr);                      \
        const T fl0 = rl * unl, fr0 = rr * unr;                                \
        F[0] = FMA(-a, rr - rl, fl0 + fr0);                                    \
        for (int k = 1; k <= 3; ++k) {                                         \
            const T ml = rl * WL[k], mr = rr * WR[k];                          \
            T fl = fl0 * WL[k], fr = fr0 * WR[k];                              \
            if (k - 1 == d) {                                                  \
                fl = fl + pl;                                                  \
                fr = fr + pr;                                                  \
            }                                                                  \
            F[k] = FMA(-a, mr - ml, fl + fr);                                  \
        }                                                                      \
        const T kel = FMA(WL[1], WL[1], FMA(WL[2], WL[2], WL[3] * WL[3]));     \
        const T ker = FMA(WR[1], WR[1], FMA(WR[2], WR[2], WR[3] * WR[3]));     \
        const T El = FMA(half * rl, kel, pl * igm1);                           \
        const T Er = FMA(half * rr, ker, pr * igm1);                           \
        const T fl4 = (El + pl) * unl, fr4 = (Er + pr) * unr;                  \
        F[4] = FMA(-a, Er - El, fl4 + fr4);                                    \
    }                                                                          \
                                                                               \
    static inline void prim_##SUF(T r, T m0, T m1, T m2, T E, T gm1, T *W)            \
    {                                                                          \
        const T inv = (T)1 / r;                                                \
        const T u = m0 * inv, v = m1 * inv, w = m2 * inv;                      \
        const T ke = (T)0.5 * FMA(m0, u, FMA(m1, v, m2 * w));                  \
        W[0] = r;                                                              \
        W[1] = u;                                                              \
        W[2] = v;                                                              \
        W[3] = w;                                                              \
        W[4] = gm1 * (E - ke);                                                 \
    }                                                                          \

DEFINE_EULER_MATH(f64, double, fma, sqrt, fabs, fmax)
DEFINE_EULER_MATH(f32, float, fmaf, sqrtf, fabsf, fmaxf)

#endif
