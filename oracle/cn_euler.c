/*
 * cn_euler.c -- CPU oracle of the compressible Euler RHS and SSP-RK3 stage.
 *
 * TEST INFRASTRUCTURE ONLY (checker for tests/, smoke and the CPU baseline).
 *
 * The reference library has no WENO / Riemann-solver / Runge-Kutta code (its
 * README.rst:28-31 and :43-44 only announce such operators), so this is a
 * restatement of the published methods on top of the restated lab fill
 * (cn_oracle.c, itself pinned against the reference's FieldLab):
 *   - WENO5-JS, Jiang & Shu, J. Comput. Phys. 126 (1996) 202-228: eps = 1e-6,
 *     linear weights (1/10, 6/10, 3/10), reconstruction of the primitive
 *     variables (rho, u, v, w, p); weights normalised with one division:
 *     omega_k = d_k prod_{j!=k} t_j / sum_i d_i prod_{j!=i} t_j, t = (eps+beta)^2;
 *   - Rusanov / local Lax-Friedrichs flux with a = max(|u_n|+c) of both sides;
 *   - SSP-RK3, Shu & Osher, J. Comput. Phys. 77 (1988) 439-471.
 * Every operation, including each fma(), is written in the same order as the
 * device code, and the file is compiled with -ffp-contract=off, so both sides
 * round identically.
 */
#include "cn_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "cn_euler_math.h"

#define DEFINE_EULER(SUF, T, FMA)                                             \
    /* One block: RHS (stage 0) or SSP-RK3 stage of all its cells.  Us, Un,    \
     * out are 5 component bases (comp_stride apart). */                       \
    static int block_##SUF(const or_geom *g, const T *Us, const T *Un, T *out,  \
                           int64_t cstride, const int32_t *const *bc_off,      \
                           const or_bc *const *bcs, int block, int stage,      \
                           T dt, T gamma, T gm1, T igm1, const T ih[3],        \
                           T *lab, uint8_t *w, T *prim, T *flux)               \
    {                                                                          \
        const int N0 = g->n[0], N1 = g->n[1], N2 = g->n[2];                    \
        const int L0 = N0 + 6, L1 = N1 + 6, L2 = N2 + 6;                       \
        const size_t le = (size_t)L0 * L1 * L2;                                \
        T *labs[5];                                                            \
        for (int c = 0; c < 5; ++c) {                                          \
            labs[c] = lab + c * le;                                            \
            int rc = or_lab_fill_##SUF(g, Us + c * cstride, bc_off[c], bcs[c], \
                                       block, labs[c], w);                     \
            if (rc)                                                            \
                return rc;                                                     \
            for (size_t i = 0; i < le; ++i)                                    \
                if (!w[i])                                                     \
                    labs[c][i] = (T)0;                                         \
        }                                                                      \
        for (size_t i = 0; i < le; ++i) {                                      \
            T W[5];                                                            \
            prim_##SUF(labs[0][i], labs[1][i], labs[2][i], labs[3][i],         \
                       labs[4][i], gm1, W);                                    \
            for (int c = 0; c < 5; ++c)                                        \
                prim[c * le + i] = W[c];                                       \
        }                                                                      \
        const size_t cells = (size_t)N0 * N1 * N2;                             \
        T *acc = flux + 5 * (size_t)(N0 + 1) * (N1 + 1) * (N2 + 1);            \
        for (int d = 0; d < 3; ++d) {                                          \
            const int E0 = N0 + (d == 0), E1 = N1 + (d == 1), E2 = N2 + (d == 2); \
            const size_t nf = (size_t)E0 * E1 * E2;                            \
            const ptrdiff_t st = d == 0 ? 1 : (d == 1 ? L0 : (ptrdiff_t)L0 * L1); \
            for (int z = 0; z < E2; ++z)                                       \
                for (int y = 0; y < E1; ++y)                                   \
                    for (int x = 0; x < E0; ++x) {                             \
                        /* face between cell (x,y,z)-e_d and (x,y,z) */        \
                        const ptrdiff_t li = (x + 3) + (ptrdiff_t)L0 *         \
                                             ((y + 3) + (ptrdiff_t)L1 * (z + 3)); \
                        T WL[5], WR[5], F[5], bl[5], nl[5], dl[5], br[5], nr[5], dr[5]; \
                        for (int c = 0; c < 5; ++c) {                          \
                            const T *P = prim + c * le + li;                   \
                            const T v0 = P[-3 * st], v1 = P[-2 * st], v2 = P[-st]; \
                            const T v3 = P[0], v4 = P[st], v5 = P[2 * st];     \
                            weno5_nd_face_##SUF(v0, v1, v2, v3, v4, v5, &bl[c], &nl[c], &dl[c], \
                                                &br[c], &nr[c], &dr[c]);        \
                        }                                                      \
                        face_states5_##SUF(bl, nl, dl, br, nr, dr, WL, WR);    \
                        rusanov_##SUF(WL, WR, d, gamma, igm1, F);              \
                        const size_t fi = x + (size_t)E0 * (y + (size_t)E1 * z); \
                        for (int c = 0; c < 5; ++c)                            \
                            flux[c * nf + fi] = F[c];                          \
                    }                                                          \
            const size_t fst = d == 0 ? 1 : (d == 1 ? (size_t)E0 : (size_t)E0 * E1); \
            for (int z = 0; z < N2; ++z)                                       \
                for (int y = 0; y < N1; ++y)                                   \
                    for (int x = 0; x < N0; ++x) {                             \
                        const size_t ci = x + (size_t)N0 * (y + (size_t)N1 * z); \
                        const size_t fi = x + (size_t)E0 * (y + (size_t)E1 * z); \
                        for (int c = 0; c < 5; ++c) {                          \
                            const T df = flux[c * nf + fi + fst] - flux[c * nf + fi]; \
                            acc[c * cells + ci] = d == 0 ? df * ih[d]          \
                                                         : FMA(df, ih[d], acc[c * cells + ci]); \
                        }                                                      \
                    }                                                          \
        }                                                                      \
        const int64_t boff = (int64_t)block * g->block_stride;                 \
        for (size_t ci = 0; ci < cells; ++ci) {                                \
            for (int c = 0; c < 5; ++c) {                                      \
                const T rhs = -acc[c * cells + ci];                            \
                const int64_t o = c * cstride + boff + (int64_t)ci;            \
                T v;                                                           \
                if (stage == 0) {                                              \
                    v = rhs;                                                   \
                } else {                                                       \
                    const T tt = FMA(dt, rhs, Us[o]);                          \
                    if (stage == 1)                                            \
                        v = tt;                                                \
                    else if (stage == 2)                                       \
                        v = FMA((T)0.75, Un[o], (T)0.25 * tt);                 \
                    else                                                       \
                        v = FMA((T)(1.0 / 3.0), Un[o], (T)(2.0 / 3.0) * tt);   \
                }                                                              \
                out[o] = v;                                                    \
            }                                                                  \
        }                                                                      \
        return 0;                                                              \
    }                                                                          \
                                                                               \
    int or_euler_stage_##SUF(const or_geom *gin, const T *Us, const T *Un,     \
                             T *out, int64_t cstride,                          \
                             const int32_t *const *bc_off,                     \
                             const or_bc *const *bcs, int stage, double dt,    \
                             double gamma, const double h[3], int nthreads)    \
    {                                                                          \
        or_geom g = *gin;                                                      \
        for (int d = 0; d < 3; ++d) {                                          \
            g.lo[d] = 3;                                                       \
            g.hi[d] = 3;                                                       \
        }                                                                      \
        g.tensorial = 0;                                                       \
        const int nblocks = g.nb[0] * g.nb[1] * g.nb[2];                       \
        /* 1/(2h): the Rusanov fluxes are twice the flux (exact) */            \
        const T ih[3] = {(T)0.5 * (T)(1.0 / h[0]), (T)0.5 * (T)(1.0 / h[1]),   \
                         (T)0.5 * (T)(1.0 / h[2])};                            \
        const size_t le = (size_t)(g.n[0] + 6) * (g.n[1] + 6) * (g.n[2] + 6);  \
        const size_t fl = 5 * (size_t)(g.n[0] + 1) * (g.n[1] + 1) * (g.n[2] + 1) + \
                          5 * (size_t)g.n[0] * g.n[1] * g.n[2];                \
        int err = 0;                                                           \
        _Pragma("omp parallel num_threads(nthreads > 0 ? nthreads : 1)")       \
        {                                                                      \
            T *lab = (T *)malloc(5 * le * sizeof(T));                          \
            T *prim = (T *)malloc(5 * le * sizeof(T));                         \
            T *flux = (T *)malloc(fl * sizeof(T));                             \
            uint8_t *w = (uint8_t *)malloc(le);                                \
            if (!lab || !prim || !flux || !w) {                                \
                _Pragma("omp atomic write") err = 2;                           \
            } else {                                                           \
                _Pragma("omp for schedule(dynamic, 1)")                        \
                for (int b = 0; b < nblocks; ++b) {                            \
                    int rc = block_##SUF(&g, Us, Un, out, cstride, bc_off,     \
                                         bcs, b, stage, (T)dt, (T)gamma,       \
                                         (T)(gamma - 1.0),                     \
                                         (T)(1.0 / (gamma - 1.0)), ih, lab, w, \
                                         prim, flux);                          \
                    if (rc) {                                                  \
                        _Pragma("omp atomic write") err = rc;                  \
                    }                                                          \
                }                                                              \
            }                                                                  \
            free(lab);                                                         \
            free(prim);                                                        \
            free(flux);                                                        \
            free(w);                                                           \
        }                                                                      \
        return err;                                                            \
    }

DEFINE_EULER(f64, double, fma)
DEFINE_EULER(f32, float, fmaf)
