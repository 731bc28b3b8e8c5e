/*
 * cn_amr.c -- CPU oracle of the two-level AMR ghost fill and the Euler stage
 * on AMR blocks.  TEST INFRASTRUCTURE ONLY.
 *
 * The reference has no AMR code (level interfaces appear only in its notes,
 * test/sandbox/doc/notes/01_notes.md:192-196); this restates the standard
 * block-structured rules in the operation order of the device code:
 *   same level: copy; coarser source: trilinear prolongation, weights 3/4,
 *   1/4 per direction (x, then y, then z), neighbour index clamped to the
 *   source block; finer source: ((c0+c1)+(c2+c3)) + ((c4+c5)+(c6+c7)) times
 *   1/8, child c = dx | dy<<1 | dz<<2.
 * Positions are in level-1 cell units on a periodic box of L[0] x L[1] x L[2]
 * cells; a block of level l has cell size 2 - l.
 */
#include "cn_euler_math.h"
#include "cn_oracle.h"

#include <stdlib.h>
#include <string.h>

typedef struct {
    int32_t level, n, ox, oy, oz, pad;
    int64_t off;
    double ih;
} or_amr_block;

static int wrapi(int x, int L) { return x < 0 ? x + L : (x >= L ? x - L : x); }
static int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

static double cellv(const double *c, const or_amr_block *B, int x, int y, int z)
{
    return c[B->off + x + (int64_t)B->n * (y + (int64_t)B->n * z)];
}

static int *build_lookup(const or_amr_block *blk, int nblocks, const int *L)
{
    const int lx = L[0] / 8, ly = L[1] / 8, lz = L[2] / 8;
    int *lk = (int *)malloc(sizeof(int) * (size_t)lx * ly * lz);
    if (!lk)
        return NULL;
    for (size_t i = 0; i < (size_t)lx * ly * lz; ++i)
        lk[i] = -1;
    for (int b = 0; b < nblocks; ++b) {
        const int cs = blk[b].level == 0 ? 2 : 1, span = blk[b].n * cs / 8;
        for (int k = 0; k < span; ++k)
            for (int j = 0; j < span; ++j)
                for (int i = 0; i < span; ++i)
                    lk[(blk[b].ox / 8 + i) + lx * ((blk[b].oy / 8 + j) + ly * (blk[b].oz / 8 + k))] = b;
    }
    return lk;
}

static double amr_value(const double *comp, const or_amr_block *blk, const int *lk, const int *L, int b, int qx,
                        int qy, int qz)
{
    const or_amr_block *B = &blk[b];
    if (qx >= 0 && qx < B->n && qy >= 0 && qy < B->n && qz >= 0 && qz < B->n)
        return cellv(comp, B, qx, qy, qz);
    const int lx = L[0] / 8, ly = L[1] / 8, cs = B->level == 0 ? 2 : 1;
    const int X = wrapi(B->ox + qx * cs, L[0]), Y = wrapi(B->oy + qy * cs, L[1]), Z = wrapi(B->oz + qz * cs, L[2]);
    const or_amr_block *S = &blk[lk[(X >> 3) + lx * ((Y >> 3) + ly * (Z >> 3))]];
    const int fx = X - S->ox, fy = Y - S->oy, fz = Z - S->oz;
    if (S->level == B->level) {
        const int css = S->level == 0 ? 2 : 1;
        return cellv(comp, S, fx / css, fy / css, fz / css);
    }
    if (S->level < B->level) {
        const int px = fx >> 1, py = fy >> 1, pz = fz >> 1;
        const int qx1 = clampi(px + ((fx & 1) ? 1 : -1), 0, S->n - 1);
        const int qy1 = clampi(py + ((fy & 1) ? 1 : -1), 0, S->n - 1);
        const int qz1 = clampi(pz + ((fz & 1) ? 1 : -1), 0, S->n - 1);
        const double e000 = cellv(comp, S, px, py, pz), e100 = cellv(comp, S, qx1, py, pz);
        const double e010 = cellv(comp, S, px, qy1, pz), e110 = cellv(comp, S, qx1, qy1, pz);
        const double e001 = cellv(comp, S, px, py, qz1), e101 = cellv(comp, S, qx1, py, qz1);
        const double e011 = cellv(comp, S, px, qy1, qz1), e111 = cellv(comp, S, qx1, qy1, qz1);
        const double a0 = 0.75 * e000 + 0.25 * e100;
        const double a1 = 0.75 * e010 + 0.25 * e110;
        const double a2 = 0.75 * e001 + 0.25 * e101;
        const double a3 = 0.75 * e011 + 0.25 * e111;
        const double b0 = 0.75 * a0 + 0.25 * a1;
        const double b1 = 0.75 * a2 + 0.25 * a3;
        return 0.75 * b0 + 0.25 * b1;
    }
    double v[8];
    for (int k = 0; k < 8; ++k)
        v[k] = cellv(comp, S, fx + (k & 1), fy + ((k >> 1) & 1), fz + (k >> 2));
    return (((v[0] + v[1]) + (v[2] + v[3])) + ((v[4] + v[5]) + (v[6] + v[7]))) * 0.125;
}

/* dense lab (n+2g)^3 of block b, face ghosts only; written[] marks defined cells */
int or_amr_lab_f64(const or_amr_block *blk, int nblocks, const int *L, const double *comp, int b, int g,
                   double *lab, uint8_t *written)
{
    int *lk = build_lookup(blk, nblocks, L);
    if (!lk)
        return 2;
    const int n = blk[b].n, E = n + 2 * g;
    for (int z = -g; z < n + g; ++z)
        for (int y = -g; y < n + g; ++y)
            for (int x = -g; x < n + g; ++x) {
                const size_t i = (x + g) + (size_t)E * ((y + g) + (size_t)E * (z + g));
                const int out = (x < 0 || x >= n) + (y < 0 || y >= n) + (z < 0 || z >= n);
                written[i] = out <= 1;
                if (out <= 1)
                    lab[i] = amr_value(comp, blk, lk, L, b, x, y, z);
            }
    free(lk);
    return 0;
}

/* Euler RHS (stage 0) / SSP-RK3 stage on all AMR blocks, FP64, periodic box;
 * face loops and stage update of cn_euler.c with each block's own 1/h. */
int or_amr_stage_f64(const or_amr_block *blk, int nblocks, const int *ext, const double *Us, const double *Un,
                     double *out, int64_t cstride, int stage, double dt, double gamma)
{
    int *lk = build_lookup(blk, nblocks, ext);
    if (!lk)
        return 2;
    const double gm1 = gamma - 1.0, igm1 = 1.0 / (gamma - 1.0);
    int rc = 0;
    /* blocks are independent: each writes its own cells of out */
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < nblocks; ++b) {
        int brc = 0;
        const int n = blk[b].n, L = n + 6;
        const size_t le = (size_t)L * L * L;
        double *prim = (double *)calloc(5 * le, sizeof(double));
        double *flux = (double *)malloc(sizeof(double) * 5 * (size_t)(n + 1) * (n + 1) * (n + 1));
        double *acc = (double *)malloc(sizeof(double) * 5 * (size_t)n * n * n);
        if (!prim || !flux || !acc) {
            brc = 2;
        } else {
            for (int z = -3; z < n + 3; ++z)
                for (int y = -3; y < n + 3; ++y)
                    for (int x = -3; x < n + 3; ++x) {
                        const int o = (x < 0 || x >= n) + (y < 0 || y >= n) + (z < 0 || z >= n);
                        if (o > 1)
                            continue;
                        double u[5], W[5];
                        for (int c = 0; c < 5; ++c)
                            u[c] = amr_value(Us + c * cstride, blk, lk, ext, b, x, y, z);
                        prim_f64(u[0], u[1], u[2], u[3], u[4], gm1, W);
                        const size_t li = (x + 3) + (size_t)L * ((y + 3) + (size_t)L * (z + 3));
                        for (int c = 0; c < 5; ++c)
                            prim[c * le + li] = W[c];
                    }
            const size_t cells = (size_t)n * n * n;
            const double ih = 0.5 * blk[b].ih; /* 1/(2h): the Rusanov fluxes are twice the flux */
            for (int d = 0; d < 3; ++d) {
                const int E0 = n + (d == 0), E1 = n + (d == 1), E2 = n + (d == 2);
                const size_t nf = (size_t)E0 * E1 * E2;
                const ptrdiff_t st = d == 0 ? 1 : (d == 1 ? L : (ptrdiff_t)L * L);
                for (int z = 0; z < E2; ++z)
                    for (int y = 0; y < E1; ++y)
                        for (int x = 0; x < E0; ++x) {
                            const ptrdiff_t li = (x + 3) + (ptrdiff_t)L * ((y + 3) + (ptrdiff_t)L * (z + 3));
                            double WL[5], WR[5], F[5], bl[5], nl[5], dl[5], br[5], nr[5], dr[5];
                            for (int c = 0; c < 5; ++c) {
                                const double *P = prim + c * le + li;
                                weno5_nd_face_f64(P[-3 * st], P[-2 * st], P[-st], P[0], P[st], P[2 * st], &bl[c],
                                                  &nl[c], &dl[c], &br[c], &nr[c], &dr[c]);
                            }
                            face_states5_f64(bl, nl, dl, br, nr, dr, WL, WR);
                            rusanov_f64(WL, WR, d, gamma, igm1, F);
                            const size_t fi = x + (size_t)E0 * (y + (size_t)E1 * z);
                            for (int c = 0; c < 5; ++c)
                                flux[c * nf + fi] = F[c];
                        }
                const size_t fst = d == 0 ? 1 : (d == 1 ? (size_t)E0 : (size_t)E0 * E1);
                for (int z = 0; z < n; ++z)
                    for (int y = 0; y < n; ++y)
                        for (int x = 0; x < n; ++x) {
                            const size_t ci = x + (size_t)n * (y + (size_t)n * z);
                            const size_t fi = x + (size_t)E0 * (y + (size_t)E1 * z);
                            for (int c = 0; c < 5; ++c) {
                                const double df = flux[c * nf + fi + fst] - flux[c * nf + fi];
                                acc[c * cells + ci] = d == 0 ? df * ih : fma(df, ih, acc[c * cells + ci]);
                            }
                        }
            }
            for (size_t ci = 0; ci < cells; ++ci)
                for (int c = 0; c < 5; ++c) {
                    const double rhs = -acc[c * cells + ci];
                    const int64_t o = c * cstride + blk[b].off + (int64_t)ci;
                    double v;
                    if (stage == 0)
                        v = rhs;
                    else {
                        const double tt = fma(dt, rhs, Us[o]);
                        if (stage == 1)
                            v = tt;
                        else if (stage == 2)
                            v = fma(0.75, Un[o], 0.25 * tt);
                        else
                            v = fma(1.0 / 3.0, Un[o], (2.0 / 3.0) * tt);
                    }
                    out[o] = v;
                }
        }
        free(prim);
        free(flux);
        free(acc);
        if (brc) {
#pragma omp atomic write
            rc = brc;
        }
    }
    free(lk);
    return rc;
}
