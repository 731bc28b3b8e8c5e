/*
 * cn_oracle.c -- CPU oracle (plain C restatement) of the CubismNova lab fill
 * and finite-difference stencils.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and bench.py's
 * CPU-baseline leg as the checker; never by the product.  Compiled with
 * -ffp-contract=off so every a*b+c rounds twice, exactly as written.
 *
 * The lab fill follows the reference step by step rather than the device
 * design (which resolves every ghost cell independently):
 *   1. loadInner    Block/FieldLabLoader.h:129-173
 *   2. periodic/skip from the BC vector, last BC per direction wins
 *                   Block/FieldLab.h:206-214
 *   3. loadGhosts   Block/FieldLabLoader.h:176-287 (26 neighbours, periodic
 *                   block wrap (p+N)%N of Block/FieldLabLoader.h:405-411)
 *   4. BCs in vector order: BC/Dirichlet.h:75-113, BC/Absorbing.h:62-104,
 *                   BC/Symmetry.h:69-114, validity BC/Base.h:73-78.
 */
#include "cn_oracle.h"

#include <string.h>

#define LAB_INDEX(g, qx, qy, qz)                                              \
    ((size_t)((qx) + (g)->lo[0]) +                                             \
     (size_t)((g)->n[0] + (g)->lo[0] + (g)->hi[0]) *                          \
         ((size_t)((qy) + (g)->lo[1]) +                                        \
          (size_t)((g)->n[1] + (g)->lo[1] + (g)->hi[1]) *                     \
              (size_t)((qz) + (g)->lo[2])))

static int geom_ok(const or_geom *g)
{
    for (int d = 0; d < 3; ++d) {
        if (g->nb[d] < 1 || g->n[d] < 1 || g->lo[d] < 0 || g->hi[d] < 0)
            return 0;
        /* ghosts wider than a block would read outside the neighbour */
        if (g->lo[d] > g->n[d] || g->hi[d] > g->n[d])
            return 0;
    }
    return 1;
}

/* extent of block coordinate bc along d (the last block of a grown
 * dimension holds one more entity than the others) */
static int block_extent(const or_geom *g, int d, int bc)
{
    return g->n[d] - (g->grow[d] && bc != g->nb[d] - 1 ? 1 : 0);
}

static int bc_valid(const or_geom *g, int dir)
{
    /* BC/Base.h:73-78: no-op if either side of the stencil has zero width */
    return !(g->lo[dir] == 0 || g->hi[dir] == 0);
}

#define DEFINE_LAB_FILL(SUFFIX, T)                                            \
    int or_lab_fill_##SUFFIX(const or_geom *g, const T *comp,                  \
                             const int32_t *bc_off, const or_bc *bcs,          \
                             int block, T *lab, uint8_t *written)              \
    {                                                                          \
        if (!geom_ok(g))                                                       \
            return 1;                                                          \
        const int nbx = g->nb[0], nby = g->nb[1], nbz = g->nb[2];              \
        const int nblocks = nbx * nby * nbz;                                   \
        if (block < 0 || block >= nblocks)                                     \
            return 1;                                                          \
        const int b[3] = {block % nbx, (block / nbx) % nby,                    \
                          block / (nbx * nby)};                                \
        /* this block's extent; the lab array has the largest extent */        \
        const int N[3] = {block_extent(g, 0, b[0]), block_extent(g, 1, b[1]),  \
                          block_extent(g, 2, b[2])};                           \
        const T *self = comp + (size_t)block * g->block_stride;                \
        memset(written, 0, (size_t)(g->n[0] + g->lo[0] + g->hi[0]) *          \
                               (g->n[1] + g->lo[1] + g->hi[1]) *               \
                               (g->n[2] + g->lo[2] + g->hi[2]));               \
        /* 1. inner */                                                         \
        for (int z = 0; z < N[2]; ++z)                                         \
            for (int y = 0; y < N[1]; ++y)                                     \
                for (int x = 0; x < N[0]; ++x) {                               \
                    const size_t li = LAB_INDEX(g, x, y, z);                   \
                    lab[li] = self[x + (size_t)N[0] * (y + (size_t)N[1] * z)]; \
                    written[li] = 1;                                           \
                }                                                              \
        /* 2. periodic / skip, last BC per direction wins */                   \
        const int b0 = bc_off ? bc_off[block] : 0;                             \
        const int b1 = bc_off ? bc_off[block + 1] : 0;                         \
        int periodic[3] = {1, 1, 1};                                           \
        int skip[3] = {1, 1, 1};                                               \
        for (int k = b0; k < b1; ++k) {                                        \
            periodic[bcs[k].dir] = (bcs[k].kind == OR_BC_BASE);                \
            skip[bcs[k].dir] = (bcs[k].side == 0) ? -1 : 1;                    \
        }                                                                      \
        /* 3. ghosts from the 26 neighbours */                                 \
        for (int i = 0; i < 27; ++i) {                                         \
            if (i == 13)                                                       \
                continue;                                                      \
            const int bi[3] = {i % 3 - 1, (i / 3) % 3 - 1, i / 9 - 1};         \
            int skipped = 0;                                                   \
            for (int d = 0; d < 3; ++d)                                        \
                if (!periodic[d] && bi[d] == skip[d])                          \
                    skipped = 1;                                               \
            if (skipped)                                                       \
                continue;                                                      \
            const int isum = (bi[0] != 0) + (bi[1] != 0) + (bi[2] != 0);       \
            if (!g->tensorial && isum > 1)                                     \
                continue;                                                      \
            const int nbi[3] = {(b[0] + bi[0] + nbx) % nbx,                    \
                                (b[1] + bi[1] + nby) % nby,                    \
                                (b[2] + bi[2] + nbz) % nbz};                   \
            const T *nb = comp + (size_t)(nbi[0] + nbx * (nbi[1] + nby * nbi[2])) \
                                     * g->block_stride;                        \
            /* neighbour extent; a lower neighbour is read from its end */     \
            const int NN[3] = {block_extent(g, 0, nbi[0]), block_extent(g, 1, nbi[1]), \
                               block_extent(g, 2, nbi[2])};                    \
            int beg[3], end[3];                                                \
            for (int d = 0; d < 3; ++d) {                                      \
                beg[d] = bi[d] < 0 ? -g->lo[d] : (bi[d] == 0 ? 0 : N[d]);      \
                end[d] = bi[d] < 0 ? 0 : (bi[d] == 0 ? N[d] : N[d] + g->hi[d]); \
            }                                                                  \
            for (int z = beg[2]; z < end[2]; ++z)                              \
                for (int y = beg[1]; y < end[1]; ++y)                          \
                    for (int x = beg[0]; x < end[0]; ++x) {                    \
                        const int sx = x - bi[0] * N[0] + (bi[0] < 0 ? NN[0] - N[0] : 0); \
                        const int sy = y - bi[1] * N[1] + (bi[1] < 0 ? NN[1] - N[1] : 0); \
                        const int sz = z - bi[2] * N[2] + (bi[2] < 0 ? NN[2] - N[2] : 0); \
                        const size_t li = LAB_INDEX(g, x, y, z);               \
                        lab[li] = nb[sx + (size_t)NN[0] * (sy + (size_t)NN[1] * sz)]; \
                        written[li] = 1;                                       \
                    }                                                          \
        }                                                                      \
        /* 4. boundary conditions in vector order */                           \
        for (int k = b0; k < b1; ++k) {                                        \
            const or_bc bc = bcs[k];                                           \
            const int dir = bc.dir;                                            \
            if (bc.kind == OR_BC_BASE || !bc_valid(g, dir))                    \
                continue;                                                      \
            /* slab: ghost layers of (dir, side); other dims span the active   \
             * range (non-tensorial) or the whole lab range (tensorial) */     \
            int beg[3], end[3];                                                \
            for (int d = 0; d < 3; ++d) {                                      \
                beg[d] = g->tensorial ? -g->lo[d] : 0;                         \
                end[d] = g->tensorial ? N[d] + g->hi[d] : N[d];                \
            }                                                                  \
            if (bc.side == 0) {                                                \
                beg[dir] = -g->lo[dir];                                        \
                end[dir] = 0;                                                  \
            } else {                                                           \
                beg[dir] = N[dir];                                             \
                end[dir] = N[dir] + g->hi[dir];                                \
            }                                                                  \
            const T cval = (T)bc.value;                                        \
            for (int z = beg[2]; z < end[2]; ++z)                              \
                for (int y = beg[1]; y < end[1]; ++y)                          \
                    for (int x = beg[0]; x < end[0]; ++x) {                    \
                        int q[3] = {x, y, z};                                  \
                        const size_t li = LAB_INDEX(g, x, y, z);               \
                        T v;                                                   \
                        uint8_t def = 1;                                       \
                        if (bc.kind == OR_BC_DIRICHLET) {                      \
                            v = cval;                                          \
                        } else if (bc.kind == OR_BC_ABSORBING) {               \
                            q[dir] = (bc.side == 0) ? 0 : N[dir] - 1;          \
                            const size_t si = LAB_INDEX(g, q[0], q[1], q[2]);  \
                            v = lab[si];                                       \
                            def = written[si];                                 \
                        } else { /* symmetry: r = roffset - q */               \
                            const int roff = (bc.side == 0) ? -1 : 2 * N[dir] - 1; \
                            q[dir] = roff - q[dir];                            \
                            const size_t si = LAB_INDEX(g, q[0], q[1], q[2]);  \
                            v = cval * lab[si];                                \
                            def = written[si];                                 \
                        }                                                      \
                        lab[li] = v;                                           \
                        written[li] = def;                                     \
                    }                                                          \
        }                                                                      \
        return 0;                                                              \
    }

DEFINE_LAB_FILL(f64, double)
DEFINE_LAB_FILL(f32, float)
DEFINE_LAB_FILL(i32, int32_t)

/* ---------------------------------------------------------------------- */
/* Finite-difference stencils on a whole grid component                    */
/* ---------------------------------------------------------------------- */

static size_t lab_elems(const or_geom *g)
{
    return (size_t)(g->n[0] + g->lo[0] + g->hi[0]) *
           (size_t)(g->n[1] + g->lo[1] + g->hi[1]) *
           (size_t)(g->n[2] + g->lo[2] + g->hi[2]);
}

#include <stdlib.h>

int or_laplacian_f64(const or_geom *gin, const double *comp,
                     const int32_t *bc_off, const or_bc *bcs,
                     const double ih2[3], double *out)
{
    or_geom g = *gin;
    for (int d = 0; d < 3; ++d) {
        g.lo[d] = 1;
        g.hi[d] = 1;
    }
    g.tensorial = 0;
    const size_t le = lab_elems(&g);
    double *lab = (double *)malloc(le * sizeof(double));
    uint8_t *w = (uint8_t *)malloc(le);
    if (!lab || !w) {
        free(lab);
        free(w);
        return 2;
    }
    const int nblocks = g.nb[0] * g.nb[1] * g.nb[2];
    const int *N = g.n;
    int rc = 0;
    for (int b = 0; b < nblocks && !rc; ++b) {
        memset(lab, 0, le * sizeof(double));
        rc = or_lab_fill_f64(&g, comp, bc_off, bcs, b, lab, w);
        double *res = out + (size_t)b * g.block_stride;
        for (int z = 0; z < N[2]; ++z)
            for (int y = 0; y < N[1]; ++y)
                for (int x = 0; x < N[0]; ++x) {
                    const double c = lab[LAB_INDEX(&g, x, y, z)];
                    const double ddx =
                        ih2[0] * (lab[LAB_INDEX(&g, x + 1, y, z)] - 2 * c +
                                  lab[LAB_INDEX(&g, x - 1, y, z)]);
                    const double ddy =
                        ih2[1] * (lab[LAB_INDEX(&g, x, y + 1, z)] - 2 * c +
                                  lab[LAB_INDEX(&g, x, y - 1, z)]);
                    const double ddz =
                        ih2[2] * (lab[LAB_INDEX(&g, x, y, z + 1)] - 2 * c +
                                  lab[LAB_INDEX(&g, x, y, z - 1)]);
                    res[x + (size_t)N[0] * (y + (size_t)N[1] * z)] =
                        ddx + ddy + ddz;
                }
    }
    free(lab);
    free(w);
    return rc;
}

int or_gradient_f64(const or_geom *gin, const double *comp,
                    const int32_t *bc_off, const or_bc *bcs, const double ih[3],
                    double *out, int64_t comp_stride)
{
    or_geom g = *gin;
    for (int d = 0; d < 3; ++d) {
        g.lo[d] = 1;
        g.hi[d] = 1;
    }
    g.tensorial = 0;
    const size_t le = lab_elems(&g);
    double *lab = (double *)malloc(le * sizeof(double));
    uint8_t *w = (uint8_t *)malloc(le);
    if (!lab || !w) {
        free(lab);
        free(w);
        return 2;
    }
    const int nblocks = g.nb[0] * g.nb[1] * g.nb[2];
    const int *N = g.n;
    int rc = 0;
    for (int b = 0; b < nblocks && !rc; ++b) {
        memset(lab, 0, le * sizeof(double));
        rc = or_lab_fill_f64(&g, comp, bc_off, bcs, b, lab, w);
        for (int z = 0; z < N[2]; ++z)
            for (int y = 0; y < N[1]; ++y)
                for (int x = 0; x < N[0]; ++x) {
                    const size_t o = (size_t)b * g.block_stride + x +
                                     (size_t)N[0] * (y + (size_t)N[1] * z);
                    const double dx = lab[LAB_INDEX(&g, x + 1, y, z)] -
                                      lab[LAB_INDEX(&g, x - 1, y, z)];
                    const double dy = lab[LAB_INDEX(&g, x, y + 1, z)] -
                                      lab[LAB_INDEX(&g, x, y - 1, z)];
                    const double dz = lab[LAB_INDEX(&g, x, y, z + 1)] -
                                      lab[LAB_INDEX(&g, x, y, z - 1)];
                    out[o] = 0.5 * (dx * ih[0]);
                    out[o + comp_stride] = 0.5 * (dy * ih[1]);
                    out[o + 2 * comp_stride] = 0.5 * (dz * ih[2]);
                }
    }
    free(lab);
    free(w);
    return rc;
}

#define DEFINE_DDX(SUFFIX, T)                                                 \
    void or_ddx_##SUFFIX(int nx, int ny, int nz, const T *src, int xps,        \
                         int xyps, T *dst, int xpd, int xypd, T factor)        \
    {                                                                          \
        const T fac = 1.0 / (factor * factor);                                 \
        for (int iz = 0; iz < nz; ++iz)                                        \
            for (int iy = 0; iy < ny; ++iy)                                    \
                for (int ix = 0; ix < nx; ++ix) {                              \
                    const T *s = src + ix + (ptrdiff_t)xps * iy +              \
                                 (ptrdiff_t)xyps * iz;                         \
                    dst[ix + (ptrdiff_t)xpd * iy + (ptrdiff_t)xypd * iz] =     \
                        fac * (s[-1] + s[1] + s[-xps] + s[xps] + s[-xyps] +    \
                               s[xyps] - (T)6 * s[0]);                         \
                }                                                              \
    }

DEFINE_DDX(f64, double)
DEFINE_DDX(f32, float)
