/*
 * cn_oracle.h -- CPU oracle for the CubismNova lab/stencil hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithms, used by tests/, the smoke check and the CPU-baseline leg of
 * bench.py as the checker.  The product (cubismnova_b200) never links or
 * calls it.
 *
 * Conventions shared with the product C-ABI:
 *   - a grid component is nblocks[0]*nblocks[1]*nblocks[2] blocks, block i at
 *     element offset i*block_stride, blocks in x-fastest block order
 *     (Grid/BlockFieldAssembler.h:189-194, Core/Index.h:101-117);
 *   - a block holds n[0]*n[1]*n[2] cells, x fastest;
 *   - a stencil is begin = -lo, end = hi + 1 per dimension
 *     (Core/Stencil.h:44-67), lo, hi >= 0;
 *   - a lab is the dense active lab range of one block, extent
 *     L_d = n_d + lo_d + hi_d, lab cell q (q_d in [-lo_d, n_d + hi_d)) at
 *     (q_x+lo_x) + L_x*((q_y+lo_y) + L_y*(q_z+lo_z)).
 */
#ifndef CN_ORACLE_H
#define CN_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_BC_BASE = 0, OR_BC_DIRICHLET = 1, OR_BC_ABSORBING = 2, OR_BC_SYMMETRY = 3 };

typedef struct {
    int32_t dir;
    int32_t side;
    int32_t kind;
    int32_t pad;
    double value; /* Dirichlet value or Symmetry sign */
} or_bc;

typedef struct {
    int32_t nb[3];    /* blocks per dimension */
    int32_t n[3];     /* largest block extent per dimension (labs are this large) */
    int32_t lo[3];    /* -stencil.begin */
    int32_t hi[3];    /* stencil.end - 1 */
    int32_t tensorial;
    int64_t block_stride; /* elements between consecutive blocks */
    /* 1 where only the last block along a dimension holds n entities and the
     * others n - 1 (node fields in every dimension, a face field along its
     * direction: Grid/BlockFieldAssembler.h:124-135); 0 for cell fields */
    int32_t grow[3];
} or_geom;

/* Lab fill of one block (FieldLab::loadData).  bc_off has nblocks+1 entries
 * (CSR over blocks, x-fastest block order), bcs the BC vectors in push order.
 * lab receives the dense active lab range; written[] (same shape) is 1 for
 * every cell whose value the reference defines: loaded cells, Dirichlet cells,
 * and Absorbing/Symmetry cells whose source cell was defined.  Cells the
 * reference leaves untouched (a skipped neighbour that no valid BC covers, or
 * corners of a non-tensorial lab) keep their previous lab content and get 0,
 * as does anything copied from them.  Returns 0 on success. */
int or_lab_fill_f64(const or_geom *g, const double *comp, const int32_t *bc_off,
                    const or_bc *bcs, int block, double *lab, uint8_t *written);
int or_lab_fill_f32(const or_geom *g, const float *comp, const int32_t *bc_off,
                    const or_bc *bcs, int block, float *lab, uint8_t *written);
int or_lab_fill_i32(const or_geom *g, const int32_t *comp, const int32_t *bc_off,
                    const or_bc *bcs, int block, int32_t *lab, uint8_t *written);

/* 7-point Laplacian over a whole grid component, lab stencil (-1,2),
 * non-tensorial, following Kernel/Laplacian/Laplacian.cpp:123-130:
 *   res = ihx2*((u[x+1] - 2u) + u[x-1]) + ihy2*(...) + ihz2*(...)
 * evaluated left to right without contraction.  out has the grid layout. */
int or_laplacian_f64(const or_geom *g, const double *comp, const int32_t *bc_off,
                     const or_bc *bcs, const double ih2[3], double *out);
/* 2nd-order central gradient, component d = 0.5*((u[+d] - u[-d]) * ih[d])
 * (per-term grouping of Kernel/Divergence/nova/nova.cpp:118-125).  out holds
 * 3 components, component stride comp_stride elements. */
int or_gradient_f64(const or_geom *g, const double *comp, const int32_t *bc_off,
                    const or_bc *bcs, const double ih[3], double *out,
                    int64_t comp_stride);
/* ddx gold kernel (ISPC/CFD_2ndOrder/DDX/ddxGold.cpp:9-53) on one pitched
 * source array: dst = fac*((((((s[x-1]+s[x+1])+s[y-1])+s[y+1])+s[z-1])+s[z+1])
 * - 6*s), fac = 1/(factor*factor). */
void or_ddx_f64(int nx, int ny, int nz, const double *src, int xps, int xyps,
                double *dst, int xpd, int xypd, double factor);
void or_ddx_f32(int nx, int ny, int nz, const float *src, int xps, int xyps,
                float *dst, int xpd, int xypd, float factor);

/* Compressible Euler (5 conserved components cstride elements apart, grid
 * layout), lab stencil (-3,4) non-tensorial with per-component BC vectors
 * bc_off[c]/bcs[c]: stage 0 writes the RHS L(Us) to out; stages 1..3 the
 * SSP-RK3 stages  out = Us + dt L | 3/4 Un + 1/4 (Us + dt L) |
 * 1/3 Un + 2/3 (Us + dt L).  out may alias Un but not Us. */
int or_euler_stage_f64(const or_geom *g, const double *Us, const double *Un, double *out,
                       int64_t cstride, const int32_t *const *bc_off, const or_bc *const *bcs,
                       int stage, double dt, double gamma, const double h[3], int nthreads);
int or_euler_stage_f32(const or_geom *g, const float *Us, const float *Un, float *out,
                       int64_t cstride, const int32_t *const *bc_off, const or_bc *const *bcs,
                       int stage, double dt, double gamma, const double h[3], int nthreads);

#ifdef __cplusplus
}
#endif
#endif
