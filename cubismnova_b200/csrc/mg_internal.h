// mg_internal.h -- multigrid solver state shared by mg.cu and learned.cu.
#pragma once

#include "cn_internal.h"

#include <vector>

struct cn_nn;

struct cn_mg {
    int nlevels;
    int nu1, nu2;
    double omega;
    std::vector<cn_grid *> p, pt, f, k; // per level (FP32); k[0] is the caller's grid
    std::vector<float *> coef;          // per level: 8 FP32 per cell (k+ faces x,y,z, k- faces x,y,z, D, 0)
    double *face64 = nullptr;           // finest level: FP64 harmonic face means, per block x, y, z faces
    cn_grid *r32 = nullptr;             // finest FP32 residual
    double *partials = nullptr;
    double *sums = nullptr;
    int *iters = nullptr;
    int nparts = 0;
    int coarse_iters_max = 0;
    // coarsest levels of at most kCoarseDenseMax cells: the inverse of the
    // regularised coarsest operator (N x N FP64, symmetric), else null (CG)
    double *coarse_inv = nullptr;
    int coarse_n = 0;
    // learned smoother: network, the levels it replaces Jacobi on (bit l),
    // and per-level work grids (features, hidden activations, output)
    cn_nn *nn = nullptr;
    unsigned nn_levels = 0;      // pre-smoothing levels (bit l)
    unsigned nn_post_levels = 0; // post-smoothing levels (bit l)
    int nn_pre_apps = -1, nn_post_apps = -1; // applications per smoothing (-1: nu1 / nu2)
    std::vector<cn_grid *> nn_bufs; // 4 per level: X (2 comps), H1 (16), H2 (16), Y (1)
    std::vector<void *> nn_act;     // 2 per level: BF16 channels-last activations (tensor-core path)
    // optional hook run at the finest level after the coarse-grid correction
    cn_status (*capture)(cn_mg *, cudaStream_t) = nullptr;
    void *capture_ctx = nullptr;
};

namespace cn {
namespace mg {
struct KArgs;
}
} // namespace cn

extern const cn_stencil kS1, kS1t;
unsigned grid_for(int64_t n);
float *fptr(cn_grid *g);
cn_status vcycle(cn_mg *m, int l, cudaStream_t st);
// learned smoothing: `apps` applications of the network on level l
extern "C" cn_status cn_mg_accumulate(cn_mg *m, cn_grid *p64, void *stream);
extern "C" cn_status cn_mg_residual(cn_mg *m, const cn_grid *p64, const cn_grid *f, cn_grid *r32, double *rr,
                                      double *ff, void *stream);
cn_status nn_smooth(cn_mg *m, int l, int apps, bool zero_guess, cudaStream_t st);
