// ref_shim.cpp -- C entry points over the reference CubismNova headers.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile against the unmodified
// reference headers (include/Cubism/...) into oracle/_ref/libcnref.so.  It
// runs the reference's own Grid::Cartesian / Block::FieldLab / BC::* code so
// that the plain-C oracle (cn_oracle.c) can be pinned against it, and it is
// the reference arm of the CPU baseline.  Nothing in the product links it.
#include "Cubism/BC/Absorbing.h"
#include "Cubism/BC/Base.h"
#include "Cubism/BC/Dirichlet.h"
#include "Cubism/BC/Symmetry.h"
#include "Cubism/Block/FieldLab.h"
#include "Cubism/Grid/Cartesian.h"
#include "Cubism/Mesh/StructuredUniform.h"

#include "cn_oracle.h"

#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace Cubism;

namespace
{
using Mesh = Mesh::StructuredUniform<double, 3>;
using MIndex = typename Mesh::MultiIndex;

template <typename T>
struct RefGrid {
    using G = Grid::Cartesian<T, Mesh, EntityType::Cell, 0>;
    using F = typename G::BaseType;
    using Lab = Block::FieldLab<F>;
    using S = typename Lab::StencilType;
    using BCPtr = BC::Base<Lab> *;

    std::unique_ptr<G> grid;
    std::vector<std::unique_ptr<BC::Base<Lab>>> owned;

    RefGrid(const int nb[3], const int n[3], const T *comp, int64_t stride)
    {
        grid.reset(new G(MIndex{nb[0], nb[1], nb[2]}, MIndex{n[0], n[1], n[2]}));
        const size_t cells = (size_t)n[0] * n[1] * n[2];
        for (size_t i = 0; i < grid->size(); ++i) {
            std::memcpy((*grid)[i].getData(), comp + i * stride, cells * sizeof(T));
        }
    }

    void attach(const int32_t *bc_off, const or_bc *bcs)
    {
        if (!bc_off) {
            return;
        }
        for (size_t i = 0; i < grid->size(); ++i) {
            auto &v = (*grid)[i].getBC();
            for (int k = bc_off[i]; k < bc_off[i + 1]; ++k) {
                const or_bc &b = bcs[k];
                BC::Base<Lab> *p = nullptr;
                if (b.kind == OR_BC_DIRICHLET) {
                    p = new BC::Dirichlet<Lab>(b.dir, b.side, (T)b.value);
                } else if (b.kind == OR_BC_ABSORBING) {
                    p = new BC::Absorbing<Lab>(b.dir, b.side);
                } else if (b.kind == OR_BC_SYMMETRY) {
                    p = new BC::Symmetry<Lab>(b.dir, b.side, (T)b.value);
                } else {
                    p = new BC::Base<Lab>(b.dir, b.side);
                }
                owned.emplace_back(p);
                v.push_back(p);
            }
        }
    }
};

template <typename T>
int labFill(const or_geom *g, const T *comp, const int32_t *bc_off,
            const or_bc *bcs, int block, T *lab_out, uint8_t *written)
{
    using R = RefGrid<T>;
    R r(g->nb, g->n, comp, g->block_stride);
    r.attach(bc_off, bcs);
    typename R::Lab lab;
    const typename R::S s(MIndex{-g->lo[0], -g->lo[1], -g->lo[2]},
                          MIndex{g->hi[0] + 1, g->hi[1] + 1, g->hi[2] + 1},
                          g->tensorial != 0);
    lab.allocate(s, (*r.grid)[0].getIndexRange());
    const int L[3] = {g->n[0] + g->lo[0] + g->hi[0], g->n[1] + g->lo[1] + g->hi[1],
                      g->n[2] + g->lo[2] + g->hi[2]};
    const size_t le = (size_t)L[0] * L[1] * L[2];
    std::vector<T> pass[2];
    const T poison[2] = {(T)-12345, (T)54321};
    for (int p = 0; p < 2; ++p) {
        T *mem = reinterpret_cast<T *>(lab.getBlockPtr());
        const size_t nmem = lab.getBlockBytes() / sizeof(T);
        for (size_t i = 0; i < nmem; ++i) {
            mem[i] = poison[p];
        }
        r.grid->loadLab((*r.grid)[block], lab);
        pass[p].resize(le);
        for (int z = 0; z < L[2]; ++z)
            for (int y = 0; y < L[1]; ++y)
                for (int x = 0; x < L[0]; ++x) {
                    pass[p][x + (size_t)L[0] * (y + (size_t)L[1] * z)] =
                        lab(x - g->lo[0], y - g->lo[1], z - g->lo[2]);
                }
    }
    for (size_t i = 0; i < le; ++i) {
        const bool same = std::memcmp(&pass[0][i], &pass[1][i], sizeof(T)) == 0;
        written[i] = same ? 1 : 0;
        if (same) {
            lab_out[i] = pass[0][i];
        }
    }
    return 0;
}

// Laplacian/gradient sweep over all blocks with the reference FieldLab and
// the stencil loops of Kernel/Laplacian/Laplacian.cpp:123-130 and
// Kernel/Divergence/nova/nova.cpp:113-126 (one lab per thread,
// schedule(dynamic,1) as in test/UnitTests/Grid/CartesianTest.cpp:283-317).
struct C1Result {
    double seconds;
};

template <typename T>
void c1Blocks(typename RefGrid<T>::G &u, T *lap, T *grad, int64_t stride,
              int64_t comp_stride, const double ih2[3], const double ih[3],
              int nthreads, int nblocks_to_run)
{
    using R = RefGrid<T>;
    const int nbk = nblocks_to_run;
#pragma omp parallel num_threads(nthreads)
    {
        typename R::Lab lab;
        const typename R::S s(-1, 2, false);
        lab.allocate(s, u[0].getIndexRange());
#pragma omp for schedule(dynamic, 1)
        for (int i = 0; i < nbk; ++i) {
            auto &bf = u[(size_t)i];
            u.loadLab(bf, lab);
            const auto e = bf.getIndexRange().getExtent();
            T *rl = lap ? lap + (size_t)i * stride : nullptr;
            T *rg = grad ? grad + (size_t)i * stride : nullptr;
            for (long z = 0; z < e[2]; ++z)
                for (long y = 0; y < e[1]; ++y)
                    for (long x = 0; x < e[0]; ++x) {
                        const size_t o = x + e[0] * (y + e[1] * z);
                        if (rl) {
                            const T ddx = ih2[0] * (lab(x + 1, y, z) - 2 * lab(x, y, z) + lab(x - 1, y, z));
                            const T ddy = ih2[1] * (lab(x, y + 1, z) - 2 * lab(x, y, z) + lab(x, y - 1, z));
                            const T ddz = ih2[2] * (lab(x, y, z + 1) - 2 * lab(x, y, z) + lab(x, y, z - 1));
                            rl[o] = ddx + ddy + ddz;
                        }
                        if (rg) {
                            const T dx = lab(x + 1, y, z) - lab(x - 1, y, z);
                            const T dy = lab(x, y + 1, z) - lab(x, y - 1, z);
                            const T dz = lab(x, y, z + 1) - lab(x, y, z - 1);
                            rg[o] = 0.5 * (dx * ih[0]);
                            rg[o + comp_stride] = 0.5 * (dy * ih[1]);
                            rg[o + 2 * comp_stride] = 0.5 * (dz * ih[2]);
                        }
                    }
        }
    }
}
} // namespace

extern "C" {

int ref_lab_fill_f64(const or_geom *g, const double *comp, const int32_t *bc_off,
                     const or_bc *bcs, int block, double *lab, uint8_t *written)
{
    return labFill<double>(g, comp, bc_off, bcs, block, lab, written);
}
int ref_lab_fill_f32(const or_geom *g, const float *comp, const int32_t *bc_off,
                     const or_bc *bcs, int block, float *lab, uint8_t *written)
{
    return labFill<float>(g, comp, bc_off, bcs, block, lab, written);
}
int ref_lab_fill_i32(const or_geom *g, const int32_t *comp, const int32_t *bc_off,
                     const or_bc *bcs, int block, int32_t *lab, uint8_t *written)
{
    return labFill<int32_t>(g, comp, bc_off, bcs, block, lab, written);
}

// Periodic grid (no BCs): Laplacian into lap and/or gradient into grad
// (3 components, comp_stride apart); both in the grid layout.  Runs
// nblocks_to_run blocks (all if <= 0) reps times on nthreads threads and
// returns the best seconds per sweep.
double ref_c1_sweep_f64(const int nb[3], const int n[3], const double *comp,
                        int64_t stride, double *lap, double *grad,
                        int64_t comp_stride, const double ih2[3],
                        const double ih[3], int nthreads, int nblocks_to_run,
                        int reps)
{
    RefGrid<double> r(nb, n, comp, stride);
    const int nall = (int)r.grid->size();
    const int nbk = (nblocks_to_run <= 0 || nblocks_to_run > nall) ? nall : nblocks_to_run;
    double best = 1e300;
    for (int k = 0; k < (reps < 1 ? 1 : reps); ++k) {
        const auto t0 = std::chrono::steady_clock::now();
        c1Blocks<double>(*r.grid, lap, grad, stride, comp_stride, ih2, ih, nthreads, nbk);
        const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        best = dt < best ? dt : best;
    }
    return best;
}

int ref_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
}
