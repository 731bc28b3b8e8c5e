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
#include "Cubism/IO/FieldAOS.h"
#include "Cubism/Mesh/StructuredUniform.h"

#include "cn_oracle.h"
#include "cn_euler_math.h"

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

// Euler RHS / SSP-RK3 stage on labs loaded by the reference FieldLab (one lab
// per component, stencil (-3,4) non-tensorial, per-component BC vectors), the
// face loops of cn_euler.c.  Runs blocks [b0, b0+cnt) on nthreads threads.
template <typename T>
static double eulerStage(const int nb[3], const int n[3], const T *Us, const T *Un, T *out,
                         int64_t stride, int64_t cstride, const int32_t *const *bc_off,
                         const or_bc *const *bcs, int stage, double dt, double gamma,
                         const double h[3], int nthreads, int b0, int cnt, int reps);

template <>
double eulerStage<double>(const int nb[3], const int n[3], const double *Us, const double *Un,
                          double *out, int64_t stride, int64_t cstride,
                          const int32_t *const *bc_off, const or_bc *const *bcs, int stage,
                          double dt, double gamma, const double h[3], int nthreads, int b0,
                          int cnt, int reps)
{
    using T = double;
    using R = RefGrid<T>;
    std::vector<std::unique_ptr<R>> g;
    for (int c = 0; c < 5; ++c) {
        g.emplace_back(new R(nb, n, Us + c * cstride, stride));
        g.back()->attach(bc_off ? bc_off[c] : nullptr, bcs ? bcs[c] : nullptr);
    }
    // 1/(2h): the Rusanov fluxes are twice the flux (exact)
    const T ih[3] = {T(0.5) * (T)(1.0 / h[0]), T(0.5) * (T)(1.0 / h[1]), T(0.5) * (T)(1.0 / h[2])};
    const T gm1 = (T)(gamma - 1.0), igm1 = (T)(1.0 / (gamma - 1.0)), gam = (T)gamma, dtt = (T)dt;
    const int N0 = n[0], N1 = n[1], N2 = n[2];
    double best = 1e300;
    for (int rep = 0; rep < (reps < 1 ? 1 : reps); ++rep) {
        const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel num_threads(nthreads)
        {
            typename R::Lab lab[5];
            const typename R::S s(-3, 4, false);
            for (int c = 0; c < 5; ++c) lab[c].allocate(s, (*g[0]->grid)[0].getIndexRange());
            const int L0 = N0 + 6, L1 = N1 + 6, L2 = N2 + 6;
            const size_t le = (size_t)L0 * L1 * L2;
            std::vector<T> prim(5 * le), flux(5 * (size_t)(N0 + 1) * (N1 + 1) * (N2 + 1)),
                acc(5 * (size_t)N0 * N1 * N2);
#pragma omp for schedule(dynamic, 1)
            for (int b = b0; b < b0 + cnt; ++b) {
                for (int c = 0; c < 5; ++c) g[c]->grid->loadLab((*g[c]->grid)[(size_t)b], lab[c]);
                for (int z = -3; z < N2 + 3; ++z)
                    for (int y = -3; y < N1 + 3; ++y)
                        for (int x = -3; x < N0 + 3; ++x) {
                            const int nout = (x < 0 || x >= N0) + (y < 0 || y >= N1) + (z < 0 || z >= N2);
                            if (nout > 1) continue; // corners of a non-tensorial lab
                            T W[5];
                            prim_f64(lab[0](x, y, z), lab[1](x, y, z), lab[2](x, y, z), lab[3](x, y, z),
                                     lab[4](x, y, z), gm1, W);
                            const size_t li = (x + 3) + (size_t)L0 * ((y + 3) + (size_t)L1 * (z + 3));
                            for (int c = 0; c < 5; ++c) prim[c * le + li] = W[c];
                        }
                const size_t cells = (size_t)N0 * N1 * N2;
                for (int d = 0; d < 3; ++d) {
                    const int E0 = N0 + (d == 0), E1 = N1 + (d == 1), E2 = N2 + (d == 2);
                    const size_t nf = (size_t)E0 * E1 * E2;
                    const ptrdiff_t st = d == 0 ? 1 : (d == 1 ? L0 : (ptrdiff_t)L0 * L1);
                    for (int z = 0; z < E2; ++z)
                        for (int y = 0; y < E1; ++y)
                            for (int x = 0; x < E0; ++x) {
                                const ptrdiff_t li = (x + 3) + (ptrdiff_t)L0 * ((y + 3) + (ptrdiff_t)L1 * (z + 3));
                                T WL[5], WR[5], F[5], bl[5], nl[5], dl[5], br[5], nr[5], dr[5];
                                for (int c = 0; c < 5; ++c) {
                                    const T *P = prim.data() + c * le + li;
                                    const T v0 = P[-3 * st], v1 = P[-2 * st], v2 = P[-st];
                                    const T v3 = P[0], v4 = P[st], v5 = P[2 * st];
                                    weno5_nd_face_f64(v0, v1, v2, v3, v4, v5, &bl[c], &nl[c], &dl[c], &br[c], &nr[c],
                                                      &dr[c]);
                                }
                                face_states5_f64(bl, nl, dl, br, nr, dr, WL, WR);
                                rusanov_f64(WL, WR, d, gam, igm1, F);
                                const size_t fi = x + (size_t)E0 * (y + (size_t)E1 * z);
                                for (int c = 0; c < 5; ++c) flux[c * nf + fi] = F[c];
                            }
                    const size_t fst = d == 0 ? 1 : (d == 1 ? (size_t)E0 : (size_t)E0 * E1);
                    for (int z = 0; z < N2; ++z)
                        for (int y = 0; y < N1; ++y)
                            for (int x = 0; x < N0; ++x) {
                                const size_t ci = x + (size_t)N0 * (y + (size_t)N1 * z);
                                const size_t fi = x + (size_t)E0 * (y + (size_t)E1 * z);
                                for (int c = 0; c < 5; ++c) {
                                    const T df = flux[c * nf + fi + fst] - flux[c * nf + fi];
                                    acc[c * cells + ci] = d == 0 ? df * ih[d] : std::fma(df, ih[d], acc[c * cells + ci]);
                                }
                            }
                }
                const int64_t boff = (int64_t)b * stride;
                for (size_t ci = 0; ci < cells; ++ci)
                    for (int c = 0; c < 5; ++c) {
                        const T rhs = -acc[c * cells + ci];
                        const int64_t o = c * cstride + boff + (int64_t)ci;
                        T v;
                        if (stage == 0) v = rhs;
                        else {
                            const T tt = std::fma(dtt, rhs, Us[o]);
                            if (stage == 1) v = tt;
                            else if (stage == 2) v = std::fma((T)0.75, Un[o], (T)0.25 * tt);
                            else v = std::fma((T)(1.0 / 3.0), Un[o], (T)(2.0 / 3.0) * tt);
                        }
                        out[o] = v;
                    }
            }
        }
        const double dts = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        best = dts < best ? dts : best;
    }
    return best;
}
// Lab of one block of a node grid or of one direction of a face container
// grid (Grid::Cartesian<T, Mesh, EntityType::Node|Face, 0>): g->n is the
// field's index-range extent, g->block_stride the storage stride.
template <typename T, EntityType E>
int labFillEntity(const or_geom *g, int face_dir, const T *comp, const int32_t *bc_off, const or_bc *bcs,
                  int block, T *lab_out, uint8_t *written)
{
    using G = Grid::Cartesian<T, Mesh, E, 0>;
    using F = typename G::BaseType::FieldType; // the scalar (face) field
    using Lab = Block::FieldLab<F>;
    using S = typename Lab::StencilType;
    int cells[3];
    for (int d = 0; d < 3; ++d)
        cells[d] = g->n[d] - ((E == EntityType::Node || d == face_dir) ? 1 : 0);
    G grid(MIndex{g->nb[0], g->nb[1], g->nb[2]}, MIndex{cells[0], cells[1], cells[2]});
    auto field = [&](size_t i) -> F & {
        if constexpr (E == EntityType::Face) {
            return grid[i][(size_t)face_dir];
        } else {
            return grid[i];
        }
    };
    const size_t ext = (size_t)g->n[0] * g->n[1] * g->n[2];
    for (size_t i = 0; i < grid.size(); ++i)
        std::memcpy(field(i).getData(), comp + i * g->block_stride, ext * sizeof(T));
    std::vector<std::unique_ptr<BC::Base<Lab>>> owned;
    if (bc_off) {
        for (size_t i = 0; i < grid.size(); ++i) {
            auto &v = field(i).getBC();
            for (int k = bc_off[i]; k < bc_off[i + 1]; ++k) {
                const or_bc &b = bcs[k];
                BC::Base<Lab> *pb = nullptr;
                if (b.kind == OR_BC_DIRICHLET) pb = new BC::Dirichlet<Lab>(b.dir, b.side, (T)b.value);
                else if (b.kind == OR_BC_ABSORBING) pb = new BC::Absorbing<Lab>(b.dir, b.side);
                else if (b.kind == OR_BC_SYMMETRY) pb = new BC::Symmetry<Lab>(b.dir, b.side, (T)b.value);
                else pb = new BC::Base<Lab>(b.dir, b.side);
                owned.emplace_back(pb);
                v.push_back(pb);
            }
        }
    }
    Lab lab;
    const S s(MIndex{-g->lo[0], -g->lo[1], -g->lo[2]}, MIndex{g->hi[0] + 1, g->hi[1] + 1, g->hi[2] + 1},
              g->tensorial != 0);
    lab.allocate(s, field(0).getIndexRange());
    const int L[3] = {g->n[0] + g->lo[0] + g->hi[0], g->n[1] + g->lo[1] + g->hi[1], g->n[2] + g->lo[2] + g->hi[2]};
    const size_t le = (size_t)L[0] * L[1] * L[2];
    std::vector<T> pass[2];
    const T poison[2] = {(T)-12345, (T)54321};
    for (int p = 0; p < 2; ++p) {
        T *mem = reinterpret_cast<T *>(lab.getBlockPtr());
        const size_t nmem = lab.getBlockBytes() / sizeof(T);
        for (size_t i = 0; i < nmem; ++i) mem[i] = poison[p];
        // Cartesian::loadLab (Grid/Cartesian.h:412-427) without its extent
        // assert, which calls FaceContainer::getIndexRange() with no face
        // index and does not compile for face containers
        auto idx = grid.getIndexFunctor((size_t)0, (size_t)(face_dir < 0 ? 0 : face_dir));
        lab.loadData(field((size_t)block).getState().block_index, idx);
        pass[p].resize(le);
        for (int z = 0; z < L[2]; ++z)
            for (int y = 0; y < L[1]; ++y)
                for (int x = 0; x < L[0]; ++x)
                    pass[p][x + (size_t)L[0] * (y + (size_t)L[1] * z)] = lab(x - g->lo[0], y - g->lo[1], z - g->lo[2]);
    }
    for (size_t i = 0; i < le; ++i) {
        const bool same = std::memcmp(&pass[0][i], &pass[1][i], sizeof(T)) == 0;
        written[i] = same ? 1 : 0;
        if (same) lab_out[i] = pass[0][i];
    }
    return 0;
}

// The block loop of IO::CartesianWriteHDF / CartesianReadHDF
// (IO/CartesianHDF.h:76-80, 182-186) over the reference's own Field2AOS /
// AOS2Field (IO/FieldAOS.h) on a reference grid holding `data` (ncomp
// arrays cstride apart, blocks bstride apart, each block dense with its own
// extent).  to_aos: fills buf; else reads buf into the grid and copies the
// grid back into data.  Returns the best seconds per pass over the blocks.
template <typename T, EntityType E, size_t RANK, typename F>
double fieldAOS(const int nb[3], const int cells[3], int face_dir, int ncomp, T *data, int64_t cstride,
                int64_t bstride, const int sb[3], const int se[3], F *buf, int to_aos, int threads, int reps)
{
    using G = Grid::Cartesian<T, Mesh, E, RANK>;
    using IR = typename Mesh::IndexRangeType;
    G grid(MIndex{nb[0], nb[1], nb[2]}, MIndex{cells[0], cells[1], cells[2]});
    auto comp = [&](size_t i, int c) -> T * {
        if constexpr (E == EntityType::Face) {
            return grid[i][(size_t)face_dir].getData();
        } else if constexpr (RANK == 0) {
            return grid[i].getData();
        } else {
            return grid[i][(size_t)c].getData();
        }
    };
    auto count = [&](size_t i) -> size_t {
        if constexpr (E == EntityType::Face) {
            return grid[i][(size_t)face_dir].getIndexRange().size();
        } else if constexpr (RANK == 0) {
            return grid[i].getIndexRange().size();
        } else {
            return grid[i][0].getIndexRange().size();
        }
    };
    for (size_t i = 0; i < grid.size(); ++i)
        for (int c = 0; c < ncomp; ++c)
            std::memcpy(comp(i, c), data + c * cstride + (int64_t)i * bstride, count(i) * sizeof(T));
    const IR span(MIndex{sb[0], sb[1], sb[2]}, MIndex{sb[0] + se[0], sb[1] + se[1], sb[2] + se[2]});
    const long nblk = (long)grid.size();
    double best = 1e30;
    for (int r = 0; r < (reps > 0 ? reps : 1); ++r) {
        const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(static)
        for (long i = 0; i < nblk; ++i) {
            if (to_aos) {
                IO::Field2AOS(grid[(size_t)i], span, buf, (size_t)(face_dir < 0 ? 0 : face_dir));
            } else if constexpr (E == EntityType::Face) {
                // AOSDriver<FaceContainer>::read (IO/FieldAOS.h:143-148) passes
                // the face field where the buffer goes and does not compile;
                // it means the scalar read of the direction's face field
                IO::AOS2Field(buf, span, grid[(size_t)i][(size_t)face_dir], (size_t)face_dir);
            } else {
                IO::AOS2Field(buf, span, grid[(size_t)i], (size_t)0);
            }
        }
        const auto t1 = std::chrono::steady_clock::now();
        const double sec = std::chrono::duration<double>(t1 - t0).count();
        best = sec < best ? sec : best;
    }
    if (!to_aos) {
        for (size_t i = 0; i < grid.size(); ++i)
            for (int c = 0; c < ncomp; ++c)
                std::memcpy(data + c * cstride + (int64_t)i * bstride, comp(i, c), count(i) * sizeof(T));
    }
    return best;
}

template <typename T, typename F>
double fieldAOSDispatch(const int nb[3], const int cells[3], int entity, int ncomp, T *data, int64_t cstride,
                        int64_t bstride, const int sb[3], const int se[3], F *buf, int to_aos, int threads,
                        int reps)
{
    if (entity == 0 && ncomp == 1)
        return fieldAOS<T, EntityType::Cell, 0, F>(nb, cells, -1, 1, data, cstride, bstride, sb, se, buf, to_aos,
                                                   threads, reps);
    if (entity == 0 && ncomp == 3)
        return fieldAOS<T, EntityType::Cell, 1, F>(nb, cells, -1, 3, data, cstride, bstride, sb, se, buf, to_aos,
                                                   threads, reps);
    if (entity == 1 && ncomp == 1)
        return fieldAOS<T, EntityType::Node, 0, F>(nb, cells, -1, 1, data, cstride, bstride, sb, se, buf, to_aos,
                                                   threads, reps);
    if (entity >= 2 && entity <= 4 && ncomp == 1)
        return fieldAOS<T, EntityType::Face, 0, F>(nb, cells, entity - 2, 1, data, cstride, bstride, sb, se, buf,
                                                   to_aos, threads, reps);
    return -1.0;
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
// entity: 1 node, 2..4 faces normal to x, y, z (cn_entity numbering)
int ref_lab_fill_entity_f64(const or_geom *g, int entity, const double *comp, const int32_t *bc_off,
                            const or_bc *bcs, int block, double *lab, uint8_t *written)
{
    if (entity == 1)
        return labFillEntity<double, EntityType::Node>(g, -1, comp, bc_off, bcs, block, lab, written);
    if (entity >= 2 && entity <= 4)
        return labFillEntity<double, EntityType::Face>(g, entity - 2, comp, bc_off, bcs, block, lab, written);
    return 1;
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

// FieldLab::loadData of every block of ncomp components (stencil (-lo, hi+1)
// in every direction, non-tensorial, per-component BC vectors): the
// reference's grids built once, one lab per thread, blocks
// schedule(dynamic, 1) as in test/UnitTests/Grid/CartesianTest.cpp:283-317.
// Returns the best seconds per sweep over reps.
double ref_lab_sweep_f64(const int nb[3], const int n[3], const double *comps, int64_t stride, int64_t cstride,
                         const int32_t *const *bc_off, const or_bc *const *bcs, int ncomp, int lo, int hi,
                         int nthreads, int reps)
{
    using R = RefGrid<double>;
    std::vector<std::unique_ptr<R>> g;
    for (int c = 0; c < ncomp; ++c) {
        g.emplace_back(new R(nb, n, comps + c * cstride, stride));
        g.back()->attach(bc_off ? bc_off[c] : nullptr, bcs ? bcs[c] : nullptr);
    }
    const int nbk = (int)g[0]->grid->size();
    double best = 1e300;
    for (int rep = 0; rep < (reps < 1 ? 1 : reps); ++rep) {
        const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel num_threads(nthreads)
        {
            typename R::Lab lab;
            const typename R::S s(-lo, hi + 1, false);
            lab.allocate(s, (*g[0]->grid)[0].getIndexRange());
#pragma omp for schedule(dynamic, 1) collapse(2)
            for (int c = 0; c < ncomp; ++c)
                for (int b = 0; b < nbk; ++b) g[c]->grid->loadLab((*g[c]->grid)[(size_t)b], lab);
        }
        const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        best = dt < best ? dt : best;
    }
    return best;
}

// Euler RHS (stage 0) / SSP-RK3 stage (1..3) of blocks [b0, b0+cnt) on the
// reference FieldLab; returns the best seconds over reps.
double ref_euler_stage_f64(const int nb[3], const int n[3], const double *Us, const double *Un,
                           double *out, int64_t stride, int64_t cstride,
                           const int32_t *const *bc_off, const or_bc *const *bcs, int stage,
                           double dt, double gamma, const double h[3], int nthreads, int b0,
                           int cnt, int reps)
{
    return eulerStage<double>(nb, n, Us, Un, out, stride, cstride, bc_off, bcs, stage, dt, gamma, h,
                              nthreads, b0, cnt, reps);
}

// Field2AOS / AOS2Field block loop on a reference grid.  entity: 0 cell,
// 1 node, 2..4 faces normal to x, y, z; ncomp 1 (rank 0) or 3 (rank-1
// cells); file_dtype 0 float, 1 double.  Returns the best seconds per pass,
// or -1 for an unsupported combination.
double ref_field_aos_f64(const int nb[3], const int cells[3], int entity, int ncomp, double *data, int64_t cstride,
                         int64_t bstride, const int sb[3], const int se[3], int file_dtype, void *buf, int to_aos,
                         int threads, int reps)
{
    if (file_dtype == 0)
        return fieldAOSDispatch<double, float>(nb, cells, entity, ncomp, data, cstride, bstride, sb, se,
                                               (float *)buf, to_aos, threads, reps);
    return fieldAOSDispatch<double, double>(nb, cells, entity, ncomp, data, cstride, bstride, sb, se,
                                            (double *)buf, to_aos, threads, reps);
}
double ref_field_aos_f32(const int nb[3], const int cells[3], int entity, int ncomp, float *data, int64_t cstride,
                         int64_t bstride, const int sb[3], const int se[3], int file_dtype, void *buf, int to_aos,
                         int threads, int reps)
{
    if (file_dtype == 0)
        return fieldAOSDispatch<float, float>(nb, cells, entity, ncomp, data, cstride, bstride, sb, se,
                                              (float *)buf, to_aos, threads, reps);
    return fieldAOSDispatch<float, double>(nb, cells, entity, ncomp, data, cstride, bstride, sb, se,
                                           (double *)buf, to_aos, threads, reps);
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
