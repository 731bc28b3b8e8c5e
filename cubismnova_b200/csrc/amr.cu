// amr.cu -- blocks of uneven sizes on two refinement levels: layout, level
// interface ghost fill, the fused Euler SSP-RK3 stage as one persistent launch
// per stage over a tile work list, the work-list/grid autotuner, and CUDA
// graph capture of whole steps.
#include "amr.cuh"
#include "cn_internal.h"
#include "euler_stage.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

namespace cn {
namespace amr {

// Euler tiles of AMR blocks: tile index -> (block, tile of 8^3 cells); a
// work item (a CTA's unit of work) is a run of consecutive tiles of the list
struct Src {
    // a level-interface ghost cell resolves its geometry once for all five
    // components (halo5)
    static constexpr bool kHalo5 = true;
    Geom A;
    const int2 *work;  // tiles: (block, tile index in the block)
    const int2 *items; // work items: (first tile, tile count)
    template <typename T> __device__ __forceinline__ void tile(int item, euler::TileInfo<T> &t) const
    {
        const int2 w = work[item];
        const BlockDev B = A.blk[w.x];
        const int tpd = B.n / 8;
        t.block = w.x;
        t.x0 = (w.y % tpd) * 8;
        t.y0 = ((w.y / tpd) % tpd) * 8;
        t.z0 = (w.y / (tpd * tpd)) * 8;
        t.N0 = t.N1 = t.N2 = B.n;
        t.boff = B.off;
        t.ih[0] = t.ih[1] = t.ih[2] = (T)B.ih;
        t.bx = t.by = t.bz = 0;
    }
    template <typename T> __device__ __forceinline__ void prepare(const euler::TileInfo<T> &, int *) const {}
    // a ghost from a block on the same level is a plain copy of its cell;
    // level-interface ghosts (prolongation, restriction) take halo()
    template <typename T>
    __device__ __forceinline__ bool plain_offset(const euler::TileInfo<T> &t, int gx, int gy, int gz, const int *,
                                                 int64_t &off) const
    {
        return same_level_offset(A, t.block, gx, gy, gz, off);
    }
    // all five components of a level-interface ghost: the geometry once
    template <typename T>
    __device__ __forceinline__ void halo5(const T *const (&U)[5], const euler::TileInfo<T> &t, int gx, int gy, int gz,
                                          const int *, T (&v)[5]) const
    {
        const Ghost g = resolve(A, t.block, gx, gy, gz);
#pragma unroll 1
        for (int c = 0; c < 5; ++c) v[c] = gather<T>(U[c], g);
    }
};

// ONE: one CTA per work item of a single tile (the schedule of one CTA per
// item with 1x1x1 work tiles): no loop around the tile, which leaves the
// compiler the registers the loops' state takes (FP64: 52 instead of 308
// bytes of spill stores per thread).  Otherwise persistent: each CTA walks
// the work items with a grid stride, the tiles of an item in order.
template <typename T, bool ONE>
__global__ void __launch_bounds__(euler::NT, 3) stage_kernel(euler::StageParams<T> p, Src src, int nitems)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T *W = reinterpret_cast<T *>(smem_raw);
    T *A = W + 5 * euler::Stg<T>::SV;
    __shared__ double red[euler::NT / 32][5];
    __shared__ int snb[28];
    __shared__ euler::TileInfo<T> ts;
    if constexpr (ONE) {
        const int tile = src.items[blockIdx.x].x;
        euler::stage_tile<T>(p, src, tile, tile, W, A, red, snb, &ts);
    } else {
        for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
            const int2 it = src.items[item];
            for (int k = 0; k < it.y; ++k)
                euler::stage_tile<T>(p, src, it.x + k, it.x + k, W, A, red, snb, &ts);
        }
    }
}

// dense lab of one block: (n+2g)^3, face ghosts only (non-tensorial)
template <typename T>
__global__ void __launch_bounds__(256) lab_kernel(const T *comp, Geom A, int b, int g, T *out)
{
    const BlockDev B = A.blk[b];
    const int E = B.n + 2 * g;
    const int64_t total = (int64_t)E * E * E;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(t % E) - g, y = (int)((t / E) % E) - g, z = (int)(t / ((int64_t)E * E)) - g;
        const int outside = (x < 0 || x >= B.n) + (y < 0 || y >= B.n) + (z < 0 || z >= B.n);
        if (outside > 1) continue;
        out[t] = value<T>(comp, A, b, x, y, z);
    }
}

} // namespace amr
} // namespace cn

using namespace cn;
using namespace cn::amr;

struct cn_amr {
    int nblocks = 0, L[3] = {0, 0, 0}, lr[3] = {0, 0, 0}, ncomp = 0;
    cn_dtype dtype = CN_FLOAT64;
    size_t es = 8;
    std::vector<BlockDev> blocks;
    int64_t total_cells = 0, comp_stride = 0;
    BlockDev *d_blocks = nullptr;
    int32_t *d_lookup = nullptr;
    void *d_data = nullptr;
    std::vector<int2> work;   // tiles in work-list order
    std::vector<int2> items;  // work items: (first tile, tile count)
    int2 *d_work = nullptr, *d_items = nullptr;
    int order = 1;   // work-list order (see cn_amr_set_schedule)
    int ctas = 0;    // persistent grid size (0: one CTA per item)
    int shape[3] = {1, 1, 1}; // work tile: 8^3 tiles per work item along x, y, z (cn_amr_set_work_shape)
};

static uint64_t spread3(uint32_t v)
{
    uint64_t x = v & 0x1fffff;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}

// Work list: each block cut into work tiles of up to shape[0] x shape[1] x
// shape[2] 8^3 tiles (clipped to the block), one work item per work tile,
// its tiles emitted x fastest; items ordered by the schedule's key of their
// first tile.
static cn_status build_work(cn_amr *a)
{
    struct Unit {
        int block, first, count, n; // tiles [first, first + count) of `tiles`
        uint64_t key;
    };
    std::vector<Unit> units;
    std::vector<int> tiles;
    for (int b = 0; b < a->nblocks; ++b) {
        const BlockDev &B = a->blocks[b];
        const int tpd = B.n / 8, cs = B.level == 0 ? 2 : 1;
        int u[3];
        for (int d = 0; d < 3; ++d) u[d] = a->shape[d] < tpd ? a->shape[d] : tpd;
        for (int bz = 0; bz < tpd; bz += u[2])
            for (int by = 0; by < tpd; by += u[1])
                for (int bx = 0; bx < tpd; bx += u[0]) {
                    const int first = (int)tiles.size();
                    for (int tz = bz; tz < bz + u[2]; ++tz)
                        for (int ty = by; ty < by + u[1]; ++ty)
                            for (int tx = bx; tx < bx + u[0]; ++tx) tiles.push_back(tx + tpd * (ty + tpd * tz));
                    const uint32_t X = (uint32_t)(B.ox + bx * 8 * cs), Y = (uint32_t)(B.oy + by * 8 * cs),
                                   Z = (uint32_t)(B.oz + bz * 8 * cs);
                    units.push_back({b, first, (int)tiles.size() - first, B.n,
                                     spread3(X) | spread3(Y) << 1 | spread3(Z) << 2});
                }
    }
    if (a->order == 1) {
        std::stable_sort(units.begin(), units.end(), [](const Unit &l, const Unit &r) { return l.n > r.n; });
    } else if (a->order == 2) {
        std::stable_sort(units.begin(), units.end(), [](const Unit &l, const Unit &r) { return l.key < r.key; });
    }
    a->work.clear();
    a->items.clear();
    for (const Unit &u : units) {
        a->items.push_back(make_int2((int)a->work.size(), u.count));
        for (int k = 0; k < u.count; ++k) a->work.push_back(make_int2(u.block, tiles[u.first + k]));
    }
    if (a->d_work) cudaFree(a->d_work);
    if (a->d_items) cudaFree(a->d_items);
    a->d_work = a->d_items = nullptr;
    CN_CUDA_TRY(cudaMalloc(&a->d_work, sizeof(int2) * a->work.size()));
    CN_CUDA_TRY(cudaMemcpy(a->d_work, a->work.data(), sizeof(int2) * a->work.size(), cudaMemcpyHostToDevice));
    CN_CUDA_TRY(cudaMalloc(&a->d_items, sizeof(int2) * a->items.size()));
    CN_CUDA_TRY(cudaMemcpy(a->d_items, a->items.data(), sizeof(int2) * a->items.size(), cudaMemcpyHostToDevice));
    return CN_OK;
}

static Geom geom(const cn_amr *a)
{
    Geom g;
    g.blk = a->d_blocks;
    g.lookup = a->d_lookup;
    for (int d = 0; d < 3; ++d) {
        g.L[d] = a->L[d];
        g.lr[d] = a->lr[d];
    }
    return g;
}

template <typename T, bool ONE> static cn_status set_smem_once()
{
    static DeviceOnce once; // per device
    const size_t smem = (size_t)(5 * euler::Stg<T>::SV + 5 * euler::NACC) * sizeof(T);
    return smem_opt_in(once, amr::stage_kernel<T, ONE>, smem);
}

template <typename T>
static cn_status launch_amr_stage(cn_amr *Us, cn_amr *Un, cn_amr *out, int stage, double dt, double gamma,
                                  cudaStream_t st)
{
    // one CTA per single-tile item: the loop-free kernel
    const bool one = Us->ctas == 0 && Us->shape[0] * Us->shape[1] * Us->shape[2] == 1;
    cn_status s = one ? set_smem_once<T, true>() : set_smem_once<T, false>();
    if (s != CN_OK) return s;
    euler::StageParams<T> p = {};
    for (int c = 0; c < 5; ++c) {
        p.U[c] = reinterpret_cast<const T *>(Us->d_data) + (size_t)c * Us->comp_stride;
        p.Un[c] = Un ? reinterpret_cast<const T *>(Un->d_data) + (size_t)c * Un->comp_stride : nullptr;
        p.out[c] = reinterpret_cast<T *>(out->d_data) + (size_t)c * out->comp_stride;
    }
    p.dt = (T)dt;
    p.gamma = (T)gamma;
    p.gm1 = (T)(gamma - 1.0);
    p.igm1 = (T)(1.0 / (gamma - 1.0));
    p.stage = stage;
    p.partials = nullptr;
    Src src;
    src.A = geom(Us);
    src.work = Us->d_work;
    src.items = Us->d_items;
    const int nitems = (int)Us->items.size();
    int grid = Us->ctas > 0 ? std::min(Us->ctas, nitems) : nitems;
    const size_t smem = (size_t)(5 * euler::Stg<T>::SV + 5 * euler::NACC) * sizeof(T);
    if (one)
        amr::stage_kernel<T, true><<<nitems, euler::NT, smem, st>>>(p, src, nitems);
    else
        amr::stage_kernel<T, false><<<grid, euler::NT, smem, st>>>(p, src, nitems);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

static bool same_layout(const cn_amr *a, const cn_amr *b)
{
    return a && b && a->nblocks == b->nblocks && a->comp_stride == b->comp_stride && a->dtype == b->dtype &&
           a->ncomp >= 5 && b->ncomp >= 5;
}

struct cn_graph {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t x = nullptr;
};

extern "C" {

cn_status cn_amr_create_box(int nblocks, const int *level, const int *cells, const int *origin,
                            const int fine_extent[3], int ncomp, cn_dtype dtype, cn_amr **out)
{
    if (!out || !level || !cells || !origin || !fine_extent || nblocks < 1 || ncomp < 1)
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_amr_create: bad argument");
    *out = nullptr;
    if (dtype != CN_FLOAT64 && dtype != CN_FLOAT32)
        return fail(CN_ERR_UNSUPPORTED, "cn_amr_create: dtype must be FLOAT32 or FLOAT64");
    for (int d = 0; d < 3; ++d)
        if (fine_extent[d] < 8 || fine_extent[d] % 8)
            return fail(CN_ERR_INVALID_ARGUMENT, "cn_amr_create: the extent must be a multiple of 8 level-1 cells");
    cn_amr *a = new cn_amr();
    a->nblocks = nblocks;
    for (int d = 0; d < 3; ++d) {
        a->L[d] = fine_extent[d];
        a->lr[d] = fine_extent[d] / 8;
    }
    a->ncomp = ncomp;
    a->dtype = dtype;
    a->es = dtype == CN_FLOAT64 ? 8 : 4;
    std::vector<int32_t> lookup((size_t)a->lr[0] * a->lr[1] * a->lr[2], -1);
    int64_t off = 0;
    for (int b = 0; b < nblocks; ++b) {
        BlockDev B;
        B.level = level[b];
        B.n = cells[b];
        B.ox = origin[3 * b];
        B.oy = origin[3 * b + 1];
        B.oz = origin[3 * b + 2];
        B.pad = 0;
        B.off = off;
        const int cs = B.level == 0 ? 2 : 1;
        B.ih = (double)fine_extent[0] / cs; // cubic cells: h = cs / Lx (the box is [0,1] x [0,Ly/Lx] x [0,Lz/Lx])
        if ((B.level != 0 && B.level != 1) || B.n < 8 || B.n % 8 || B.ox % 8 || B.oy % 8 || B.oz % 8 || B.ox < 0 ||
            B.oy < 0 || B.oz < 0 || B.ox + B.n * cs > fine_extent[0] || B.oy + B.n * cs > fine_extent[1] ||
            B.oz + B.n * cs > fine_extent[2]) {
            delete a;
            return fail(CN_ERR_INVALID_ARGUMENT, "cn_amr_create: block level, cells or origin out of range");
        }
        const int span = B.n * cs / 8;
        for (int k = 0; k < span; ++k)
            for (int j = 0; j < span; ++j)
                for (int i = 0; i < span; ++i) {
                    int32_t &e = lookup[(B.ox / 8 + i) + (size_t)a->lr[0] * ((B.oy / 8 + j) + (size_t)a->lr[1] * (B.oz / 8 + k))];
                    if (e != -1) {
                        delete a;
                        return fail(CN_ERR_INVALID_ARGUMENT, "cn_amr_create: blocks overlap");
                    }
                    e = b;
                }
        a->blocks.push_back(B);
        off += (int64_t)B.n * B.n * B.n;
    }
    for (int32_t e : lookup)
        if (e < 0) {
            delete a;
            return fail(CN_ERR_INVALID_ARGUMENT, "cn_amr_create: blocks do not cover the domain");
        }
    a->total_cells = off;
    a->comp_stride = off;
    cudaError_t e = cudaMalloc(&a->d_blocks, sizeof(BlockDev) * nblocks);
    if (e == cudaSuccess) e = cudaMemcpy(a->d_blocks, a->blocks.data(), sizeof(BlockDev) * nblocks, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&a->d_lookup, sizeof(int32_t) * lookup.size());
    if (e == cudaSuccess)
        e = cudaMemcpy(a->d_lookup, lookup.data(), sizeof(int32_t) * lookup.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&a->d_data, a->es * (size_t)a->comp_stride * ncomp);
    if (e == cudaSuccess) e = cudaMemset(a->d_data, 0, a->es * (size_t)a->comp_stride * ncomp);
    cn_status s = e == cudaSuccess ? build_work(a) : cuda_fail(e, "cn_amr_create");
    if (s != CN_OK) {
        extern cn_status cn_amr_destroy(cn_amr *);
        cn_amr_destroy(a);
        return s;
    }
    *out = a;
    return CN_OK;
}

cn_status cn_amr_create(int nblocks, const int *level, const int *cells, const int *origin, int fine_extent,
                        int ncomp, cn_dtype dtype, cn_amr **out)
{
    const int e[3] = {fine_extent, fine_extent, fine_extent};
    return cn_amr_create_box(nblocks, level, cells, origin, e, ncomp, dtype, out);
}

cn_status cn_amr_destroy(cn_amr *a)
{
    if (!a) return CN_OK;
    if (a->d_blocks) cudaFree(a->d_blocks);
    if (a->d_lookup) cudaFree(a->d_lookup);
    if (a->d_data) cudaFree(a->d_data);
    if (a->d_work) cudaFree(a->d_work);
    if (a->d_items) cudaFree(a->d_items);
    delete a;
    return CN_OK;
}

cn_status cn_amr_info(const cn_amr *a, int64_t *total_cells, int64_t *comp_stride, int *nitems)
{
    if (!a) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    if (total_cells) *total_cells = a->total_cells;
    if (comp_stride) *comp_stride = a->comp_stride;
    if (nitems) *nitems = (int)a->work.size();
    return CN_OK;
}

cn_status cn_amr_block_offset(const cn_amr *a, int block, int64_t *off)
{
    if (!a || !off || block < 0 || block >= a->nblocks) return fail(CN_ERR_INVALID_ARGUMENT, "bad block");
    *off = a->blocks[block].off;
    return CN_OK;
}

cn_status cn_amr_data(cn_amr *a, int comp, void **ptr)
{
    if (!a || !ptr || comp < 0 || comp >= a->ncomp) return fail(CN_ERR_INVALID_ARGUMENT, "bad component");
    *ptr = (char *)a->d_data + a->es * (size_t)a->comp_stride * comp;
    return CN_OK;
}

cn_status cn_amr_lab_fill(cn_amr *a, int comp, int ghost, int block, void *d_lab, void *stream)
{
    if (!a || !d_lab || comp < 0 || comp >= a->ncomp || block < 0 || block >= a->nblocks)
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_amr_lab_fill: bad argument");
    if (ghost < 0 || ghost > 8) return fail(CN_ERR_STENCIL_TOO_WIDE, "cn_amr_lab_fill: ghost width must be <= 8");
    const Geom g = geom(a);
    cudaStream_t st = as_stream(stream);
    const int E = a->blocks[block].n + 2 * ghost;
    const unsigned grid = (unsigned)std::min<int64_t>(((int64_t)E * E * E + 255) / 256, 148 * 8);
    if (a->dtype == CN_FLOAT64) {
        const double *c = reinterpret_cast<const double *>(a->d_data) + (size_t)comp * a->comp_stride;
        amr::lab_kernel<double><<<grid, 256, 0, st>>>(c, g, block, ghost, reinterpret_cast<double *>(d_lab));
    } else {
        const float *c = reinterpret_cast<const float *>(a->d_data) + (size_t)comp * a->comp_stride;
        amr::lab_kernel<float><<<grid, 256, 0, st>>>(c, g, block, ghost, reinterpret_cast<float *>(d_lab));
    }
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

// One SSP-RK3 stage (stage 0: out = L(Us)) of the Euler equations on an AMR
// layout, periodic box, one persistent launch over the tile work list.
cn_status cn_amr_rk3_stage(cn_amr *Us, cn_amr *Un, cn_amr *out, int stage, double dt, double gamma, void *stream)
{
    if (stage < 0 || stage > 3) return fail(CN_ERR_INVALID_ARGUMENT, "stage must be 0..3");
    if (!same_layout(Us, out) || (stage > 1 && !same_layout(Us, Un)))
        return fail(CN_ERR_SIZE_MISMATCH, "Cartesian: Can not assign two grids of unequal size.");
    cudaStream_t st = as_stream(stream);
    if (Us->dtype == CN_FLOAT64) return launch_amr_stage<double>(Us, stage > 1 ? Un : nullptr, out, stage, dt, gamma, st);
    return launch_amr_stage<float>(Us, stage > 1 ? Un : nullptr, out, stage, dt, gamma, st);
}

cn_status cn_amr_rk3_step(cn_amr *U, cn_amr *w1, cn_amr *w2, double dt, double gamma, void *stream)
{
    cn_status s;
    if ((s = cn_amr_rk3_stage(U, nullptr, w1, 1, dt, gamma, stream)) != CN_OK) return s;
    if ((s = cn_amr_rk3_stage(w1, U, w2, 2, dt, gamma, stream)) != CN_OK) return s;
    return cn_amr_rk3_stage(w2, U, U, 3, dt, gamma, stream);
}

// Work-list order (0: block order, 1: largest blocks first, 2: Morton order
// of tile positions) and persistent grid size (0: one CTA per work item).
// Every layout sharing a step should use the same schedule (the stage
// kernels take the schedule of the state they read).
cn_status cn_amr_set_schedule(cn_amr *a, int order, int ctas)
{
    if (!a || order < 0 || order > 2 || ctas < 0) return fail(CN_ERR_INVALID_ARGUMENT, "bad schedule");
    a->ctas = ctas;
    if (order != a->order) {
        a->order = order;
        return build_work(a);
    }
    return CN_OK;
}

// Work tile of a CTA's work item: shape[d] in {1, 2, 4} 8^3 tiles along d
// (8x8x8 up to 32x32x32 cells, clipped to the block).
cn_status cn_amr_set_work_shape(cn_amr *a, const int shape[3])
{
    if (!a || !shape) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    for (int d = 0; d < 3; ++d)
        if (shape[d] != 1 && shape[d] != 2 && shape[d] != 4) return fail(CN_ERR_INVALID_ARGUMENT, "bad work shape");
    if (shape[0] != a->shape[0] || shape[1] != a->shape[1] || shape[2] != a->shape[2]) {
        for (int d = 0; d < 3; ++d) a->shape[d] = shape[d];
        return build_work(a);
    }
    return CN_OK;
}

// 1, 2 or 4 consecutive tiles along x: the work shape (tiles, 1, 1)
cn_status cn_amr_set_work_unit(cn_amr *a, int tiles)
{
    if (!a || (tiles != 1 && tiles != 2 && tiles != 4)) return fail(CN_ERR_INVALID_ARGUMENT, "bad work unit");
    const int shape[3] = {tiles, 1, 1};
    return cn_amr_set_work_shape(a, shape);
}

cn_status cn_amr_get_work_shape(const cn_amr *a, int shape[3])
{
    if (!a || !shape) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    for (int d = 0; d < 3; ++d) shape[d] = a->shape[d];
    return CN_OK;
}

cn_status cn_amr_get_schedule(const cn_amr *a, int out[3])
{
    if (!a || !out) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    out[0] = a->order;
    out[1] = a->ctas;
    out[2] = a->shape[0] * a->shape[1] * a->shape[2];
    return CN_OK;
}

// Times every schedule candidate (orders 0..2; work tiles of 1x1x1, 2x1x1,
// 4x1x1, 1x2x1, 1x1x2, 2x2x1 and 2x2x2 8^3 tiles; grid = k x SMs x 3 CTAs
// for k in {1, 2, 4} or one CTA per work item) over `reps` RK3 steps and
// keeps the fastest on all three layouts.  U is advanced by the trial steps.
cn_status cn_amr_autotune(cn_amr *U, cn_amr *w1, cn_amr *w2, double dt, double gamma, int reps, int *order_out,
                          int *ctas_out, double *ms_out, void *stream)
{
    if (!same_layout(U, w1) || !same_layout(U, w2)) return fail(CN_ERR_SIZE_MISMATCH, "layouts differ");
    cudaStream_t st = as_stream(stream);
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grids[4] = {0, sms * 3, sms * 6, sms * 12};
    const int shapes[7][3] = {{1, 1, 1}, {2, 1, 1}, {4, 1, 1}, {1, 2, 1}, {1, 1, 2}, {2, 2, 1}, {2, 2, 2}};
    double best = 1e300;
    int bo = 1, bc = 0, bs = 0;
    cudaEvent_t e0, e1;
    CN_CUDA_TRY(cudaEventCreate(&e0));
    CN_CUDA_TRY(cudaEventCreate(&e1));
    for (int si = 0; si < 7; ++si)
        for (int order = 0; order < 3; ++order)
            for (int gi = 0; gi < 4; ++gi) {
                cn_status s;
                cn_amr *all[3] = {U, w1, w2};
                for (cn_amr *a : all) {
                    if ((s = cn_amr_set_work_shape(a, shapes[si])) != CN_OK) return s;
                    if ((s = cn_amr_set_schedule(a, order, grids[gi])) != CN_OK) return s;
                }
                if ((s = cn_amr_rk3_step(U, w1, w2, dt, gamma, stream)) != CN_OK) return s; // warm-up
                CN_CUDA_TRY(cudaEventRecord(e0, st));
                for (int r = 0; r < (reps < 1 ? 1 : reps); ++r)
                    if ((s = cn_amr_rk3_step(U, w1, w2, dt, gamma, stream)) != CN_OK) return s;
                CN_CUDA_TRY(cudaEventRecord(e1, st));
                CN_CUDA_TRY(cudaEventSynchronize(e1));
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                ms /= (reps < 1 ? 1 : reps);
                if (ms < best) {
                    best = ms;
                    bo = order;
                    bc = grids[gi];
                    bs = si;
                }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cn_amr *all[3] = {U, w1, w2};
    for (cn_amr *a : all) {
        cn_status s = cn_amr_set_work_shape(a, shapes[bs]);
        if (s == CN_OK) s = cn_amr_set_schedule(a, bo, bc);
        if (s != CN_OK) return s;
    }
    if (order_out) *order_out = bo;
    if (ctas_out) *ctas_out = bc;
    if (ms_out) *ms_out = best;
    return CN_OK;
}

// ------------------------------------------------------------ CUDA graphs
// Captures the work issued on `stream` between begin and end into an
// executable graph (thread-local capture mode).  Kernels of the captured
// calls must have been run once before (first use sets kernel attributes),
// and grids' BC tables must be synchronised (cn_bc_sync) before capture.
cn_status cn_graph_begin(void *stream)
{
    CN_CUDA_TRY(cudaStreamBeginCapture(as_stream(stream), cudaStreamCaptureModeThreadLocal));
    return CN_OK;
}

cn_status cn_graph_end(void *stream, cn_graph **out)
{
    if (!out) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    cn_graph *g = new cn_graph();
    cudaError_t e = cudaStreamEndCapture(as_stream(stream), &g->g);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&g->x, g->g, 0);
    if (e != cudaSuccess) {
        if (g->g) cudaGraphDestroy(g->g);
        delete g;
        return cuda_fail(e, "cn_graph_end");
    }
    *out = g;
    return CN_OK;
}

cn_status cn_graph_launch(cn_graph *g, void *stream)
{
    if (!g) return fail(CN_ERR_INVALID_ARGUMENT, "NULL graph");
    CN_CUDA_TRY(cudaGraphLaunch(g->x, as_stream(stream)));
    return CN_OK;
}

cn_status cn_graph_destroy(cn_graph *g)
{
    if (!g) return CN_OK;
    if (g->x) cudaGraphExecDestroy(g->x);
    if (g->g) cudaGraphDestroy(g->g);
    delete g;
    return CN_OK;
}

} // extern "C"
