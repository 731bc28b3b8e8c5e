// mg_tile.cuh -- tiles of a block for the level operators of the multigrid
// solver and the learned smoother's features: tile geometry, asynchronous
// staging of a tile plus its one-cell halo into shared memory, and the
// variable-coefficient 7-point operator evaluated from the staged region.
#pragma once

#include "cn_fastdiv.h"
#include "cn_internal.h"
#include "cn_tma.cuh"

namespace cn {
namespace mg {

template <typename T> __device__ __forceinline__ T harm(T a, T b)
{
    const T t = a * b;
    return (t + t) / (a + b);
}

// L p and the diagonal D at one cell from its 13 values; TP is the solution
// type (float in the V-cycle, double in the outer residual), k is FP32.
template <typename TP>
__device__ __forceinline__ void op7_math(const TP (&v)[14], TP ih2, TP &Lp, TP &D, TP &pc)
{
    pc = v[0];
    const TP kc = v[1];
    TP f[3], s[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const TP pp = v[2 + 4 * d], pm = v[3 + 4 * d];
        const TP kp = harm<TP>(kc, v[4 + 4 * d]);
        const TP km = harm<TP>(v[5 + 4 * d], kc);
        f[d] = kp * (pp - pc) - km * (pc - pm);
        s[d] = kp + km;
    }
    Lp = ih2 * ((f[0] + f[1]) + f[2]);
    D = ih2 * ((s[0] + s[1]) + s[2]);
}

// Operator coefficients of a level, precomputed once from k (they depend on
// k only): per cell 8 contiguous values, the harmonic face means
// kp_d = harm(k, k(+e_d)) (d = x, y, z), km_d = harm(k(-e_d), k) (neighbours
// through the lab), the diagonal D = ih2 ((s0 + s1) + s2) with
// s_d = kp_d + km_d, and a zero pad, so one cell's set is two (FP32) or four
// (FP64) 16-byte loads.  Cell (block b, dense in-block index c) at
// (b cells_per_block + c) * 8.  Evaluated with the same operations as
// op7_math, so L p and D come out bit for bit the same.
constexpr int kCoefPerCell = 8;

template <typename TC> __device__ __forceinline__ void load_coef8(const TC *cv, TC (&c)[8])
{
    if constexpr (sizeof(TC) == 4) {
        const float4 a = __ldg(reinterpret_cast<const float4 *>(cv)), b = __ldg(reinterpret_cast<const float4 *>(cv) + 1);
        c[0] = a.x; c[1] = a.y; c[2] = a.z; c[3] = a.w;
        c[4] = b.x; c[5] = b.y; c[6] = b.z; c[7] = b.w;
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const double2 v = __ldg(reinterpret_cast<const double2 *>(cv) + i);
            c[2 * i] = v.x;
            c[2 * i + 1] = v.y;
        }
    }
}

template <typename TP, typename TC>
__device__ __forceinline__ void op7_coef(const TP *sp, int u, const int (&st)[3], const TC *cv, TP ih2, TP &Lp,
                                         TP &D, TP &pc)
{
    TC c[8];
    load_coef8<TC>(cv, c);
    pc = sp[u];
    TP f[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const TP kp = (TP)c[d], km = (TP)c[3 + d];
        f[d] = kp * (sp[u + st[d]] - pc) - km * (pc - sp[u - st[d]]);
    }
    Lp = ih2 * ((f[0] + f[1]) + f[2]);
    D = (TP)c[6];
}

// ---------------------------------------------------------------- tiles
// The level operators work on tiles of one block: up to 32 x 8 x 4 cells
// (extents: the largest divisors of the block's cells within those caps,
// even when the block's extent is even, so fine tiles hold whole coarse
// cells).  A CTA stages its tile plus a one-cell halo of p and k into shared
// memory (halo cells outside the block through cn::lab_fetch: periodic
// neighbour or the BC chain), then every thread evaluates its cells from
// shared memory with the same operation order as the per-cell form.
struct Tile {
    int t[3];      // tile extent (cells)
    int per[3];    // tiles per block along x, y, z
    int count;     // tiles per block
    int sh[2];     // log2 of t[0], t[1] when powers of two, else -1
    int zs;        // z groups: threads take (x, y) columns, split into zs runs along z
    FastDiv dv_count, dv_per0, dv_per1; // CTA index -> (block, tile) without divisions
};

constexpr int kTileCap[3] = {32, 8, 4};
// staged region: tile + one-cell halo; rows padded to t0 + 8 entries so that
// the in-block part of a row starts 16-byte aligned (vector staging)
constexpr int kRegionMax = (32 + 8) * (8 + 2) * (4 + 2); // 2400
constexpr int kTileThreads = 256;
constexpr int kTileMinCtas = 6; // resident CTAs per SM the tile kernels are compiled for (<= 40 registers)

inline int tile_extent(int n, int cap)
{
    for (int t = n < cap ? n : cap; t >= 1; --t)
        if (n % t == 0 && (n % 2 != 0 || t % 2 == 0 || t == 1))
            return t;
    return 1;
}

inline Tile tile_of(const int n[3])
{
    Tile T;
    T.count = 1;
    for (int d = 0; d < 3; ++d) {
        T.t[d] = tile_extent(n[d], kTileCap[d]);
        T.per[d] = n[d] / T.t[d];
        T.count *= T.per[d];
    }
    for (int d = 0; d < 2; ++d) {
        T.sh[d] = -1;
        for (int b = 0; b < 31; ++b)
            if (T.t[d] == (1 << b)) T.sh[d] = b;
    }
    T.dv_count = FastDiv((uint32_t)T.count);
    T.dv_per0 = FastDiv((uint32_t)T.per[0]);
    T.dv_per1 = FastDiv((uint32_t)T.per[1]);
    const int cols = T.t[0] * T.t[1];
    T.zs = 1;
    for (int g = T.t[2]; g >= 1; --g)
        if (T.t[2] % g == 0 && g * cols <= kTileThreads) {
            T.zs = g;
            break;
        }
    return T;
}

// This thread's run of cells: column (x, y) of the tile and z0 .. z0+zl-1;
// false for threads without work (more threads than columns x z groups).
__device__ __forceinline__ bool column_run(const Tile &T, int &x, int &y, int &z0, int &zl)
{
    const int cols = T.t[0] * T.t[1];
    const int g = threadIdx.x / cols, col = threadIdx.x - g * cols;
    if (g >= T.zs) return false;
    if (T.sh[0] >= 0) {
        x = col & (T.t[0] - 1);
        y = col >> T.sh[0];
    } else {
        x = col % T.t[0];
        y = col / T.t[0];
    }
    zl = T.t[2] / T.zs;
    z0 = g * zl;
    return true;
}

// tile-local cell c -> (x, y, z)
__device__ __forceinline__ void tile_cell(const Tile &T, int c, int &x, int &y, int &z)
{
    if (T.sh[0] >= 0 && T.sh[1] >= 0) {
        x = c & (T.t[0] - 1);
        y = (c >> T.sh[0]) & (T.t[1] - 1);
        z = c >> (T.sh[0] + T.sh[1]);
    } else {
        x = c % T.t[0];
        y = (c / T.t[0]) % T.t[1];
        z = c / (T.t[0] * T.t[1]);
    }
}

struct TilePos {
    int block, x0, y0, z0;
    int ex, ey, ez; // staged region extents (tile + 2)
    int xo, rs;     // region row: position of cell x = 0, row stride
};

// region index of tile-local cell (x, y, z), x in [-1, t0], y, z in [-1, t]
__device__ __forceinline__ int ridx(const TilePos &q, int x, int y, int z)
{
    return (x + q.xo) + q.rs * ((y + 1) + q.ey * (z + 1));
}

__device__ __forceinline__ TilePos tile_pos(const Tile &T)
{
    TilePos q;
    q.block = T.dv_count.div((int)blockIdx.x);
    const int r = blockIdx.x - q.block * T.count;
    const int ry = T.dv_per0.div(r), rz = T.dv_per1.div(ry);
    q.x0 = (r - ry * T.per[0]) * T.t[0];
    q.y0 = (ry - rz * T.per[1]) * T.t[1];
    q.z0 = rz * T.t[2];
    q.ex = T.t[0] + 2;
    q.ey = T.t[1] + 2;
    q.ez = T.t[2] + 2;
    q.xo = 1;
    q.rs = q.ex;
    return q;
}

// Vector layout for a field of T on geometry L when the tile's rows allow it:
// in-block row segments start 16-byte aligned in global and shared memory.
template <typename T> __device__ __forceinline__ void region_layout(TilePos &q, const LabGeom &L)
{
    constexpr int V = 16 / (int)sizeof(T);
    const int t0 = q.ex - 2;
    if (t0 % V == 0 && L.n[0] % V == 0 && L.bstride % V == 0 && q.x0 % V == 0) {
        q.xo = V;
        q.rs = t0 + 2 * V;
    }
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// The 27 periodic neighbour blocks of block b (itself included), index
// (r0+1) + 3 (r1+1) + 9 (r2+1) for the offsets r in {-1, 0, 1}^3, written to
// shared memory by the first 27 threads; a barrier must follow.
__device__ __forceinline__ void neighbour_blocks(const int nb[3], int b, int *snb)
{
    if (threadIdx.x < 27) {
        const int t = threadIdx.x;
        int bx = b % nb[0] + t % 3 - 1, by = (b / nb[0]) % nb[1] + (t / 3) % 3 - 1, bz = b / (nb[0] * nb[1]) + t / 9 - 1;
        bx = bx < 0 ? bx + nb[0] : (bx >= nb[0] ? bx - nb[0] : bx);
        by = by < 0 ? by + nb[1] : (by >= nb[1] ? by - nb[1] : by);
        bz = bz < 0 ? bz + nb[2] : (bz >= nb[2] ? bz - nb[2] : bz);
        snb[t] = bx + nb[0] * (by + nb[1] * bz);
    }
}

// Stage one field over the region.  Cells inside the block, and outside it
// in blocks without BCs or skip flags (the periodic neighbour, from the
// table snb of neighbour_blocks), are asynchronous copies: 16-byte chunks of
// the in-block row segments in the vector layout (region_layout), single
// cells otherwise; cells of blocks with BCs resolve through the lab
// (cn::lab_fetch_slow).  Edge and corner cells of the region are zero unless
// tensorial (the 7-point operator does not read them).  The caller waits with
// cp_async_wait_all() and a barrier.
template <typename T>
__device__ __forceinline__ void stage_cell(const T *comp, const LabGeom &L, const BcView &bc, const TilePos &q,
                                           bool tensorial, const int *snb, bool plain, int x, int y, int z, T *dst)
{
    const int r0 = x < 0 ? -1 : (x >= L.n[0] ? 1 : 0), r1 = y < 0 ? -1 : (y >= L.n[1] ? 1 : 0),
              r2 = z < 0 ? -1 : (z >= L.n[2] ? 1 : 0);
    const int outside = (r0 != 0) + (r1 != 0) + (r2 != 0);
    if (!tensorial && outside > 1) {
        *dst = T(0);
    } else if (outside == 0 || plain) {
        const int sb = outside == 0 ? q.block : snb[(r0 + 1) + 3 * (r1 + 1) + 9 * (r2 + 1)];
        const T *src = comp + (int64_t)sb * L.bstride + (x - r0 * L.n[0]) +
                       (int64_t)L.n[0] * ((y - r1 * L.n[1]) + (int64_t)L.n[1] * (z - r2 * L.n[2]));
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"((int)sizeof(T))
                     : "memory");
    } else {
        *dst = lab_fetch_slow<T>(comp, L, bc, q.block, x, y, z);
    }
}

template <typename T>
__device__ __forceinline__ void stage_region(const T *comp, const LabGeom &L, const BcView &bc, const TilePos &q,
                                             bool tensorial, const int *snb, T *s)
{
    static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte cells");
    constexpr int V = 16 / (int)sizeof(T);
    const int rows = q.ey * q.ez;
    const bool plain = __ldg(bc.mode + q.block) == 0;
    const int t0 = q.ex - 2;
    if (q.xo == V) {
        // per row: t0 / V in-block 16-byte chunks and the two x-halo cells;
        // work item it = r per + k, row r = j + ey kz, indices advanced with
        // carries instead of divided anew
        const int per = t0 / V + 2;
        int r = threadIdx.x / per, k = threadIdx.x - r * per;
        int j = r % q.ey, kz = r / q.ey;
        const int dr = kTileThreads / per, dk = kTileThreads - dr * per;
        const int dj = dr % q.ey, dkz = dr / q.ey;
        for (int it = threadIdx.x; it < rows * per; it += kTileThreads) {
            const int y = q.y0 + j - 1, z = q.z0 + kz - 1;
            T *row = s + q.rs * r;
            if (k < per - 2) {
                const int x = q.x0 + k * V;
                const int r1 = y < 0 ? -1 : (y >= L.n[1] ? 1 : 0), r2 = z < 0 ? -1 : (z >= L.n[2] ? 1 : 0);
                const int outside = (r1 != 0) + (r2 != 0);
                T *dst = row + q.xo + k * V;
                if (!tensorial && outside > 1) {
#pragma unroll
                    for (int v = 0; v < V; ++v) dst[v] = T(0);
                } else if (outside == 0 || plain) {
                    const int sb = outside == 0 ? q.block : snb[1 + 3 * (r1 + 1) + 9 * (r2 + 1)]; // r0 = 0
                    const T *src = comp + (int64_t)sb * L.bstride + x +
                                   (int64_t)L.n[0] * ((y - r1 * L.n[1]) + (int64_t)L.n[1] * (z - r2 * L.n[2]));
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
                } else {
#pragma unroll
                    for (int v = 0; v < V; ++v) dst[v] = lab_fetch_slow<T>(comp, L, bc, q.block, x + v, y, z);
                }
            } else {
                const int xl = k == per - 2 ? -1 : t0; // tile-local x of the halo cell
                stage_cell<T>(comp, L, bc, q, tensorial, snb, plain, q.x0 + xl, y, z, row + q.xo + xl);
            }
            k += dk;
            r += dr;
            j += dj;
            kz += dkz;
            if (k >= per) {
                k -= per;
                ++r;
                ++j;
            }
            if (j >= q.ey) {
                j -= q.ey;
                ++kz;
            }
        }
    } else {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        for (int r = warp; r < rows; r += kTileThreads / 32) {
            const int j = r % q.ey, kz = r / q.ey;
            const int y = q.y0 + j - 1, z = q.z0 + kz - 1;
            for (int i = lane; i < q.ex; i += 32)
                stage_cell<T>(comp, L, bc, q, tensorial, snb, plain, q.x0 + i - 1, y, z, s + (i - 1 + q.xo) + q.rs * r);
        }
    }
}

// the 13 operator values of tile cell (x, y, z) from the staged region
template <typename TP>
__device__ __forceinline__ void region7(const TP *sp, const float *sk, const TilePos &q, int x, int y, int z,
                                        TP (&v)[14])
{
    const int u = ridx(q, x, y, z);
    const int st[3] = {1, q.rs, q.rs * q.ey};
    v[0] = sp[u];
    v[1] = (TP)sk[u];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        v[2 + 4 * d] = sp[u + st[d]];
        v[3 + 4 * d] = sp[u - st[d]];
        v[4 + 4 * d] = (TP)sk[u + st[d]];
        v[5 + 4 * d] = (TP)sk[u - st[d]];
    }
}

} // namespace mg
} // namespace cn
