// amr.cuh -- ghost cells of blocks on two refinement levels (ratio 2).
//
// A layout is a set of cubic blocks tiling a periodic box of Lx x Ly x Lz
// level-1 cells; each block has a level (0 coarse, 1 fine; cell size 2 or 1
// in level-1 units), n^3 cells and an origin in level-1 cell units (multiples
// of 8).  A lookup grid with one entry per 8^3 level-1 cells maps a position
// to the block that covers it.
// A ghost cell of block b takes its value from the block s covering it:
//   same level   copy of the cell;
//   s coarser    trilinear prolongation from s (cell-centred weights 3/4, 1/4
//                per direction, x then y then z), the stencil's neighbour
//                index clamped to s's cells;
//   s finer      conservative restriction: mean of the 8 fine cells,
//                ((c0+c1)+(c2+c3)) + ((c4+c5)+(c6+c7)), child c = dx|dy<<1|dz<<2.
// The reference describes level interfaces only in notes
// (test/sandbox/doc/notes/01_notes.md:192-196); this is the standard
// block-structured AMR ghost fill.
#pragma once

#include <cstdint>

namespace cn {
namespace amr {

struct BlockDev {
    int level;  // 0 or 1
    int n;      // cells per dimension
    int ox, oy, oz; // origin in level-1 cell units
    int pad;
    int64_t off; // element offset of the block in each component
    double ih;   // 1 / h
};

struct Geom {
    const BlockDev *blk;
    const int32_t *lookup; // lr[0] x lr[1] x lr[2] block ids
    int L[3];              // domain extents in level-1 cells (periodic)
    int lr[3];             // L / 8
    __device__ __forceinline__ int block_at(int X, int Y, int Z) const
    {
        return lookup[(X >> 3) + lr[0] * ((Y >> 3) + lr[1] * (Z >> 3))];
    }
};

__device__ __forceinline__ int wrap(int x, int L) { return x < 0 ? x + L : (x >= L ? x - L : x); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

template <typename T>
__device__ __forceinline__ T cell(const T *comp, const BlockDev &B, int x, int y, int z)
{
    return comp[B.off + x + (int64_t)B.n * (y + (int64_t)B.n * z)];
}

// Element offset (in every component) of lab cell q of block b, outside b,
// when the block covering it is on b's level: the ghost is a plain copy of
// that cell, as value() gives it.  False for level-interface ghosts.
__device__ __forceinline__ bool same_level_offset(const Geom &A, int b, int qx, int qy, int qz, int64_t &off)
{
    const BlockDev B = A.blk[b];
    const int cs = B.level == 0 ? 2 : 1;
    const int X = wrap(B.ox + qx * cs, A.L[0]), Y = wrap(B.oy + qy * cs, A.L[1]), Z = wrap(B.oz + qz * cs, A.L[2]);
    const int s = A.block_at(X, Y, Z);
    const BlockDev S = A.blk[s];
    if (S.level != B.level) return false;
    const int fx = (X - S.ox) / cs, fy = (Y - S.oy) / cs, fz = (Z - S.oz) / cs;
    off = S.off + fx + (int64_t)S.n * (fy + (int64_t)S.n * fz);
    return true;
}

// Where lab cell q (tile coordinates of block b, possibly outside it) takes
// its value from: a cell of b or of a block on b's level (kind 0, cell
// (fx, fy, fz) of S), trilinear prolongation from the coarser S (kind 1),
// or the mean of 8 cells of the finer S (kind 2); (fx, fy, fz) are level-1
// offsets inside S for kinds 1 and 2.  The geometry does not depend on the
// component, so a halo cell resolves it once for all of them.
struct Ghost {
    int kind;
    BlockDev S;
    int fx, fy, fz;
};

__device__ __forceinline__ Ghost resolve(const Geom &A, int b, int qx, int qy, int qz)
{
    Ghost g;
    const BlockDev B = A.blk[b];
    if ((unsigned)qx < (unsigned)B.n && (unsigned)qy < (unsigned)B.n && (unsigned)qz < (unsigned)B.n) {
        g.kind = 0;
        g.S = B;
        g.fx = qx;
        g.fy = qy;
        g.fz = qz;
        return g;
    }
    const int cs = B.level == 0 ? 2 : 1;
    const int X = wrap(B.ox + qx * cs, A.L[0]), Y = wrap(B.oy + qy * cs, A.L[1]), Z = wrap(B.oz + qz * cs, A.L[2]);
    g.S = A.blk[A.block_at(X, Y, Z)];
    g.fx = X - g.S.ox;
    g.fy = Y - g.S.oy;
    g.fz = Z - g.S.oz;
    if (g.S.level == B.level) {
        const int css = g.S.level == 0 ? 2 : 1;
        g.kind = 0;
        g.fx /= css;
        g.fy /= css;
        g.fz /= css;
    } else {
        g.kind = g.S.level < B.level ? 1 : 2;
    }
    return g;
}

template <typename T> __device__ __forceinline__ T gather(const T *comp, const Ghost &g)
{
    const BlockDev &S = g.S;
    if (g.kind == 0) return cell<T>(comp, S, g.fx, g.fy, g.fz);
    if (g.kind == 1) {
        // fine ghost cell inside a coarse block: trilinear prolongation
        const int px = g.fx >> 1, py = g.fy >> 1, pz = g.fz >> 1;
        const int qx1 = clampi(px + ((g.fx & 1) ? 1 : -1), 0, S.n - 1);
        const int qy1 = clampi(py + ((g.fy & 1) ? 1 : -1), 0, S.n - 1);
        const int qz1 = clampi(pz + ((g.fz & 1) ? 1 : -1), 0, S.n - 1);
        const T e000 = cell<T>(comp, S, px, py, pz), e100 = cell<T>(comp, S, qx1, py, pz);
        const T e010 = cell<T>(comp, S, px, qy1, pz), e110 = cell<T>(comp, S, qx1, qy1, pz);
        const T e001 = cell<T>(comp, S, px, py, qz1), e101 = cell<T>(comp, S, qx1, py, qz1);
        const T e011 = cell<T>(comp, S, px, qy1, qz1), e111 = cell<T>(comp, S, qx1, qy1, qz1);
        // weights 3/4, 1/4 per direction; products and sums rounded one by
        // one (never contracted, whatever the compiler's FMA setting)
        const T a = T(0.75), c = T(0.25);
        const T a0 = add_rn(mul_rn(a, e000), mul_rn(c, e100));
        const T a1 = add_rn(mul_rn(a, e010), mul_rn(c, e110));
        const T a2 = add_rn(mul_rn(a, e001), mul_rn(c, e101));
        const T a3 = add_rn(mul_rn(a, e011), mul_rn(c, e111));
        const T b0 = add_rn(mul_rn(a, a0), mul_rn(c, a1));
        const T b1 = add_rn(mul_rn(a, a2), mul_rn(c, a3));
        return add_rn(mul_rn(a, b0), mul_rn(c, b1));
    }
    // coarse ghost cell over a fine block: mean of its 8 children
    T v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
        v[k] = cell<T>(comp, S, g.fx + (k & 1), g.fy + ((k >> 1) & 1), g.fz + (k >> 2));
    return (((v[0] + v[1]) + (v[2] + v[3])) + ((v[4] + v[5]) + (v[6] + v[7]))) * T(0.125);
}

// value of lab cell q (tile coordinates of block b, possibly outside it)
template <typename T>
__device__ __forceinline__ T value(const T *comp, const Geom &A, int b, int qx, int qy, int qz)
{
    return gather<T>(comp, resolve(A, b, qx, qy, qz));
}

} // namespace amr
} // namespace cn
