// euler_stage.cuh -- the fused lab + WENO5-JS + Rusanov + flux-divergence +
// SSP-RK3 stage computation of one 8x8x8 tile, shared by the uniform-grid
// kernel (euler.cu) and the AMR block kernel (amr.cu).  Where the tile comes
// from and how halo cells outside the tile's block are resolved is a policy
// (`Src`): the uniform grid uses the Cartesian lab resolution of FieldLab,
// the AMR layout its own interface ghost fill.
#pragma once

#include "cn_internal.h"
#include "euler_math.cuh"

namespace cn {
namespace euler {

constexpr int TB = 8;                 // tile edge
constexpr int G = 3;                  // ghost width
constexpr int NCORE = TB * TB * TB;   // tile cells: 512
constexpr int NHALO = 2 * G * TB * TB; // one direction's halo slabs: 384
// FP64 stages one direction's halo at a time (smaller shared memory, three
// CTAs per SM); FP32 has room for all three halo slots at once and stages
// them together, saving two barrier-separated load phases.
template <typename T> struct Stg {
    static constexpr bool all = sizeof(T) == 4;
    static constexpr int SV = NCORE + (all ? 3 : 1) * NHALO; // staged cells per variable
};
constexpr int SV = NCORE + NHALO; // FP64 staged cells per variable (896)
constexpr int NCELL = TB * TB * TB;   // 512
constexpr int NFACE = (TB + 1) * TB * TB; // 576
constexpr int NT = 192;               // threads per CTA (576 = 3 * 192)
constexpr int CPT = (NCELL + NT - 1) / NT; // cells per thread: 3

template <typename T> struct StageParams {
    const T *U[5];   // state whose lab is loaded (component bases)
    const T *Un[5];  // U^n (stages 2 and 3)
    T *out[5];
    T dt;
    T gamma, gm1, igm1;
    int stage;       // 0: out = L(U); 1..3: SSP-RK3 stage
    double *partials; // per-tile FP64 sums of the 5 outputs (may be null)
    int *err;
};

// One tile of work: its block, tile origin, block extents and storage.
template <typename T> struct TileInfo {
    int block;
    int x0, y0, z0;
    int N0, N1, N2;
    int64_t boff;     // element offset of the block in each component
    T ih[3];          // 1/h of the block
    int bx, by, bz;   // block coordinates (uniform grid)
};

// Uniform Cartesian grid: tiles in block order, halo cells through the
// FieldLab lab resolution (cn::lab_value) with each component's BC vector.
struct CartSrc {
    LabGeom L;
    BcView bc[5];
    double ih[3];
    template <typename T> __device__ __forceinline__ void tile(int item, TileInfo<T> &t) const
    {
        const int tx = L.n[0] / 8, ty = L.n[1] / 8, tz = L.n[2] / 8;
        const int tiles = tx * ty * tz;
        t.block = item / tiles;
        int r = item - t.block * tiles;
        t.x0 = (r % tx) * 8;
        r /= tx;
        t.y0 = (r % ty) * 8;
        t.z0 = (r / ty) * 8;
        t.N0 = L.n[0];
        t.N1 = L.n[1];
        t.N2 = L.n[2];
        t.boff = (int64_t)t.block * L.bstride;
        t.ih[0] = (T)ih[0];
        t.ih[1] = (T)ih[1];
        t.ih[2] = (T)ih[2];
        t.bx = t.block % L.nb[0];
        t.by = (t.block / L.nb[0]) % L.nb[1];
        t.bz = t.block / (L.nb[0] * L.nb[1]);
    }
    // Per tile, in shared memory (a barrier must follow): snb[0..26] the 27
    // periodic neighbour blocks of the tile's block (index (r0+1) + 3 (r1+1) +
    // 9 (r2+1)), snb[27] the mask of the components whose block carries
    // neither BCs nor skip flags (lab mode byte 0).
    template <typename T>
    __device__ __forceinline__ void prepare(const TileInfo<T> &t, int *snb) const
    {
        if (threadIdx.x < 27) {
            const int q = threadIdx.x;
            int nx = t.bx + q % 3 - 1, ny = t.by + (q / 3) % 3 - 1, nz = t.bz + q / 9 - 1;
            nx = nx < 0 ? nx + L.nb[0] : (nx >= L.nb[0] ? nx - L.nb[0] : nx);
            ny = ny < 0 ? ny + L.nb[1] : (ny >= L.nb[1] ? ny - L.nb[1] : ny);
            nz = nz < 0 ? nz + L.nb[2] : (nz >= L.nb[2] ? nz - L.nb[2] : nz);
            snb[q] = nx + L.nb[0] * (ny + L.nb[1] * nz);
        }
        if (threadIdx.x == 32) {
            unsigned plain = 0;
#pragma unroll
            for (int c = 0; c < 5; ++c)
                plain |= (__ldg(bc[c].mode + t.block) == 0 ? 1u : 0u) << c;
            snb[27] = (int)plain;
        }
    }
    // A halo cell outside the tile's block: for a plain component the
    // periodic neighbour (what cn::lab_value gives for mode 0), else the lab.
    template <typename T>
    __device__ __forceinline__ T halo(const T *comp, int c, const TileInfo<T> &t, int gx, int gy, int gz,
                                      const int *snb) const
    {
        if (((unsigned)snb[27] >> c) & 1u) {
            const int r0 = gx < 0 ? -1 : (gx >= L.n[0] ? 1 : 0), r1 = gy < 0 ? -1 : (gy >= L.n[1] ? 1 : 0),
                      r2 = gz < 0 ? -1 : (gz >= L.n[2] ? 1 : 0);
            // the halo of a face sweep leaves the block along one direction only
            const int sb = snb[(r0 + 1) + 3 * (r1 + 1) + 9 * (r2 + 1)];
            return comp[(int64_t)sb * L.bstride + (gx - r0 * L.n[0]) +
                        (int64_t)L.n[0] * ((gy - r1 * L.n[1]) + (int64_t)L.n[1] * (gz - r2 * L.n[2]))];
        }
        T v;
        if (!lab_value<T>(comp, L, bc[c], t.block, t.bx, t.by, t.bz, gx, gy, gz, true, v)) v = T(0);
        return v;
    }
};

// Shared-memory layout per variable: the tile's 512 core cells x-fastest,
// then the halo slot(s).  The halo slot of direction D holds the two 3-cell
// slabs of that direction, slab coordinate h = 0..5 (cells -3..-1 and 8..10
// along D) with the same stride along D as the core (1, 8, 64):
//   D = 0: (z*8 + y)*6 + h,   D = 1: (z*6 + h)*8 + x,   D = 2: (h*8 + y)*8 + x.
// FP64 keeps one slot and restages it before each sweep; FP32 keeps all three.
//
// The direction is a runtime (warp-uniform) value: one copy of the face code
// serves all three sweeps, which keeps the kernel's hot code small enough for
// the instruction caches.

// tile-local coordinates of halo slot i of direction D
__device__ __forceinline__ void halo_cell(int D, int i, int &x, int &y, int &z)
{
    int h;
    if (D == 0) {
        h = i % (2 * G);
        y = (i / (2 * G)) % TB;
        z = i / (2 * G * TB);
        x = h < G ? h - G : h - G + TB;
    } else if (D == 1) {
        x = i % TB;
        h = (i / TB) % (2 * G);
        z = i / (TB * 2 * G);
        y = h < G ? h - G : h - G + TB;
    } else {
        x = i % TB;
        y = (i / TB) % TB;
        h = i / (TB * TB);
        z = h < G ? h - G : h - G + TB;
    }
}

// Face fluxes of direction D for the whole tile (one thread per face, each
// face once), then flux differences into the per-cell accumulators.
template <typename T>
__device__ __forceinline__ void sweep(int D, const T *__restrict__ W, T *__restrict__ F, T (&acc)[CPT][5],
                                      T gamma, T igm1, T ihd)
{
    constexpr bool ALL = Stg<T>::all;
    const int cs = D == 0 ? 1 : (D == 1 ? TB : TB * TB); // stride along D (core and halo slot)
    const int hslot = NCORE + (ALL ? D * NHALO : 0);
    for (int f = threadIdx.x; f < NFACE; f += NT) {
        // (x, y, z): the cell on the high side of face f; a: its coordinate along D
        int x, y, z, a;
        if (D == 0) {
            x = f % (TB + 1);
            y = (f / (TB + 1)) % TB;
            z = f / ((TB + 1) * TB);
            a = x;
        } else if (D == 1) {
            x = f % TB;
            y = (f / TB) % (TB + 1);
            z = f / (TB * (TB + 1));
            a = y;
        } else {
            x = f % TB;
            y = (f / TB) % TB;
            z = f / (TB * TB);
            a = z;
        }
        // row bases: core cell with coordinate 0 along D, halo slab cell h = 0
        const int cbase = x + TB * (y + TB * z) - a * cs;
        const int hbase = hslot + (D == 0 ? (z * TB + y) * (2 * G) : (D == 1 ? z * (2 * G * TB) + x : y * TB + x));
        // cells a-3 .. a+2 along D
        int idx[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int q = a + k - 3;
            idx[k] = (unsigned)q < (unsigned)TB ? cbase + q * cs : hbase + (q < 0 ? q + G : q - TB + G) * cs;
        }
        T WL[5], WR[5];
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            const T *Wc = W + c * Stg<T>::SV;
            const T v0 = Wc[idx[0]], v1 = Wc[idx[1]], v2 = Wc[idx[2]];
            const T v3 = Wc[idx[3]], v4 = Wc[idx[4]], v5 = Wc[idx[5]];
            weno5_pair(v0, v1, v2, v3, v4, v5, WL[c], WR[c]);
        }
        T Fl[5];
        rusanov<T>(WL, WR, D, gamma, igm1, Fl);
#pragma unroll
        for (int c = 0; c < 5; ++c)
            F[c * NFACE + f] = Fl[c];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const int cidx = threadIdx.x + k * NT;
        if (cidx < NCELL) {
            const int x = cidx % TB, y = (cidx / TB) % TB, z = cidx / (TB * TB);
            const int flo = D == 0 ? x + (TB + 1) * (y + TB * z)
                                   : (D == 1 ? x + TB * (y + (TB + 1) * z) : x + TB * (y + TB * z));
#pragma unroll
            for (int c = 0; c < 5; ++c) {
                const T df = F[c * NFACE + flo + cs] - F[c * NFACE + flo];
                acc[k][c] = D == 0 ? df * ihd : dfma(df, ihd, acc[k][c]);
            }
        }
    }
    __syncthreads();
}

// Loads the two 3-cell halo slabs of direction D into the halo slot:
// cells inside the block are plain loads, cells outside are resolved by the
// source policy (for the Cartesian grid cn::lab_value: periodic neighbour,
// skip rule, BC chain per component).  The out-of-block path resolves one
// component at a time into the slot and converts in place, so its code
// exists once.
template <typename T, typename Src>
__device__ __forceinline__ void stage_halo(int D, const StageParams<T> &p, const Src &src, const TileInfo<T> &t,
                                           T *W, const int *snb)
{
    T *slot = W + NCORE + (Stg<T>::all ? D * NHALO : 0);
    for (int i = threadIdx.x; i < NHALO; i += NT) {
        int x, y, z;
        halo_cell(D, i, x, y, z);
        const int gx = t.x0 + x, gy = t.y0 + y, gz = t.z0 + z;
        T u[5];
        if ((unsigned)gx < (unsigned)t.N0 && (unsigned)gy < (unsigned)t.N1 && (unsigned)gz < (unsigned)t.N2) {
            const int64_t o = t.boff + gx + (int64_t)t.N0 * (gy + (int64_t)t.N1 * gz);
#pragma unroll
            for (int c = 0; c < 5; ++c)
                u[c] = p.U[c][o];
        } else {
#pragma unroll 1
            for (int c = 0; c < 5; ++c)
                slot[c * Stg<T>::SV + i] = src.halo(p.U[c], c, t, gx, gy, gz, snb);
#pragma unroll
            for (int c = 0; c < 5; ++c)
                u[c] = slot[c * Stg<T>::SV + i];
        }
        T w[5];
        to_primitive<T>(u[0], u[1], u[2], u[3], u[4], p.gm1, w);
#pragma unroll
        for (int c = 0; c < 5; ++c)
            slot[c * Stg<T>::SV + i] = w[c];
    }
}

// The whole stage for one tile: staging, three sweeps, RK epilogue and the
// tile's FP64 sums (written to p.partials[slot] if requested).  Uses
// W [5][Stg<T>::SV], F [5][NFACE] and red [NT/32][5] in shared memory.
template <typename T, typename Src>
__device__ __forceinline__ void stage_tile(const StageParams<T> &p, const Src &src, int item, int slot, T *W, T *F,
                                           double (*red)[5], int *snb, TileInfo<T> *ts)
{
    // the tile's geometry is kept in shared memory (ts) and re-read after each
    // barrier, so it does not occupy registers across the three sweeps
    {
        TileInfo<T> t0;
        src.template tile<T>(item, t0);
        if (threadIdx.x == 0) *ts = t0;
    }
    __syncthreads();
    const TileInfo<T> &t = *ts;
    src.template prepare<T>(t, snb);
    __syncthreads(); // snb
    // ---- stage the tile's cells as primitives (the halo slot follows per sweep)
    for (int i = threadIdx.x; i < NCORE; i += NT) {
        const int x = i % TB, y = (i / TB) % TB, z = i / (TB * TB);
        const int64_t o = t.boff + (t.x0 + x) + (int64_t)t.N0 * ((t.y0 + y) + (int64_t)t.N1 * (t.z0 + z));
        T w[5];
        to_primitive<T>(p.U[0][o], p.U[1][o], p.U[2][o], p.U[3][o], p.U[4][o], p.gm1, w);
#pragma unroll
        for (int c = 0; c < 5; ++c)
            W[c * Stg<T>::SV + i] = w[c];
    }
    if (Stg<T>::all) {
#pragma unroll 1
        for (int D = 0; D < 3; ++D)
            stage_halo<T>(D, p, src, t, W, snb);
    } else {
        stage_halo<T>(0, p, src, t, W, snb);
    }
    __syncthreads();

    T acc[CPT][5];
#pragma unroll
    for (int k = 0; k < CPT; ++k)
#pragma unroll
        for (int c = 0; c < 5; ++c)
            acc[k][c] = T(0);

#pragma unroll 1
    for (int D = 0; D < 3; ++D) {
        if (!Stg<T>::all && D > 0) {
            stage_halo<T>(D, p, src, t, W, snb);
            __syncthreads();
        }
        const T ihd = D == 0 ? t.ih[0] : (D == 1 ? t.ih[1] : t.ih[2]);
        sweep<T>(D, W, F, acc, p.gamma, p.igm1, ihd);
    }

    // ---- epilogue: RHS or SSP-RK3 stage, coalesced along x of the tile rows
    double sums[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const int cidx = threadIdx.x + k * NT;
        if (cidx < NCELL) {
            const int x = cidx % TB, y = (cidx / TB) % TB, z = cidx / (TB * TB);
            const int64_t o = t.boff + (t.x0 + x) + (int64_t)t.N0 * ((t.y0 + y) + (int64_t)t.N1 * (t.z0 + z));
#pragma unroll
            for (int c = 0; c < 5; ++c) {
                const T rhs = -acc[k][c];
                T v;
                if (p.stage == 0) {
                    v = rhs;
                } else {
                    const T us = p.U[c][o];
                    const T tt = dfma(p.dt, rhs, us);
                    if (p.stage == 1) {
                        v = tt;
                    } else if (p.stage == 2) {
                        v = dfma(T(0.75), p.Un[c][o], T(0.25) * tt);
                    } else {
                        v = dfma(T(1.0 / 3.0), p.Un[c][o], T(2.0 / 3.0) * tt);
                    }
                }
                p.out[c][o] = v;
                sums[c] += (double)v;
            }
        }
    }
    if (p.partials) {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            double s = sums[c];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1)
                s += __shfl_down_sync(0xffffffffu, s, off);
            if (lane == 0)
                red[warp][c] = s;
        }
        __syncthreads();
        if (threadIdx.x < 5) {
            double s = 0;
            for (int w = 0; w < NT / 32; ++w)
                s += red[w][threadIdx.x];
            p.partials[(int64_t)slot * 5 + threadIdx.x] = s;
        }
    }
    __syncthreads(); // shared memory is reused by the next tile
}

} // namespace euler
} // namespace cn
