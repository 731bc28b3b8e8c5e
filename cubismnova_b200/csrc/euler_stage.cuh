// euler_stage.cuh -- the fused lab + WENO5-JS + Rusanov + flux-divergence +
// SSP-RK3 stage computation of one 8x8x8 tile, shared by the uniform-grid
// kernel (euler.cu) and the AMR block kernel (amr.cu).  Where the tile comes
// from and how halo cells outside the tile's block are resolved is a policy
// (`Src`): the uniform grid uses the Cartesian lab resolution of FieldLab,
// the AMR layout its own interface ghost fill.
#pragma once

#include "cn_internal.h"
#include "cn_tma.cuh"
#include "euler_math.cuh"

namespace cn {
namespace euler {

constexpr int TB = 8;                 // tile edge
constexpr int G = 3;                  // ghost width
constexpr int NCORE = TB * TB * TB;   // tile cells: 512
constexpr int NHALO = 2 * G * TB * TB; // one direction's halo slabs: 384
// Shared-memory strides of the core (x: 1): rows padded to 9 entries and
// planes to 72, so that the 16 lines of a half-warp in a sweep (8 values of
// one coordinate x 2 of the other) hit distinct banks in every direction.
constexpr int CY = 9, CZ = 72;
constexpr int NCORE_SM = TB * CZ;     // 576 shared entries of the core
// Halo slot of direction D (slab coordinate h = 0..5 along D: cells -3..-1
// and 8..10), with the core's stride along D and padded like the core:
//   D = 0: h + 6 y + 49 z,   D = 1: x + 9 h + 56 z,   D = 2: x + 9 y + 72 h.
constexpr int HS0 = 392, HS1 = 448, HS2 = 432;
// FP64 stages one direction's halo at a time (smaller shared memory, three
// CTAs per SM); FP32 has room for all three halo slots at once and stages
// them together, saving two barrier-separated load phases.
template <typename T> struct Stg {
    static constexpr bool all = sizeof(T) == 4;
    static constexpr int SV = NCORE_SM + (all ? HS0 + HS1 + HS2 : HS1); // shared entries per variable
    // first entry of direction D's halo slot
    static __device__ __forceinline__ int slot(int D)
    {
        return NCORE_SM + (all ? (D == 0 ? 0 : (D == 1 ? HS0 : HS0 + HS1)) : 0);
    }
};
// Where primitive variable c of shared entry e (core cell or halo-slot cell)
// lives.  FP64: one array per variable, [5][SV].  FP32: variables (0, 1) and
// (2, 3) interleaved as pairs, so that one 64-bit shared access and one
// packed FP32x2 instruction serve two variables, and variable 4 alone:
// [pairs (0,1): 2 SV][pairs (2,3): 2 SV][variable 4: SV].
__device__ __forceinline__ double &prim(double *W, int c, int e) { return W[c * Stg<double>::SV + e]; }
__device__ __forceinline__ float &prim(float *W, int c, int e)
{
    constexpr int SV = Stg<float>::SV;
    return c < 2 ? W[2 * e + c] : (c < 4 ? W[2 * SV + 2 * e + (c - 2)] : W[4 * SV + e]);
}
constexpr int NCELL = TB * TB * TB;   // 512
// per variable: the cells' flux-difference accumulators (core layout) and
// the 2 x 64 face fluxes exchanged between the runs of a line
constexpr int NACC = NCORE_SM + 2 * 64;
constexpr int NT = 192;               // threads per CTA: 64 lines x 3 runs of 3 faces
constexpr int CPT = (NCELL + NT - 1) / NT; // cells per thread: 3

__device__ __forceinline__ int core_sm(int x, int y, int z) { return x + CY * y + CZ * z; }

// entry of halo cell (x, y, z) with slab coordinate h in direction D's slot
__device__ __forceinline__ int halo_sm(int D, int x, int y, int z, int h)
{
    return D == 0 ? h + 6 * y + 49 * z : (D == 1 ? x + 9 * h + 56 * z : x + 9 * y + 72 * h);
}

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
    // halo cells resolve per component (each has its own BC chain)
    static constexpr bool kHalo5 = false;
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
    // neither BCs nor skip flags (lab mode byte 0), snb[28] the union over
    // the components of the block's face masks (BcView::faces).
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
            unsigned plain = 0, faces = 0;
#pragma unroll
            for (int c = 0; c < 5; ++c) {
                plain |= (__ldg(bc[c].mode + t.block) == 0 ? 1u : 0u) << c;
                faces |= __ldg(bc[c].faces + t.block);
            }
            snb[27] = (int)plain;
            snb[28] = (int)faces;
        }
    }
    // Element offset (in every component) of a halo cell outside the tile's
    // block when it is the periodic neighbour's cell in all five components
    // (what cn::lab_value gives): every component's block is plain (mode 0),
    // or the cell lies across one face that carries no BC other than Base
    // and no skip flag in any component.  False otherwise.
    template <typename T>
    __device__ __forceinline__ bool plain_offset(const TileInfo<T> &t, int gx, int gy, int gz, const int *snb,
                                                 int64_t &off) const
    {
        const int r0 = gx < 0 ? -1 : (gx >= L.n[0] ? 1 : 0), r1 = gy < 0 ? -1 : (gy >= L.n[1] ? 1 : 0),
                  r2 = gz < 0 ? -1 : (gz >= L.n[2] ? 1 : 0);
        if (snb[27] != 31) {
            if ((r0 != 0) + (r1 != 0) + (r2 != 0) != 1) return false;
            const int bit = r0 != 0 ? (r0 < 0 ? 0 : 1) : (r1 != 0 ? (r1 < 0 ? 2 : 3) : (r2 < 0 ? 4 : 5));
            if ((snb[28] >> bit) & 1) return false;
        }
        const int sb = snb[(r0 + 1) + 3 * (r1 + 1) + 9 * (r2 + 1)];
        off = (int64_t)sb * L.bstride + (gx - r0 * L.n[0]) +
              (int64_t)L.n[0] * ((gy - r1 * L.n[1]) + (int64_t)L.n[1] * (gz - r2 * L.n[2]));
        return true;
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

// Shared-memory layout per variable: the tile's core (strides 1, CY, CZ),
// then the halo slot(s), each with the core's stride along its direction.
// FP64 keeps one slot and restages it before each sweep; FP32 keeps all three.
//
// The direction is a runtime (warp-uniform) value: one copy of the face code
// serves all three sweeps, which keeps the kernel's hot code small enough for
// the instruction caches.

// tile-local coordinates and slab coordinate h of halo cell i (0..383) of
// direction D
__device__ __forceinline__ void halo_cell(int D, int i, int &x, int &y, int &z, int &h)
{
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

// WENO5 states along a line of a sweep: a cell's smoothness indicators serve
// its right-biased state (lower face) and its left-biased state (upper face);
// the left state waits in a carry for the next face.  id[0..4]: shared
// entries of the cells a-2 .. a+2 around cell a.
template <typename T>
__device__ __forceinline__ T cell_left(const T *Wc, const int (&id)[5], bool scaled = true)
{
    const T u2 = Wc[id[2]];
    const Diff5<T> df = weno5_diff(Wc[id[0]], Wc[id[1]], u2, Wc[id[3]], Wc[id[4]]);
    T p12, p02, p01, nl, dl;
    weno5_beta(df, p12, p02, p01, scaled);
    weno5_left(df, p12, K<T>::d1 * p02, p01, nl, dl);
    return weno5_value(u2, nl, dl);
}
// face a: WL = carried left state of cell a-1, WR = right state of cell a;
// with `more` the carry becomes cell a's left state
template <typename T>
__device__ __forceinline__ void cell_face(const T *Wc, const int (&id)[5], bool more, T &carry, T &wl, T &wr,
                                          bool scaled = true)
{
    const T u2 = Wc[id[2]];
    const Diff5<T> df = weno5_diff(Wc[id[0]], Wc[id[1]], u2, Wc[id[3]], Wc[id[4]]);
    T p12, p02, p01, nr, dr;
    weno5_beta(df, p12, p02, p01, scaled);
    const T w1 = K<T>::d1 * p02;
    weno5_right(df, p12, w1, p01, nr, dr);
    wr = weno5_value(u2, nr, dr);
    wl = carry;
    if (more) {
        T nl, dl;
        weno5_left(df, p12, w1, p01, nl, dl);
        carry = weno5_value(u2, nl, dl);
    }
}
__device__ __forceinline__ float2 pair_left(const float2 *P, const int (&id)[5], bool scaled)
{
    const float2 u2 = P[id[2]];
    const Diff5x2 df = weno5_diff2(P[id[0]], P[id[1]], u2, P[id[3]], P[id[4]]);
    float2 p12, p02, p01, nl, dl;
    weno5_beta2(df, p12, p02, p01, scaled);
    weno5_left2(df, p12, mul2(f2(K<float>::d1), p02), p01, nl, dl);
    return weno5_value2(u2, nl, dl);
}
__device__ __forceinline__ void pair_face(const float2 *P, const int (&id)[5], bool more, float2 &carry, float2 &wl,
                                          float2 &wr, bool scaled)
{
    const float2 u2 = P[id[2]];
    const Diff5x2 df = weno5_diff2(P[id[0]], P[id[1]], u2, P[id[3]], P[id[4]]);
    float2 p12, p02, p01, nr, dr;
    weno5_beta2(df, p12, p02, p01, scaled);
    const float2 w1 = mul2(f2(K<float>::d1), p02);
    weno5_right2(df, p12, w1, p01, nr, dr);
    wr = weno5_value2(u2, nr, dr);
    wl = carry;
    if (more) {
        float2 nl, dl;
        weno5_left2(df, p12, w1, p01, nl, dl);
        carry = weno5_value2(u2, nl, dl);
    }
}

// Carried left states of the five variables: FP64 one by one, FP32 as the
// pairs (0,1), (2,3) and variable 4.
struct CarryD {
    double v[5];
};
struct CarryF {
    float2 p01, p23;
    float v4;
};
__device__ __forceinline__ void line_left(const double *W, const int (&id)[5], CarryD &cl, bool)
{
#pragma unroll
    for (int c = 0; c < 5; ++c)
        cl.v[c] = cell_left(W + c * Stg<double>::SV, id);
}
__device__ __forceinline__ void line_face(const double *W, const int (&id)[5], bool more, CarryD &cl,
                                          double (&WL)[5], double (&WR)[5], bool)
{
#pragma unroll
    for (int c = 0; c < 5; ++c)
        cell_face(W + c * Stg<double>::SV, id, more, cl.v[c], WL[c], WR[c]);
}
__device__ __forceinline__ void line_left(const float *W, const int (&id)[5], CarryF &cl, bool scaled)
{
    constexpr int SV = Stg<float>::SV;
    cl.p01 = pair_left(reinterpret_cast<const float2 *>(W), id, scaled);
    cl.p23 = pair_left(reinterpret_cast<const float2 *>(W + 2 * SV), id, scaled);
    cl.v4 = cell_left(W + 4 * SV, id, scaled);
}
__device__ __forceinline__ void line_face(const float *W, const int (&id)[5], bool more, CarryF &cl,
                                          float (&WL)[5], float (&WR)[5], bool scaled)
{
    constexpr int SV = Stg<float>::SV;
    float2 l01, r01, l23, r23;
    pair_face(reinterpret_cast<const float2 *>(W), id, more, cl.p01, l01, r01, scaled);
    pair_face(reinterpret_cast<const float2 *>(W + 2 * SV), id, more, cl.p23, l23, r23, scaled);
    cell_face(W + 4 * SV, id, more, cl.v4, WL[4], WR[4], scaled);
    WL[0] = l01.x;
    WL[1] = l01.y;
    WL[2] = l23.x;
    WL[3] = l23.y;
    WR[0] = r01.x;
    WR[1] = r01.y;
    WR[2] = r23.x;
    WR[3] = r23.y;
}
template <typename T> struct CarryOf;
template <> struct CarryOf<double> {
    using type = CarryD;
};
template <> struct CarryOf<float> {
    using type = CarryF;
};

// Face fluxes of direction D for the whole tile, differenced into the
// per-cell accumulators R (shared memory, the core's padded layout).  Each of
// the tile's 64 lines along D has 9 faces (face a between cells a-1 and a);
// thread t takes the run of faces 3r .. 3r+2, r = t / 64, of line t % 64,
// walking up the line so that each cell's smoothness indicators serve both of
// its faces: the left-biased state of cell a-1 is carried from one face to
// the next (line_left / line_face).  The flux of the previous face stays in registers, so a run
// completes its cells 3r and 3r+1 by itself; the third cell of runs 0 and 1
// takes the next run's first face through the exchange slots X after a
// barrier.  R and X: [5][NACC] with R at entry core_sm(x, y, z) and X at
// NCORE_SM + 64 (r - 1) + line.
template <typename T>
__device__ __forceinline__ void sweep(int D, const T *__restrict__ W, T *__restrict__ A, T gamma, T igm1, T ihd,
                                      bool scaled)
{
    const int cs = D == 0 ? 1 : (D == 1 ? CY : CZ);     // shared stride along D (core and halo slot)
    const int run = threadIdx.x >> 6, line = threadIdx.x & 63;
    const int l0 = line & 7, l1 = line >> 3;
    const int x = D == 0 ? 0 : l0, y = D == 1 ? 0 : (D == 0 ? l0 : l1), z = D == 2 ? 0 : l1;
    const int cbase = core_sm(x, y, z);                          // the line's cell 0
    const int hbase = Stg<T>::slot(D) + halo_sm(D, x, y, z, 0);  // the line's slab cell h = 0
    const int f0 = 3 * run;
    auto sidx = [&](int a) {
        return (unsigned)a < (unsigned)TB ? cbase + a * cs : hbase + (a < 0 ? a + G : a - TB + G) * cs;
    };
    // left-biased state of cell f0-1, the lower cell of the run's first face
    typename CarryOf<T>::type carry;
    // shared entries of the stencil cells a-2 .. a+2.  FP32 shifts the window
    // by one cell per face (one new entry); FP64 recomputes it (its registers
    // are the scarcer resource)
    int id[5];
#pragma unroll
    for (int k = 0; k < 5; ++k)
        id[k] = sidx(f0 - 3 + k);
    line_left(W, id, carry, scaled);
    T Fq[5]; // flux of the previous face of the run
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
        const int a = f0 + i; // face a: cells a-1 (left state carried in VL) and a
        if constexpr (sizeof(T) == 4) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                id[k] = id[k + 1];
            id[4] = sidx(a + 2);
        } else {
#pragma unroll
            for (int k = 0; k < 5; ++k)
                id[k] = sidx(a - 2 + k);
        }
        T WL[5], WR[5];
        line_face(W, id, i < 2, carry, WL, WR, scaled);
        T Fl[5];
        rusanov<T>(WL, WR, D, gamma, igm1, Fl);
        if (i == 0) {
            if (run > 0) {
#pragma unroll
                for (int c = 0; c < 5; ++c)
                    A[c * NACC + NCORE_SM + 64 * (run - 1) + line] = Fl[c];
            }
        } else {
            // cell a-1 is complete: faces a-1 (Fq) and a (Fl)
            const int e = cbase + (a - 1) * cs;
#pragma unroll
            for (int c = 0; c < 5; ++c) {
                const T df = Fl[c] - Fq[c];
                A[c * NACC + e] = D == 0 ? df * ihd : dfma(df, ihd, A[c * NACC + e]);
            }
        }
#pragma unroll
        for (int c = 0; c < 5; ++c)
            Fq[c] = Fl[c];
    }
    __syncthreads(); // X
    if (run < 2) {
        // cell f0+2: faces f0+2 (Fq) and f0+3, the first face of run r+1
        const int e = cbase + (f0 + 2) * cs;
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            const T df = A[c * NACC + NCORE_SM + 64 * run + line] - Fq[c];
            A[c * NACC + e] = D == 0 ? df * ihd : dfma(df, ihd, A[c * NACC + e]);
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
                                           T *W, const int *snb, T &vmax)
{
    static_assert(NHALO % NT == 0, "whole halo cells per thread");
    constexpr int HPT = NHALO / NT; // halo cells per thread: 2
    const int sb = Stg<T>::slot(D); // first shared entry of the halo slot
    // first pass: the plain loads of all of the thread's cells (inside the
    // block, or the periodic neighbour's cell when every component is plain)
    // are issued together; the other cells are resolved into the slot
    T u[HPT][5];
    bool inb[HPT];
    int si[HPT];
#pragma unroll
    for (int j = 0; j < HPT; ++j) {
        const int i = threadIdx.x + j * NT;
        int x, y, z, h;
        halo_cell(D, i, x, y, z, h);
        si[j] = halo_sm(D, x, y, z, h);
        const int gx = t.x0 + x, gy = t.y0 + y, gz = t.z0 + z;
        int64_t o = 0;
        inb[j] = (unsigned)gx < (unsigned)t.N0 && (unsigned)gy < (unsigned)t.N1 && (unsigned)gz < (unsigned)t.N2;
        if (inb[j])
            o = t.boff + gx + (int64_t)t.N0 * (gy + (int64_t)t.N1 * gz);
        else
            inb[j] = src.plain_offset(t, gx, gy, gz, snb, o);
        if (inb[j]) {
#pragma unroll
            for (int c = 0; c < 5; ++c)
                u[j][c] = p.U[c][o];
        } else if constexpr (Src::kHalo5) {
            T v[5];
            src.halo5(p.U, t, gx, gy, gz, snb, v);
#pragma unroll
            for (int c = 0; c < 5; ++c)
                prim(W, c, sb + si[j]) = v[c];
        } else {
#pragma unroll 1
            for (int c = 0; c < 5; ++c)
                prim(W, c, sb + si[j]) = src.halo(p.U[c], c, t, gx, gy, gz, snb);
        }
    }
    // second pass: conversion to primitives in place
#pragma unroll
    for (int j = 0; j < HPT; ++j) {
        if (!inb[j]) {
#pragma unroll
            for (int c = 0; c < 5; ++c)
                u[j][c] = prim(W, c, sb + si[j]);
        }
        T w[5];
        to_primitive<T>(u[j][0], u[j][1], u[j][2], u[j][3], u[j][4], p.gm1, w);
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            prim(W, c, sb + si[j]) = w[c];
            if constexpr (sizeof(T) == 4) vmax = fmaxf(vmax, fabsf(w[c]));
        }
    }
}

// The whole stage for one tile: staging, three sweeps, RK epilogue and the
// tile's FP64 sums (written to p.partials[slot] if requested).  Uses
// W [5][Stg<T>::SV], A [5][NACC] and red [NT/32][5] in shared memory.
// With CORE_TMA, `core_map` (a tensor map over the five components of U as
// [comp][block][z][y][x], box 8 x 8 x 8 x 1 x 5) brings the tile's cells by
// one TMA copy into A, which is free until the sweeps; `core_bar`
// (initialised with count 1, used once per CTA: parity 0) signals its
// completion.  Without it each thread loads its cells.
template <typename T, typename Src, bool CORE_TMA = false>
__device__ __forceinline__ void stage_tile(const StageParams<T> &p, const Src &src, int item, int slot, T *W, T *A,
                                           double (*red)[5], int *snb, TileInfo<T> *ts,
                                           const void *core_map = nullptr, uint64_t *core_bar = nullptr)
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
    // ---- stage the tile's cells as primitives (the halo slot follows per
    // sweep): all of a thread's loads are issued before any conversion
    // FP32: the largest primitive magnitude the thread stages (NaN data
    // gives NaN states on either form of the weights)
    T vmax = T(0);
    auto convert_core = [&](T (&u)[CPT][5]) {
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int i = threadIdx.x + k * NT;
            if (i < NCORE) {
                T w[5];
                to_primitive<T>(u[k][0], u[k][1], u[k][2], u[k][3], u[k][4], p.gm1, w);
                const int e = core_sm(i % TB, (i / TB) % TB, i / (TB * TB));
#pragma unroll
                for (int c = 0; c < 5; ++c) {
                    prim(W, c, e) = w[c];
                    if constexpr (sizeof(T) == 4) vmax = fmaxf(vmax, fabsf(w[c]));
                }
            }
        }
    };
    if constexpr (CORE_TMA) {
        // one copy brings the tile's cells of all five components, dense
        // [5][8][8][8] in A; converted before the halo staging (converting
        // after it keeps both sets of values live and spills)
        if (threadIdx.x == 0) {
            mbar_arrive_expect_tx(core_bar, 5u * NCORE * (uint32_t)sizeof(T));
            tma_load_5d(A, core_map, t.x0, t.y0, t.z0, t.block, 0, core_bar);
        }
        if (!mbar_wait_bounded_sleep(core_bar, 0, 100)) {
            // record the error, then give the copy a second bounded wait so
            // that it is not left writing into this CTA's shared memory
            if (p.err) atomicExch(p.err, kDevErrTimeout);
            mbar_wait_bounded_sleep(core_bar, 0, 100);
        }
        T u[CPT][5];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int i = threadIdx.x + k * NT;
#pragma unroll
            for (int c = 0; c < 5; ++c)
                u[k][c] = i < NCORE ? A[c * NCORE + i] : T(0);
        }
        convert_core(u);
    } else {
        T u[CPT][5];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int i = threadIdx.x + k * NT;
            if (i < NCORE) {
                const int x = i % TB, y = (i / TB) % TB, z = i / (TB * TB);
                const int64_t o =
                    t.boff + (t.x0 + x) + (int64_t)t.N0 * ((t.y0 + y) + (int64_t)t.N1 * (t.z0 + z));
#pragma unroll
                for (int c = 0; c < 5; ++c)
                    u[k][c] = p.U[c][o];
            }
        }
        convert_core(u);
    }
    // FP32 stages all three halo slots here; the tile's WENO5 weights skip
    // the range rescaling when every staged primitive is within
    // kUnscaledMax (same values, fewer instructions: see euler_math.cuh)
    bool scaled = true;
    if (Stg<T>::all) {
#pragma unroll 1
        for (int D = 0; D < 3; ++D)
            stage_halo<T>(D, p, src, t, W, snb, vmax);
        scaled = __syncthreads_or(!(vmax <= T(kUnscaledMax))) != 0;
    } else {
        stage_halo<T>(0, p, src, t, W, snb, vmax);
        __syncthreads();
    }

#pragma unroll 1
    for (int D = 0; D < 3; ++D) {
        if (!Stg<T>::all && D > 0) {
            stage_halo<T>(D, p, src, t, W, snb, vmax);
            __syncthreads();
        }
        // the Rusanov fluxes are twice the flux: 1/(2h) (exact)
        const T ihd = T(0.5) * (D == 0 ? t.ih[0] : (D == 1 ? t.ih[1] : t.ih[2]));
        sweep<T>(D, W, A, p.gamma, p.igm1, ihd, scaled);
    }

    // ---- epilogue: RHS or SSP-RK3 stage, coalesced along x of the tile rows.
    // One component at a time, with the next component's loads of U_s and
    // U^n issued before this component's stores: `out` may alias U^n (stage
    // 3 updates U in place), so loads cannot move above earlier stores, and
    // issuing them early keeps one memory latency per tile instead of one per
    // value.  Each (component, cell) is loaded before it is stored.
    double sums[5] = {0, 0, 0, 0, 0};
    int64_t eo[CPT];
    int ea[CPT];
    bool eok[CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const int cidx = threadIdx.x + k * NT;
        eok[k] = cidx < NCELL;
        const int x = cidx % TB, y = (cidx / TB) % TB, z = cidx / (TB * TB);
        eo[k] = t.boff + (t.x0 + x) + (int64_t)t.N0 * ((t.y0 + y) + (int64_t)t.N1 * (t.z0 + z));
        ea[k] = core_sm(x, y, z);
    }
    T us[2][CPT], un[2][CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        us[0][k] = (p.stage >= 1 && eok[k]) ? p.U[0][eo[k]] : T(0);
        un[0][k] = (p.stage >= 2 && eok[k]) ? p.Un[0][eo[k]] : T(0);
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        const int b = c & 1;
        if (c + 1 < 5) {
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                us[b ^ 1][k] = (p.stage >= 1 && eok[k]) ? p.U[c + 1][eo[k]] : T(0);
                un[b ^ 1][k] = (p.stage >= 2 && eok[k]) ? p.Un[c + 1][eo[k]] : T(0);
            }
        }
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            if (eok[k]) {
                const T rhs = -A[c * NACC + ea[k]];
                T v;
                if (p.stage == 0) {
                    v = rhs;
                } else {
                    const T tt = dfma(p.dt, rhs, us[b][k]);
                    if (p.stage == 1) {
                        v = tt;
                    } else if (p.stage == 2) {
                        v = dfma(T(0.75), un[b][k], T(0.25) * tt);
                    } else {
                        v = dfma(T(1.0 / 3.0), un[b][k], T(2.0 / 3.0) * tt);
                    }
                }
                p.out[c][eo[k]] = v;
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
