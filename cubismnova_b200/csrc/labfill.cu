// labfill.cu -- K0: explicit lab fill (Cartesian::loadLab into lab buffers).
//
// One CTA per (block, slab of lab planes along z).  The slab's lab cells
// fall into four classes: the block's own cells, the x ghosts of the rows
// inside the block, the y-ghost rows of the inside planes and the z-ghost
// planes (non-tensorial labs: edges and corners stay undefined, as in the
// reference).  The block's own planes are one contiguous run of memory,
// brought by one bulk copy into shared memory; meanwhile the threads walk
// the ghosts, those behind faces without a BC or a skipped neighbour in
// closed form (the periodic neighbour's cell), eight loads in flight per
// thread; ghost rows behind faces with BCs are resolved once per row (x
// passes through the FieldLab resolution unchanged), other BC-chain cells
// one by one (cn::lab_resolve: skip rule, BC chain); this one-pass form is
// lab_fill_rows_kernel.  Tensorial labs and labs with ghost rows longer than
// its row table (lab_fill_kernel), node and face grids
// (lab_fill_grow_kernel) take per-class or per-cell resolution.  Stores
// are coalesced along the lab's rows; the kernel is bound by memory
// latency and HBM.  The stencil kernels fuse the same resolution into their
// shared-memory staging; this kernel gives the reference's FieldLab
// contents for user stencils and the bit-exact comparison with it.
#include "cn_fastdiv.h"
#include "cn_internal.h"
#include "cn_tma.cuh"

#include <algorithm>

namespace cn {

constexpr int KL = 4;              // cells per thread resolved before their loads
constexpr int KL0 = 8;             // pairs of the block's own cells per thread in flight
constexpr int KLM = 8;             // cells per thread in flight in the one-pass form
constexpr int kBulkBytes = 24576;  // largest bulk copy of a slab's block planes
// target cells of a CTA's slab: three planes of the 38^2 lab of 32^3 blocks
// with three ghosts.  Thinner slabs leave more of the SM's on-chip memory
// to the L1 cache (the shared-memory carve-out follows the resident CTAs'
// needs), which measured faster than thicker slabs
constexpr int kCellsPerCta = 4332;
constexpr int kRowsCtas = 4;       // resident CTAs per SM of the one-pass kernel

// a cell's source, collected from lab_resolve
template <typename T> struct LabSource {
    int kind = 0; // 0 undefined, 1 the value v, 2 comp[idx] times the signs
    int nsign = 0;
    int64_t idx = 0;
    T v = T(0), s0 = T(1), s1 = T(1), s2 = T(1);
    __device__ __forceinline__ void value(T x)
    {
        kind = 1;
        v = x;
    }
    __device__ __forceinline__ void load(int64_t i, int n, T a, T b, T c)
    {
        kind = 2;
        idx = i;
        nsign = n;
        s0 = a;
        s1 = b;
        s2 = c;
    }
};

// Loads the sources of up to KL cells, then stores them: src[k] for cell
// dst[k] (offsets in the CTA's output, -1: no cell).
template <typename T>
__device__ __forceinline__ void lab_store(const T *__restrict__ comp, const LabSource<T> (&src)[KL],
                                          const int (&dst)[KL], T *__restrict__ o)
{
    T v[KL];
#pragma unroll
    for (int k = 0; k < KL; ++k)
        v[k] = src[k].kind == 2 ? comp[src[k].idx] : src[k].v;
#pragma unroll
    for (int k = 0; k < KL; ++k) {
        if (dst[k] < 0 || src[k].kind == 0) continue;
        T x = v[k];
        if (src[k].kind == 2) {
            if (src[k].nsign > 2) x = src[k].s2 * x;
            if (src[k].nsign > 1) x = src[k].s1 * x;
            if (src[k].nsign > 0) x = src[k].s0 * x;
        }
        o[dst[k]] = x;
    }
}

// Node and face grids (per-block extents): every cell of the CTA's slab
// resolved on its own.
template <typename T>
__global__ void __launch_bounds__(256)
    lab_fill_grow_kernel(const T *__restrict__ comp, LabGeom L, BcView bc, int block_begin, int pz, FastDiv dE0,
                         FastDiv dPlane, int apply_bc, T *__restrict__ out)
{
    const int E0 = L.n[0] + L.lo[0] + L.hi[0];
    const int E1 = L.n[1] + L.lo[1] + L.hi[1];
    const int E2 = L.n[2] + L.lo[2] + L.hi[2];
    const int plane = E0 * E1;
    const int bl = blockIdx.y, z0 = blockIdx.x * pz; // block-major, as lab_fill_rows_kernel
    const int nz = min(pz, E2 - z0);
    const int block = block_begin + bl;
    const int bx = block % L.nb[0];
    const int by = (block / L.nb[0]) % L.nb[1];
    const int bz = block / (L.nb[0] * L.nb[1]);
    const uint8_t mode = bc.mode[block];
    const int cells = nz * plane;
    T *o = out + ((int64_t)bl * E2 + z0) * plane;
    for (int t0 = threadIdx.x; t0 < cells; t0 += KL * blockDim.x) {
        LabSource<T> src[KL];
        int dst[KL];
#pragma unroll
        for (int k = 0; k < KL; ++k) {
            const int t = t0 + k * blockDim.x;
            dst[k] = -1;
            if (t < cells) {
                const int zz = dPlane.div(t), r = t - zz * plane;
                const int y = dE0.div(r), x = r - y * E0;
                dst[k] = t;
                lab_resolve<T, true>(L, bc, mode, block, bx, by, bz, x - L.lo[0], y - L.lo[1], z0 + zz - L.lo[2],
                                     apply_bc != 0, src[k]);
            }
        }
        lab_store<T>(comp, src, dst, o);
    }
}

// a row of class 2 or 3: the source of its first cell and its first cell's
// offset in the lab
template <typename T> struct RowSrc {
    LabSource<T> s;
    int dst;
};
constexpr int kRows = 96; // rows resolved per round

template <typename T> struct Vec2;
template <> struct Vec2<double> {
    using type = double2;
};
template <> struct Vec2<float> {
    using type = float2;
};
template <> struct Vec2<int32_t> {
    using type = int2;
};

// Divisors of the cell-grid kernel's four cell classes (fixed per launch).
struct LabDivs {
    FastDiv n0, n1;   // block extents along x, y
    FastDiv gx;       // x ghosts per row: lo0 + hi0
    FastDiv wrow, gy; // cells per ghost row (n0, or E0 if tensorial); y ghost rows: lo1 + hi1
    FastDiv wpl;      // rows per z-ghost plane (n1, or E1 if tensorial)
};

// lab coordinates of class-1 cell u (the x ghosts of the inside rows)
__device__ __forceinline__ void class1_cell(const LabDivs &dv, int u, int gx, int n0, int n1, int lo0, int lo1, int zi0,
                                            int &x, int &y, int &z)
{
    const int r = dv.gx.div(u), zp = dv.n1.div(r);
    const int g = u - r * gx;
    x = g < lo0 ? g : g + n0;
    y = r - zp * n1 + lo1;
    z = zi0 + zp;
}

// Row `row` of classes 2 and 3 of a non-tensorial lab (rows [0, ny): the
// y-ghost rows of the slab's inside planes; then the rows of its z-ghost
// planes): the source of its first cell (x = 0 of the block) and that
// cell's offset in the lab.  x passes through every step of the resolution
// unchanged, so cell x of the row is the source shifted by x (or the same
// value).
template <typename T>
__device__ __forceinline__ RowSrc<T> lab_row(const LabGeom &L, const BcView &bc, uint8_t mode, uint8_t faces,
                                             int block, int bx, int by, int bz, bool abc, const LabDivs &dv, int row,
                                             int ny, int gy, int zi0, int nlo, int zhi, int z0, int E0, int E1)
{
    const int n0 = L.n[0], n1 = L.n[1], n2 = L.n[2];
    int y, z; // lab coordinates of the row
    if (row < ny) {
        const int zp = dv.gy.div(row), g = row - zp * gy;
        y = g < L.lo[1] ? g : g + n1;
        z = zi0 + zp;
    } else {
        const int rr = row - ny, zp = dv.n1.div(rr);
        y = rr - zp * n1 + L.lo[1];
        z = zp < nlo ? z0 + zp : zhi + (zp - nlo);
    }
    const int q1 = y - L.lo[1], q2 = z - L.lo[2];
    const int r1 = q1 < 0 ? -1 : (q1 >= n1 ? 1 : 0), r2 = q2 < 0 ? -1 : (q2 >= n2 ? 1 : 0);
    const int crossed = (r1 ? (r1 < 0 ? 4 : 8) : 0) | (r2 ? (r2 < 0 ? 16 : 32) : 0);
    RowSrc<T> R;
    if (faces & crossed) {
        lab_resolve<T, false>(L, bc, mode, block, bx, by, bz, 0, q1, q2, abc, R.s);
    } else {
        int nby = by + r1, nbz = bz + r2;
        nby = nby < 0 ? nby + L.nb[1] : (nby >= L.nb[1] ? nby - L.nb[1] : nby);
        nbz = nbz < 0 ? nbz + L.nb[2] : (nbz >= L.nb[2] ? nbz - L.nb[2] : nbz);
        R.s.kind = 2;
        R.s.idx = (int64_t)(bx + L.nb[0] * (nby + L.nb[1] * nbz)) * L.bstride + n0 * ((q1 - r1 * n1) + n1 * (q2 - r2 * n2));
    }
    R.dst = L.lo[0] + E0 * (y + E1 * z);
    return R;
}

// Lab planes [z0, z1) of a CTA's slab: the planes inside the block
// [zi0, zi0 + nin), nlo z-ghost planes below them and the z-ghost planes
// from zhi up (nghost in all).
struct SlabPlanes {
    int zi0, nin, nlo, zhi, nghost;
};
__host__ __device__ __forceinline__ int imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ SlabPlanes slab_planes(const LabGeom &L, int z0, int z1)
{
    SlabPlanes P;
    P.zi0 = imax(z0, L.lo[2]);
    P.nin = imax(0, imin(z1, L.lo[2] + L.n[2]) - P.zi0);
    P.nlo = imax(0, imin(z1, L.lo[2]) - z0);
    P.zhi = imax(z0, L.lo[2] + L.n[2]);
    P.nghost = P.nlo + imax(0, z1 - P.zhi);
    return P;
}

// one cell's source stored (kind 0: nothing)
template <typename T>
__device__ __forceinline__ void lab_store1(const T *__restrict__ comp, const LabSource<T> &s, int dst, T *__restrict__ o)
{
    if (dst < 0 || s.kind == 0) return;
    T x = s.kind == 2 ? comp[s.idx] : s.v;
    if (s.kind == 2) {
        if (s.nsign > 2) x = s.s2 * x;
        if (s.nsign > 1) x = s.s1 * x;
        if (s.nsign > 0) x = s.s0 * x;
    }
    o[dst] = x;
}

// Cell grids with non-tensorial labs whose ghost rows (classes 2 and 3
// below) fit in shared memory (kRows per slab), the common case: the
// one-pass form.  It is a kernel of its own so that the general form's
// per-class loops do not set its register count (it holds none of their
// spill slots and runs at kRowsCtas CTAs per SM).
template <typename T>
__global__ void __launch_bounds__(256, kRowsCtas)
    lab_fill_rows_kernel(const T *__restrict__ comp, LabGeom L, BcView bc, int block_begin, int pz, LabDivs dv,
                         int apply_bc, int bulk, int *err, T *__restrict__ out)
{
    const int n0 = L.n[0], n1 = L.n[1];
    const int E0 = n0 + L.lo[0] + L.hi[0];
    const int E1 = n1 + L.lo[1] + L.hi[1];
    const int E2 = L.n[2] + L.lo[2] + L.hi[2];
    // one CTA per (slab, block): x the slab, so that a block's slabs run
    // together (CTAs start in the order of their linear index) and the ghost
    // planes read from a block's z neighbours are read close in time to the
    // neighbours' own CTAs, while they are in L2
    const int bl = blockIdx.y, z0 = blockIdx.x * pz;
    const int block = block_begin + bl;
    const int bx = block % L.nb[0];
    const int by = (block / L.nb[0]) % L.nb[1];
    const int bz = block / (L.nb[0] * L.nb[1]);
    const uint8_t mode = bc.mode[block];
    const uint8_t faces = bc.faces[block];
    const bool abc = apply_bc != 0;
    const SlabPlanes P = slab_planes(L, z0, min(z0 + pz, E2));
    const int zi0 = P.zi0, nin = P.nin, nlo = P.nlo, zhi = P.zhi;
    const int gx = L.lo[0] + L.hi[0], gy = L.lo[1] + L.hi[1];
    T *o = out + (int64_t)bl * E0 * E1 * E2;
    const int ny = nin * gy, nrows = ny + P.nghost * n1;
    __shared__ __align__(16) unsigned char rows_raw[kRows * sizeof(RowSrc<T>)];
    RowSrc<T> *rows = reinterpret_cast<RowSrc<T> *>(rows_raw);
    // One pass over all three kinds of plain copies, KLM loads in flight
    // per thread: the block's own cells, the x ghosts behind clear faces
    // and the rows (classes 2, 3) whose source is a plain cell run.  The
    // rows are resolved first; cells that need BC chains or skips are
    // left to a second pass.
    const int A = nin * n1 * n0, B = nin * n1 * gx, tot = A + B + nrows * n0;
    const int64_t bbase = (int64_t)block * L.bstride + (int64_t)n0 * n1 * (zi0 - L.lo[2]);
    // The block's own planes of the slab are one contiguous run of
    // memory: with room in the dynamic shared memory (`bulk` bytes) one
    // bulk copy brings them while the threads work on the ghosts.
    extern __shared__ __align__(128) unsigned char lab_bulk[];
    __shared__ __align__(8) uint64_t bulk_bar;
    const uint32_t bytes0 = (uint32_t)A * (uint32_t)sizeof(T);
    const bool use_bulk = A > 0 && bytes0 <= (uint32_t)bulk && ((uint32_t)(n0 * n1) * sizeof(T)) % 16 == 0;
    if (use_bulk && threadIdx.x == 0) {
        mbar_init(&bulk_bar, 1);
        fence_mbar_init();
        mbar_arrive_expect_tx(&bulk_bar, bytes0);
        bulk_g2s(lab_bulk, comp + bbase, bytes0, &bulk_bar);
    }
    for (int j = threadIdx.x; j < nrows; j += blockDim.x)
        rows[j] = lab_row<T>(L, bc, mode, faces, block, bx, by, bz, abc, dv, j, ny, gy, zi0, nlo, zhi, z0, E0, E1);
    __syncthreads(); // the rows, and the barrier's initialisation
    bool deferred = false;
    const int base = use_bulk ? A : 0; // the first item of the pass
    for (int t0 = base + threadIdx.x; t0 < tot; t0 += KLM * blockDim.x) {
        int64_t idx[KLM];
        int dst[KLM];
#pragma unroll
        for (int k = 0; k < KLM; ++k) {
            const int t = t0 + k * blockDim.x;
            dst[k] = -1;
            idx[k] = 0;
            if (t < A) {
                const int r = dv.n0.div(t), zp = dv.n1.div(r);
                dst[k] = (t - r * n0 + L.lo[0]) + E0 * ((r - zp * n1 + L.lo[1]) + E1 * (zi0 + zp));
                idx[k] = bbase + t;
            } else if (t < A + B) {
                int x, y, z;
                class1_cell(dv, t - A, gx, n0, n1, L.lo[0], L.lo[1], zi0, x, y, z);
                const int q0 = x - L.lo[0], r0 = q0 < 0 ? -1 : 1;
                if (faces & (r0 < 0 ? 1 : 2)) {
                    deferred = true;
                } else {
                    const int nbx = bx + r0 < 0 ? bx + r0 + L.nb[0] : (bx + r0 >= L.nb[0] ? bx + r0 - L.nb[0] : bx + r0);
                    dst[k] = x + E0 * (y + E1 * z);
                    idx[k] = (int64_t)(nbx + L.nb[0] * (by + L.nb[1] * bz)) * L.bstride + (q0 - r0 * n0) +
                             n0 * ((y - L.lo[1]) + n1 * (z - L.lo[2]));
                }
            } else if (t < tot) {
                const int u = t - A - B, j = dv.n0.div(u), x = u - j * n0;
                const RowSrc<T> &R = rows[j];
                if (R.s.kind == 2 && R.s.nsign == 0) {
                    dst[k] = R.dst + x;
                    idx[k] = R.s.idx + x;
                } else {
                    deferred = true;
                }
            }
        }
        T v[KLM];
#pragma unroll
        for (int k = 0; k < KLM; ++k)
            if (dst[k] >= 0) v[k] = comp[idx[k]];
#pragma unroll
        for (int k = 0; k < KLM; ++k)
            if (dst[k] >= 0) o[dst[k]] = v[k];
    }
    if (use_bulk) {
        // the block's cells from shared memory
        if (!mbar_wait_bounded_sleep(&bulk_bar, 0, 200)) {
            // record the error; a second bounded wait keeps the copy from
            // landing in a later CTA's shared memory
            if (threadIdx.x == 0 && err) atomicExch(err, kDevErrTimeout);
            mbar_wait_bounded_sleep(&bulk_bar, 0, 200);
        } else {
            const T *sb = reinterpret_cast<const T *>(lab_bulk);
            for (int t0 = threadIdx.x; t0 < A; t0 += KLM * blockDim.x) {
#pragma unroll
                for (int k = 0; k < KLM; ++k) {
                    const int t = t0 + k * blockDim.x;
                    if (t < A) {
                        const int r = dv.n0.div(t), zp = dv.n1.div(r);
                        o[(t - r * n0 + L.lo[0]) + E0 * ((r - zp * n1 + L.lo[1]) + E1 * (zi0 + zp))] = sb[t];
                    }
                }
            }
        }
    }
    if (deferred) {
        // the second pass: the same items of this thread
        const int nt = (int)blockDim.x;
        for (int t = A + ((((int)threadIdx.x + base - A) % nt) + nt) % nt; t < tot; t += nt) {
            LabSource<T> src[1];
            int dst[1] = {-1};
            if (t < A + B) {
                int x, y, z;
                class1_cell(dv, t - A, gx, n0, n1, L.lo[0], L.lo[1], zi0, x, y, z);
                if (!(faces & (x < L.lo[0] ? 1 : 2))) continue;
                lab_resolve<T, false>(L, bc, mode, block, bx, by, bz, x - L.lo[0], y - L.lo[1], z - L.lo[2], abc,
                                      src[0]);
                dst[0] = x + E0 * (y + E1 * z);
            } else {
                const int u = t - A - B, j = dv.n0.div(u), x = u - j * n0;
                const RowSrc<T> &R = rows[j];
                if (R.s.kind == 2 && R.s.nsign == 0) continue;
                src[0] = R.s;
                src[0].idx += x;
                dst[0] = R.dst + x;
            }
            lab_store1<T>(comp, src[0], dst[0], o);
        }
    }
}

// Cell grids: the CTA's slab of lab planes as four classes of cells, each
// walked by all threads so that a warp's cells take the same path:
//   0  the block's own cells (planes and rows inside): plain copies;
//   1  the x ghosts of those rows;
//   2  the y-ghost rows of inside planes (x inside, or the whole row when
//      tensorial);
//   3  the z-ghost planes (x, y inside, or the whole plane when tensorial).
// Class 1-3 cells beyond faces that carry no BC and no skipped neighbour are
// the periodic neighbour's cells (closed form); the others take lab_resolve
// (skips, BC chains).  Without tensorial ghosts, classes 2 and 3 are walked
// as rows resolved once each.  Cells no class lists are the edges and corners of a
// non-tensorial lab, which the reference leaves undefined.
template <typename T>
__global__ void __launch_bounds__(256, 4)
    lab_fill_kernel(const T *__restrict__ comp, LabGeom L, BcView bc, int block_begin, int pz, LabDivs dv,
                    int apply_bc, T *__restrict__ out)
{
    const int n0 = L.n[0], n1 = L.n[1], n2 = L.n[2];
    const int E0 = n0 + L.lo[0] + L.hi[0];
    const int E1 = n1 + L.lo[1] + L.hi[1];
    const int E2 = n2 + L.lo[2] + L.hi[2];
    const int bl = blockIdx.y, z0 = blockIdx.x * pz; // block-major, as lab_fill_rows_kernel
    const int z1 = min(z0 + pz, E2);
    const int block = block_begin + bl;
    const int bx = block % L.nb[0];
    const int by = (block / L.nb[0]) % L.nb[1];
    const int bz = block / (L.nb[0] * L.nb[1]);
    const uint8_t mode = bc.mode[block];
    // faces of the block that carry a BC (other than Base) or a skipped
    // neighbour: cells beyond them take the full resolution
    const uint8_t faces = bc.faces[block];
    const bool abc = apply_bc != 0, tens = L.tensorial != 0;
    // planes of the slab inside the block, and its z-ghost planes below / above
    const SlabPlanes P = slab_planes(L, z0, z1);
    const int zi0 = P.zi0, nin = P.nin, nlo = P.nlo, zhi = P.zhi, nghost = P.nghost;
    const int wrow = tens ? E0 : n0, wpl = tens ? E1 : n1;
    const int gx = L.lo[0] + L.hi[0], gy = L.lo[1] + L.hi[1];
    T *o = out + (int64_t)bl * E0 * E1 * E2;
    const int ny = nin * gy, nrows = ny + nghost * n1;
    __shared__ __align__(16) unsigned char rows_raw[kRows * sizeof(RowSrc<T>)];
    RowSrc<T> *rows = reinterpret_cast<RowSrc<T> *>(rows_raw);
    // class 0: rows of the block's own cells, plain copies (KL loads in flight)
    {
        const T *blk = comp + (int64_t)block * L.bstride + (int64_t)n0 * n1 * (zi0 - L.lo[2]);
        T *ob = o + L.lo[0] + E0 * (L.lo[1] + E1 * zi0);
        const int cnt = nin * n1 * n0;
        if ((n0 & 1) == 0) {
            // pairs of cells along x: one 2-element load (the block's rows
            // start on 2-element boundaries), two stores (lab rows need not)
            using V = typename Vec2<T>::type;
            const V *blk2 = reinterpret_cast<const V *>(blk);
            const int cnt2 = cnt >> 1;
            for (int p0 = threadIdx.x; p0 < cnt2; p0 += KL0 * blockDim.x) {
                V v[KL0];
                int d[KL0];
#pragma unroll
                for (int k = 0; k < KL0; ++k) {
                    const int p = p0 + k * blockDim.x, t = 2 * p;
                    const int r = dv.n0.div(t), zp = dv.n1.div(r);
                    d[k] = p < cnt2 ? (t - r * n0) + E0 * ((r - zp * n1) + E1 * zp) : -1;
                    if (p < cnt2) v[k] = blk2[p];
                }
#pragma unroll
                for (int k = 0; k < KL0; ++k)
                    if (d[k] >= 0) {
                        ob[d[k]] = v[k].x;
                        ob[d[k] + 1] = v[k].y;
                    }
            }
        } else {
            for (int t0 = threadIdx.x; t0 < cnt; t0 += KL * blockDim.x) {
                T v[KL];
                int d[KL];
#pragma unroll
                for (int k = 0; k < KL; ++k) {
                    const int t = t0 + k * blockDim.x;
                    const int r = dv.n0.div(t), zp = dv.n1.div(r);
                    d[k] = t < cnt ? (t - r * n0) + E0 * ((r - zp * n1) + E1 * zp) : -1;
                    v[k] = t < cnt ? blk[t] : T(0);
                }
#pragma unroll
                for (int k = 0; k < KL; ++k)
                    if (d[k] >= 0) ob[d[k]] = v[k];
            }
        }
    }
    // classes 1-3 cell by cell; without tensorial ghosts, classes 2 and 3 go
    // by rows below
#pragma unroll 1
    for (int cls = 1; cls < (tens ? 4 : 2); ++cls) {
        const int cnt = cls == 1 ? nin * n1 * gx : (cls == 2 ? nin * gy * wrow : nghost * wpl * wrow);
        for (int t0 = threadIdx.x; t0 < cnt; t0 += KL * blockDim.x) {
            LabSource<T> src[KL];
            int dst[KL];
#pragma unroll
            for (int k = 0; k < KL; ++k) {
                const int t = t0 + k * blockDim.x;
                dst[k] = -1;
                if (t >= cnt) continue;
                int x, y, z; // lab coordinates
                if (cls == 1) {
                    const int r = dv.gx.div(t), zp = dv.n1.div(r);
                    const int g = t - r * gx;
                    x = g < L.lo[0] ? g : g + n0;
                    y = r - zp * n1 + L.lo[1];
                    z = zi0 + zp;
                } else if (cls == 2) {
                    const int r = dv.wrow.div(t), zp = dv.gy.div(r);
                    const int g = r - zp * gy;
                    x = t - r * wrow + (tens ? 0 : L.lo[0]);
                    y = g < L.lo[1] ? g : g + n1;
                    z = zi0 + zp;
                } else {
                    const int r = dv.wrow.div(t), zp = dv.wpl.div(r);
                    x = t - r * wrow + (tens ? 0 : L.lo[0]);
                    y = r - zp * wpl + (tens ? 0 : L.lo[1]);
                    z = zp < nlo ? z0 + zp : zhi + (zp - nlo);
                }
                dst[k] = x + E0 * (y + E1 * z);
                {
                    const int q0 = x - L.lo[0], q1 = y - L.lo[1], q2 = z - L.lo[2];
                    const int r0 = q0 < 0 ? -1 : (q0 >= n0 ? 1 : 0), r1 = q1 < 0 ? -1 : (q1 >= n1 ? 1 : 0),
                              r2 = q2 < 0 ? -1 : (q2 >= n2 ? 1 : 0);
                    const int crossed = (r0 ? (r0 < 0 ? 1 : 2) : 0) | (r1 ? (r1 < 0 ? 4 : 8) : 0) |
                                        (r2 ? (r2 < 0 ? 16 : 32) : 0);
                    if (faces & crossed) {
                        lab_resolve<T, false>(L, bc, mode, block, bx, by, bz, q0, q1, q2, abc, src[k]);
                    } else {
                        // beyond clear faces only: no BC covers the cell, and it is the
                        // periodic neighbour's cell (as lab_resolve gives it)
                        int nbx = bx + r0, nby = by + r1, nbz = bz + r2;
                        nbx = nbx < 0 ? nbx + L.nb[0] : (nbx >= L.nb[0] ? nbx - L.nb[0] : nbx);
                        nby = nby < 0 ? nby + L.nb[1] : (nby >= L.nb[1] ? nby - L.nb[1] : nby);
                        nbz = nbz < 0 ? nbz + L.nb[2] : (nbz >= L.nb[2] ? nbz - L.nb[2] : nbz);
                        src[k].kind = 2;
                        src[k].idx = (int64_t)(nbx + L.nb[0] * (nby + L.nb[1] * nbz)) * L.bstride + (q0 - r0 * n0) +
                                     n0 * ((q1 - r1 * n1) + n1 * (q2 - r2 * n2));
                    }
                }
            }
            lab_store<T>(comp, src, dst, o);
        }
    }
    if (tens) return;
    // Classes 2 and 3 of a non-tensorial lab by rows: a y-ghost row of an
    // inside plane, or a row of a z-ghost plane, holds the n0 cells with x
    // inside the block, and x passes through every step of the resolution
    // unchanged (no x BC covers them, the neighbour is the same), so the
    // cells of a row are the row's first cell's source shifted by x (or its
    // one value).  One thread resolves a row's first cell into shared
    // memory; all threads then copy the rows' cells.
#pragma unroll 1
    for (int rb = 0; rb < nrows; rb += kRows) {
        const int nr = min(kRows, nrows - rb);
        __syncthreads(); // the previous rows are copied
        for (int j = threadIdx.x; j < nr; j += blockDim.x)
            rows[j] = lab_row<T>(L, bc, mode, faces, block, bx, by, bz, abc, dv, rb + j, ny, gy, zi0, nlo, zhi, z0, E0,
                                 E1);
        __syncthreads();
        const int cells = nr * n0;
        for (int t0 = threadIdx.x; t0 < cells; t0 += KL * blockDim.x) {
            LabSource<T> src[KL];
            int dst[KL];
#pragma unroll
            for (int k = 0; k < KL; ++k) {
                const int t = t0 + k * blockDim.x;
                dst[k] = -1;
                if (t >= cells) continue;
                const int j = dv.n0.div(t), x = t - j * n0;
                src[k] = rows[j].s;
                src[k].idx += x;
                dst[k] = rows[j].dst + x;
            }
            lab_store<T>(comp, src, dst, o);
        }
    }
}

template <typename T>
static cn_status launch_fill(cn_grid *g, int comp, const cn_stencil *s, int b0, int cnt,
                             int apply_bc, void *d_labs, cudaStream_t st)
{
    const LabGeom L = make_geom(g, s);
    const T *src = reinterpret_cast<const T *>(g->d_data) + (size_t)comp * g->comp_stride;
    const int64_t E0 = L.n[0] + L.lo[0] + L.hi[0], E1 = L.n[1] + L.lo[1] + L.hi[1], E2 = L.n[2] + L.lo[2] + L.hi[2];
    const int64_t plane = E0 * E1;
    if (plane * E2 >= (int64_t(1) << 31))
        return fail(CN_ERR_UNSUPPORTED, "cn_lab_fill: labs of 2^31 cells or more");
    // planes per CTA: about kCellsPerCta cells
    int pz = (int)std::max<int64_t>(1, std::min<int64_t>(E2, kCellsPerCta / plane));
    const bool grow = L.grow[0] || L.grow[1] || L.grow[2];
    // The one-pass kernel holds a slab's ghost rows (classes 2, 3) in a
    // table of kRows: slabs of fewer planes until every slab's rows fit.
    auto rows_fit = [&](int p) {
        for (int z0 = 0; z0 < E2; z0 += p) {
            const SlabPlanes P = slab_planes(L, z0, (int)std::min<int64_t>(z0 + p, E2));
            if (P.nin * (L.lo[1] + L.hi[1]) + P.nghost * L.n[1] > kRows) return false;
        }
        return true;
    };
    bool rows_form = !grow && !L.tensorial;
    if (rows_form) {
        while (pz > 1 && !rows_fit(pz)) --pz;
        rows_form = rows_fit(pz);
    }
    const int64_t slabs = (E2 + pz - 1) / pz;
    if (slabs > 65535) return fail(CN_ERR_UNSUPPORTED, "cn_lab_fill: more than 65535 lab slabs per block");
    const int threads = plane * pz >= 1024 ? 256 : 128;
    LabDivs dv;
    dv.n0 = FastDiv((uint32_t)L.n[0]);
    dv.n1 = FastDiv((uint32_t)L.n[1]);
    dv.gx = FastDiv((uint32_t)(L.lo[0] + L.hi[0]));
    dv.wrow = FastDiv((uint32_t)(L.tensorial ? E0 : L.n[0]));
    dv.gy = FastDiv((uint32_t)(L.lo[1] + L.hi[1]));
    dv.wpl = FastDiv((uint32_t)(L.tensorial ? E1 : L.n[1]));
    // dynamic shared memory for the bulk copy of a slab's block planes
    const int64_t bulk = (int64_t)pz * L.n[0] * L.n[1] * (int64_t)sizeof(T);
    const int nbulk = rows_form && bulk <= kBulkBytes ? (int)bulk : 0;
    if (rows_form) {
        static DeviceOnce once;
        cn_status r = smem_opt_in(once, lab_fill_rows_kernel<T>, (size_t)kBulkBytes);
        if (r != CN_OK) return r;
    }
    // CTAs in block-major order: the slab along x, the block along y (a
    // block's slabs run together), at most 65535 blocks per launch
    for (int c0 = 0; c0 < cnt; c0 += 65535) {
        const dim3 grid((unsigned)slabs, (unsigned)std::min(65535, cnt - c0));
        T *out = reinterpret_cast<T *>(d_labs) + (int64_t)c0 * plane * E2;
        if (grow) {
            lab_fill_grow_kernel<T><<<grid, threads, 0, st>>>(src, L, bc_view(g, comp), b0 + c0, pz,
                                                              FastDiv((uint32_t)E0), FastDiv((uint32_t)plane),
                                                              apply_bc, out);
        } else if (rows_form) {
            lab_fill_rows_kernel<T><<<grid, threads, nbulk, st>>>(src, L, bc_view(g, comp), b0 + c0, pz, dv,
                                                                  apply_bc, nbulk, g->d_err, out);
        } else {
            lab_fill_kernel<T><<<grid, threads, 0, st>>>(src, L, bc_view(g, comp), b0 + c0, pz, dv, apply_bc, out);
        }
    }
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

} // namespace cn

using namespace cn;

extern "C" cn_status cn_lab_fill(cn_grid *g, int comp, const cn_stencil *s, int block_begin,
                                 int block_count, int apply_bc, void *d_labs, void *stream)
{
    if (!g) {
        return fail(CN_ERR_NOT_ALLOCATED, "FieldLab: can not load lab data when not allocated first");
    }
    if (comp < 0 || comp >= g->ncomp) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_lab_fill: bad component");
    }
    if (!d_labs) {
        return fail(CN_ERR_NOT_ALLOCATED, "FieldLab: can not load lab data when not allocated first");
    }
    cn_status st = check_lab(g, s);
    if (st != CN_OK) return st;
    if (block_begin < 0 || block_count < 0 || block_begin + (int64_t)block_count > g->nblocks) {
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_lab_fill: block range outside the grid");
    }
    if (block_count == 0) return CN_OK;
    cudaStream_t cs = as_stream(stream);
    st = sync_bc(g, cs);
    if (st != CN_OK) return st;
    switch (g->dtype) {
    case CN_FLOAT64:
        return launch_fill<double>(g, comp, s, block_begin, block_count, apply_bc, d_labs, cs);
    case CN_FLOAT32:
        return launch_fill<float>(g, comp, s, block_begin, block_count, apply_bc, d_labs, cs);
    case CN_INT32:
        return launch_fill<int32_t>(g, comp, s, block_begin, block_count, apply_bc, d_labs, cs);
    }
    return fail(CN_ERR_UNSUPPORTED, "cn_lab_fill: dtype");
}
