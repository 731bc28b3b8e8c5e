// fd.cu -- K1: lab fill fused with the 2nd-order finite-difference stencils
// (7-point Laplacian, central gradient, divergence) and the ddx kernel ABI.
//
// Design (one CTA per z-slab tile of one block, N0 x N1 x TZ cells):
//   * the tile's inner cells are one contiguous range of the block (x-fastest
//     block storage), so a single 1-D TMA bulk copy (cp.async.bulk, mbarrier
//     completion, bounded wait) stages them into shared memory;
//   * while that copy is in flight the threads gather the six one-cell faces
//     of the tile with cn::lab_value (periodic neighbours, BC chain), i.e. the
//     lab of a stencil (-1,2) non-tensorial (Block/FieldLab.h:180-224);
//   * each thread then evaluates the stencil from shared memory and writes
//     coalesced rows of the output blocks.
// Arithmetic uses __d*_rn / __f*_rn intrinsics so nothing is contracted into
// an FMA: results are bit-identical to the reference loops compiled without
// contraction (Kernel/Laplacian/Laplacian.cpp:123-130,
// Kernel/Divergence/nova/nova.cpp:113-126, ISPC .../ddxGold.cpp:9-33).
#include <algorithm>

#include "cn_fastdiv.h"
#include "cn_internal.h"
#include "cn_tma.cuh"

namespace cn {

template <typename T> struct Arith;
template <> struct Arith<double> {
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
};
template <> struct Arith<float> {
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
};

enum FdOp { kLap = 0, kGrad = 1, kLapGrad = 2, kDiv = 3 };

template <typename T> struct FdParams {
    const T *in[3];  // input component bases (kDiv: 3 components)
    BcView bc[3];
    LabGeom L;
    T *lap;          // kLap / kLapGrad / kDiv output component base
    T *grad;         // kGrad / kLapGrad: first of 3 components
    int64_t out_cstride;
    T ih[3], ih2[3];
    int TZ;
    int use_bulk;
    int *err;
    FastDiv dv0, dv1, dv01, dvh; // N0, N1, N0 * N1, N0 / 2: cell index -> (x, y, z) without divisions
};

// Shared-memory tile of one component: inner cells + the six faces.
template <typename T> struct Tile {
    T *in, *xlo, *xhi, *ylo, *yhi, *zlo, *zhi;
};

// Every array of a tile starts on a multiple of 4 elements, so each one (and
// the next component's tile) is 16-byte aligned for the bulk copy and the
// two-element vector loads.
__host__ __device__ __forceinline__ size_t pad4(size_t n) { return (n + 3) & ~(size_t)3; }

__host__ __device__ __forceinline__ size_t tile_elems(int N0, int N1, int TZ)
{
    return pad4((size_t)N0 * N1 * TZ) + 2 * (pad4((size_t)N1 * TZ) + pad4((size_t)N0 * TZ) + pad4((size_t)N0 * N1));
}

template <typename T>
__device__ __forceinline__ Tile<T> carve(T *base, int N0, int N1, int TZ)
{
    Tile<T> t;
    t.in = base;
    t.xlo = t.in + pad4((size_t)N0 * N1 * TZ);
    t.xhi = t.xlo + pad4((size_t)N1 * TZ);
    t.ylo = t.xhi + pad4((size_t)N1 * TZ);
    t.yhi = t.ylo + pad4((size_t)N0 * TZ);
    t.zlo = t.yhi + pad4((size_t)N0 * TZ);
    t.zhi = t.zlo + pad4((size_t)N0 * N1);
    return t;
}

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// Outputs of one cell from its six neighbours (kDiv: x neighbours of the
// first component, y of the second, z of the third; c0 unused).
template <typename T, int OP>
__device__ __forceinline__ void cell_eval(const FdParams<T> &p, T c0, T xp, T xm, T yp, T ym, T zp, T zm,
                                          T &lap, T &g0, T &g1, T &g2)
{
    using A = Arith<T>;
    if (OP == kDiv) {
        const T t0 = A::mul(A::sub(xp, xm), p.ih[0]);
        const T t1 = A::mul(A::sub(yp, ym), p.ih[1]);
        const T t2 = A::mul(A::sub(zp, zm), p.ih[2]);
        lap = A::mul(T(0.5), A::add(A::add(t0, t1), t2));
        return;
    }
    if (OP == kLap || OP == kLapGrad) {
        const T c2 = A::mul(T(2), c0);
        const T ddx = A::mul(p.ih2[0], A::add(A::sub(xp, c2), xm));
        const T ddy = A::mul(p.ih2[1], A::add(A::sub(yp, c2), ym));
        const T ddz = A::mul(p.ih2[2], A::add(A::sub(zp, c2), zm));
        lap = A::add(A::add(ddx, ddy), ddz);
    }
    if (OP == kGrad || OP == kLapGrad) {
        g0 = A::mul(T(0.5), A::mul(A::sub(xp, xm), p.ih[0]));
        g1 = A::mul(T(0.5), A::mul(A::sub(yp, ym), p.ih[1]));
        g2 = A::mul(T(0.5), A::mul(A::sub(zp, zm), p.ih[2]));
    }
}

// Stages one lab cell of a tile face into shared memory.  Cells inside the
// block, and every cell of a block without BCs or skip flags (lab mode byte
// 0: the periodic neighbour from the table snb, index (r0+1) + 3 (r1+1) +
// 9 (r2+1)), are asynchronous copies (cp.async), so all of a thread's face
// loads are in flight at once alongside the bulk copy of the interior; the
// others are resolved with cn::lab_value.  Undefined lab cells (never read by
// these stencils unless the BC set-up leaves a face undefined) are zero.
template <typename T>
__device__ __forceinline__ void face_cell(const T *comp, const LabGeom &L, const BcView &bc, bool plain,
                                          const int *snb, int block, int bx, int by, int bz, int x, int y, int z,
                                          T *dst)
{
    const int r0 = x < 0 ? -1 : (x >= L.n[0] ? 1 : 0), r1 = y < 0 ? -1 : (y >= L.n[1] ? 1 : 0),
              r2 = z < 0 ? -1 : (z >= L.n[2] ? 1 : 0);
    if (plain || (r0 | r1 | r2) == 0) {
        const int sb = snb[(r0 + 1) + 3 * (r1 + 1) + 9 * (r2 + 1)];
        const T *src = comp + (int64_t)sb * L.bstride + (x - r0 * L.n[0]) +
                       (int64_t)L.n[0] * ((y - r1 * L.n[1]) + (int64_t)L.n[1] * (z - r2 * L.n[2]));
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src),
                     "n"((int)sizeof(T))
                     : "memory");
        return;
    }
    T v;
    if (!lab_value<T>(comp, L, bc, block, bx, by, bz, x, y, z, true, v))
        v = T(0);
    *dst = v;
}

__device__ __forceinline__ void fd_cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Gathers the faces selected by mask (bit 0: x, 1: y, 2: z) of the tile that
// starts at z0; the caller waits for the copies (fd_cp_async_wait_all) and
// synchronises the CTA before reading them.
template <typename T>
__device__ __forceinline__ void gather_faces(const T *comp, const LabGeom &L, const BcView &bc,
                                             int block, int bx, int by, int bz, int z0, int TZ,
                                             const Tile<T> &t, unsigned mask, const int *snb,
                                             const FastDiv &dv0, const FastDiv &dv1)
{
    const int N0 = L.n[0], N1 = L.n[1];
    const int nth = blockDim.x;
    const bool plain = __ldg(bc.mode + block) == 0;
    if (mask & 1u) {
        const int m = N1 * TZ;
        for (int i = threadIdx.x; i < 2 * m; i += nth) {
            const int side = i >= m, r = side ? i - m : i;
            const int z = dv1.div(r), y = r - z * N1;
            face_cell<T>(comp, L, bc, plain, snb, block, bx, by, bz, side ? N0 : -1, y, z0 + z,
                         (side ? t.xhi : t.xlo) + r);
        }
    }
    if (mask & 2u) {
        const int m = N0 * TZ;
        for (int i = threadIdx.x; i < 2 * m; i += nth) {
            const int side = i >= m, r = side ? i - m : i;
            const int z = dv0.div(r), x = r - z * N0;
            face_cell<T>(comp, L, bc, plain, snb, block, bx, by, bz, x, side ? N1 : -1, z0 + z,
                         (side ? t.yhi : t.ylo) + r);
        }
    }
    if (mask & 4u) {
        const int m = N0 * N1;
        for (int i = threadIdx.x; i < 2 * m; i += nth) {
            const int side = i >= m, r = side ? i - m : i;
            const int y = dv0.div(r), x = r - y * N0;
            face_cell<T>(comp, L, bc, plain, snb, block, bx, by, bz, x, y, side ? z0 + TZ : z0 - 1,
                         (side ? t.zhi : t.zlo) + r);
        }
    }
}

template <typename T, int OP>
__global__ void __launch_bounds__(256, 8) fd_kernel(FdParams<T> p)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw);
    T *base = reinterpret_cast<T *>(smem_raw + 128);
    const LabGeom &L = p.L;
    const int N0 = L.n[0], N1 = L.n[1], N2 = L.n[2];
    const int TZ = p.TZ;
    const int tiles_per_block = N2 / TZ;
    const int block = blockIdx.x / tiles_per_block;
    const int z0 = (blockIdx.x - block * tiles_per_block) * TZ;
    constexpr int NC = (OP == kDiv) ? 3 : 1;
    const size_t te = tile_elems(N0, N1, TZ);
    Tile<T> tl[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c)
        tl[c] = carve<T>(base + c * te, N0, N1, TZ);
    const uint32_t in_bytes = (uint32_t)((size_t)N0 * N1 * TZ * sizeof(T));
    const int64_t in_off = (int64_t)block * L.bstride + (int64_t)z0 * N0 * N1;
    // the interior's bulk copy goes out first; the barrier below publishes
    // the mbarrier's initialisation to the other threads
    if (p.use_bulk && threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
        mbar_arrive_expect_tx(bar, in_bytes * NC);
#pragma unroll
        for (int c = 0; c < NC; ++c)
            bulk_g2s(tl[c].in, p.in[c] + in_off, in_bytes, bar);
    }
    const int bx = block % L.nb[0];
    const int by = (block / L.nb[0]) % L.nb[1];
    const int bz = block / (L.nb[0] * L.nb[1]);
    __shared__ int snb[27]; // periodic neighbour blocks
    if (threadIdx.x < 27) {
        const int t = threadIdx.x;
        int nx = bx + t % 3 - 1, ny = by + (t / 3) % 3 - 1, nz = bz + t / 9 - 1;
        nx = nx < 0 ? nx + L.nb[0] : (nx >= L.nb[0] ? nx - L.nb[0] : nx);
        ny = ny < 0 ? ny + L.nb[1] : (ny >= L.nb[1] ? ny - L.nb[1] : ny);
        nz = nz < 0 ? nz + L.nb[2] : (nz >= L.nb[2] ? nz - L.nb[2] : nz);
        snb[t] = nx + L.nb[0] * (ny + L.nb[1] * nz);
    }
    if (!p.use_bulk) {
        const int m = N0 * N1 * TZ;
#pragma unroll
        for (int c = 0; c < NC; ++c)
            for (int i = threadIdx.x; i < m; i += blockDim.x)
                tl[c].in[i] = p.in[c][in_off + i];
    }
    __syncthreads(); // snb, mbarrier initialised
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        const unsigned mask = (OP == kDiv) ? (1u << c) : 7u;
        gather_faces<T>(p.in[c], L, p.bc[c], block, bx, by, bz, z0, TZ, tl[c], mask, snb, p.dv0, p.dv1);
    }
    fd_cp_async_wait_all();
    if (p.use_bulk) {
        if (!mbar_wait_bounded_sleep(bar, 0)) {
            atomicExch(p.err, kDevErrTimeout);
        }
    }
    __syncthreads();

    // x-even blocks: two neighbouring cells of a row per thread, with
    // two-element shared loads and global stores
    if ((N0 & 1) == 0) {
        using V = typename Vec2<T>::type;
        const int h0 = N0 >> 1;
        const int mp = h0 * N1 * TZ;
        const Tile<T> &a = tl[0], &b = tl[NC > 1 ? 1 : 0], &c = tl[NC > 2 ? 2 : 0];
        for (int j = threadIdx.x; j < mp; j += blockDim.x) {
            const int row = p.dvh.div(j), x = 2 * (j - row * h0); // row = y + N1 z
            const int z = p.dv1.div(row), y = row - z * N1;
            const int i = x + N0 * row;
            const int64_t o = in_off + i;
            const V ac = *reinterpret_cast<const V *>(a.in + i);
            const T xm = x > 0 ? a.in[i - 1] : a.xlo[row];
            const T xp = x + 2 < N0 ? a.in[i + 2] : a.xhi[row];
            const V yp = *reinterpret_cast<const V *>(y + 1 < N1 ? b.in + i + N0 : b.yhi + x + N0 * z);
            const V ym = *reinterpret_cast<const V *>(y > 0 ? b.in + i - N0 : b.ylo + x + N0 * z);
            const V zp = *reinterpret_cast<const V *>(z + 1 < TZ ? c.in + i + N0 * N1 : c.zhi + x + N0 * y);
            const V zm = *reinterpret_cast<const V *>(z > 0 ? c.in + i - N0 * N1 : c.zlo + x + N0 * y);
            T l0 = T(0), l1 = T(0), g00 = T(0), g01 = T(0), g02 = T(0), g10 = T(0), g11 = T(0), g12 = T(0);
            cell_eval<T, OP>(p, ac.x, ac.y, xm, yp.x, ym.x, zp.x, zm.x, l0, g00, g01, g02);
            cell_eval<T, OP>(p, ac.y, xp, ac.x, yp.y, ym.y, zp.y, zm.y, l1, g10, g11, g12);
            if (OP == kLap || OP == kLapGrad || OP == kDiv)
                *reinterpret_cast<V *>(p.lap + o) = V{l0, l1};
            if (OP == kGrad || OP == kLapGrad) {
                *reinterpret_cast<V *>(p.grad + o) = V{g00, g10};
                *reinterpret_cast<V *>(p.grad + o + p.out_cstride) = V{g01, g11};
                *reinterpret_cast<V *>(p.grad + o + 2 * p.out_cstride) = V{g02, g12};
            }
        }
        return;
    }
    const int m = N0 * N1 * TZ;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int z = p.dv01.div(i), r = i - z * (N0 * N1);
        const int y = p.dv0.div(r), x = r - y * N0;
        const int64_t o = in_off + i;
        const Tile<T> &a = tl[0], &b = tl[NC > 1 ? 1 : 0], &c = tl[NC > 2 ? 2 : 0];
        const T c0 = a.in[i];
        const T xp = x + 1 < N0 ? a.in[i + 1] : a.xhi[y + N1 * z];
        const T xm = x > 0 ? a.in[i - 1] : a.xlo[y + N1 * z];
        const T yp = y + 1 < N1 ? b.in[i + N0] : b.yhi[x + N0 * z];
        const T ym = y > 0 ? b.in[i - N0] : b.ylo[x + N0 * z];
        const T zp = z + 1 < TZ ? c.in[i + N0 * N1] : c.zhi[x + N0 * y];
        const T zm = z > 0 ? c.in[i - N0 * N1] : c.zlo[x + N0 * y];
        T l = T(0), g0 = T(0), g1 = T(0), g2 = T(0);
        cell_eval<T, OP>(p, c0, xp, xm, yp, ym, zp, zm, l, g0, g1, g2);
        if (OP == kLap || OP == kLapGrad || OP == kDiv) p.lap[o] = l;
        if (OP == kGrad || OP == kLapGrad) {
            p.grad[o] = g0;
            p.grad[o + p.out_cstride] = g1;
            p.grad[o + 2 * p.out_cstride] = g2;
        }
    }
}

static size_t fd_smem_bytes(int N0, int N1, int TZ, size_t es, int nc)
{
    return 128 + tile_elems(N0, N1, TZ) * es * nc;
}

// z-slab height: the largest divisor of N2 whose tile fits the budget and
// holds at most 2048 cells (more, smaller CTAs balance the SMs and overlap
// the staging of one tile with the stencil of another); at least 1.
static int pick_tz(int N0, int N1, int N2, size_t es, int nc, size_t budget)
{
    for (int tz = N2; tz >= 1; --tz) {
        if (N2 % tz) continue;
        if (fd_smem_bytes(N0, N1, tz, es, nc) > budget) continue;
        if (tz > 1 && (size_t)N0 * N1 * tz > 2048) continue;
        return tz;
    }
    return 0;
}

static cn_status check_out(const cn_grid *in, const cn_grid *out, int out_comp, int ncomp_out)
{
    if (!out) return fail(CN_ERR_INVALID_ARGUMENT, "output grid is NULL");
    if (out->nblocks != in->nblocks || out->n[0] != in->n[0] || out->n[1] != in->n[1] ||
        out->n[2] != in->n[2] || out->dtype != in->dtype)
        return fail(CN_ERR_SIZE_MISMATCH, "Cartesian: Can not assign two grids of unequal size.");
    if (out_comp < 0 || out_comp + ncomp_out > out->ncomp)
        return fail(CN_ERR_INVALID_ARGUMENT, "output component out of range");
    return CN_OK;
}

template <typename T, int OP>
static cn_status launch_fd(cn_grid *u, int comp, cn_grid *o1, int c1, cn_grid *o2, int c2,
                           cudaStream_t st)
{
    cn_stencil s = {{-1, -1, -1}, {2, 2, 2}, 0};
    cn_status stt = check_lab(u, &s);
    if (stt != CN_OK) return stt;
    stt = sync_bc(u, st);
    if (stt != CN_OK) return stt;
    FdParams<T> p = {};
    p.L = make_geom(u, &s);
    const int NC = OP == kDiv ? 3 : 1;
    for (int c = 0; c < NC; ++c) {
        p.in[c] = reinterpret_cast<const T *>(u->d_data) + (size_t)(comp + c) * u->comp_stride;
        p.bc[c] = bc_view(u, comp + c);
    }
    if (o1) p.lap = reinterpret_cast<T *>(o1->d_data) + (size_t)c1 * o1->comp_stride;
    if (o2) {
        p.grad = reinterpret_cast<T *>(o2->d_data) + (size_t)c2 * o2->comp_stride;
        p.out_cstride = o2->comp_stride;
    }
    for (int d = 0; d < 3; ++d) {
        p.ih[d] = (T)(1. / u->h[d]);
        p.ih2[d] = (T)(1. / (u->h[d] * u->h[d]));
    }
    const int N0 = u->n[0], N1 = u->n[1], N2 = u->n[2];
    const int tz = pick_tz(N0, N1, N2, sizeof(T), NC, 100 * 1024);
    if (tz == 0) return fail(CN_ERR_UNSUPPORTED, "block too large for the fused stencil tile");
    p.TZ = tz;
    p.dv0 = FastDiv((uint32_t)N0);
    p.dv1 = FastDiv((uint32_t)N1);
    p.dv01 = FastDiv((uint32_t)(N0 * N1));
    p.dvh = FastDiv((uint32_t)(N0 / 2 > 0 ? N0 / 2 : 1));
    const size_t tile_bytes = (size_t)N0 * N1 * tz * sizeof(T);
    p.use_bulk = (tile_bytes % 16 == 0) && ((u->block_stride * sizeof(T)) % 16 == 0);
    p.err = u->d_err;
    const size_t smem = fd_smem_bytes(N0, N1, tz, sizeof(T), NC);
    CN_CUDA_TRY(cudaFuncSetAttribute(fd_kernel<T, OP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
    // eight 256-thread CTAs per SM fit the registers (32 per thread): ask for
    // the shared-memory carve-out that lets their tiles fit as well
    CN_CUDA_TRY(cudaFuncSetAttribute(fd_kernel<T, OP>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
    const int64_t ctas = (int64_t)u->nblocks * (N2 / tz);
    fd_kernel<T, OP><<<(unsigned)ctas, 256, smem, st>>>(p);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

template <int OP>
static cn_status dispatch_fd(cn_grid *u, int comp, int ncin, cn_grid *o1, int c1, cn_grid *o2,
                             int c2, void *stream)
{
    if (!u) return fail(CN_ERR_INVALID_ARGUMENT, "input grid is NULL");
    if (u->entity != CN_ENTITY_CELL)
        return fail(CN_ERR_UNSUPPORTED, "finite-difference stencils need cell-centred grids");
    if (comp < 0 || comp + ncin > u->ncomp)
        return fail(CN_ERR_INVALID_ARGUMENT, "input component out of range");
    cn_status s;
    if (o1 && (s = check_out(u, o1, c1, 1)) != CN_OK) return s;
    if (o2 && (s = check_out(u, o2, c2, 3)) != CN_OK) return s;
    cudaStream_t st = as_stream(stream);
    if (u->dtype == CN_FLOAT64) return launch_fd<double, OP>(u, comp, o1, c1, o2, c2, st);
    if (u->dtype == CN_FLOAT32) return launch_fd<float, OP>(u, comp, o1, c1, o2, c2, st);
    return fail(CN_ERR_UNSUPPORTED, "finite-difference stencils need FLOAT32 or FLOAT64 grids");
}

// ---------------------------------------------------------------- ddx ABI
// One thread per (x, y) column of 32 x 8 tiles, looping over z: no index
// divisions, coalesced rows along x.
template <typename T>
__global__ void __launch_bounds__(256)
    ddx_kernel(int nx, int ny, int nz, const T *__restrict__ src, int xps, int xyps,
               T *__restrict__ dst, int xpd, int xypd, T fac)
{
    using A = Arith<T>;
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    if (x >= nx) return;
    for (int y = blockIdx.y * 8 + (threadIdx.x >> 5); y < ny; y += gridDim.y * 8) {
        for (int z = blockIdx.z; z < nz; z += gridDim.z) {
            const T *s = src + x + (int64_t)xps * y + (int64_t)xyps * z;
            T acc = A::add(s[-1], s[1]);
            acc = A::add(acc, s[-xps]);
            acc = A::add(acc, s[xps]);
            acc = A::add(acc, s[-xyps]);
            acc = A::add(acc, s[xyps]);
            acc = A::sub(acc, A::mul(T(6), s[0]));
            dst[x + (int64_t)xpd * y + (int64_t)xypd * z] = A::mul(fac, acc);
        }
    }
}

template <typename T>
static cn_status launch_ddx(int nx, int ny, int nz, const T *src, int xps, int xyps, T *dst,
                            int xpd, int xypd, T fac, cudaStream_t st)
{
    if (nx < 1 || ny < 1 || nz < 1 || !src || !dst)
        return fail(CN_ERR_INVALID_ARGUMENT, "ddx: bad extent or pointer");
    const int gx = (nx + 31) / 32;
    const dim3 grid((unsigned)gx, (unsigned)std::min((ny + 7) / 8, 65535), (unsigned)std::min(nz, 65535));
    ddx_kernel<T><<<grid, 256, 0, st>>>(nx, ny, nz, src, xps, xyps, dst, xpd, xypd, fac);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

} // namespace cn

using namespace cn;

extern "C" {

cn_status cn_laplacian(cn_grid *u, int comp, cn_grid *out, int out_comp, void *stream)
{
    if (!out) return fail(CN_ERR_INVALID_ARGUMENT, "output grid is NULL");
    return dispatch_fd<kLap>(u, comp, 1, out, out_comp, nullptr, 0, stream);
}

cn_status cn_gradient(cn_grid *u, int comp, cn_grid *out, int out_comp, void *stream)
{
    if (!out) return fail(CN_ERR_INVALID_ARGUMENT, "output grid is NULL");
    return dispatch_fd<kGrad>(u, comp, 1, nullptr, 0, out, out_comp, stream);
}

cn_status cn_lap_grad(cn_grid *u, int comp, cn_grid *lap, int lap_comp, cn_grid *grad,
                      int grad_comp, void *stream)
{
    if (!lap || !grad) return fail(CN_ERR_INVALID_ARGUMENT, "output grid is NULL");
    return dispatch_fd<kLapGrad>(u, comp, 1, lap, lap_comp, grad, grad_comp, stream);
}

cn_status cn_divergence(cn_grid *v, int comp, cn_grid *out, int out_comp, void *stream)
{
    if (!out) return fail(CN_ERR_INVALID_ARGUMENT, "output grid is NULL");
    return dispatch_fd<kDiv>(v, comp, 3, out, out_comp, nullptr, 0, stream);
}

void cn_ddx_f64(int Nx, int Ny, int Nz, const double *src, int xps, int xyps, double *dst,
                int xpd, int xypd, double factor)
{
    // ddxGold.cpp:49: fac = 1.0 / (factor * factor)
    (void)launch_ddx<double>(Nx, Ny, Nz, src, xps, xyps, dst, xpd, xypd,
                             1.0 / (factor * factor), nullptr);
}

void cn_ddx_f32(int Nx, int Ny, int Nz, const float *src, int xps, int xyps, float *dst,
                int xpd, int xypd, float factor)
{
    // computed in double, stored as float, as `const Real fac = 1.0 / (f*f)`
    const float fac = (float)(1.0 / (double)(factor * factor));
    (void)launch_ddx<float>(Nx, Ny, Nz, src, xps, xyps, dst, xpd, xypd, fac, nullptr);
}

cn_status cn_ddx_async(cn_dtype dtype, int Nx, int Ny, int Nz, const void *src, int xps,
                       int xyps, void *dst, int xpd, int xypd, double factor, void *stream)
{
    cudaStream_t st = as_stream(stream);
    if (dtype == CN_FLOAT64)
        return launch_ddx<double>(Nx, Ny, Nz, (const double *)src, xps, xyps, (double *)dst, xpd,
                                  xypd, 1.0 / (factor * factor), st);
    if (dtype == CN_FLOAT32) {
        const float f = (float)factor;
        return launch_ddx<float>(Nx, Ny, Nz, (const float *)src, xps, xyps, (float *)dst, xpd,
                                 xypd, (float)(1.0 / (double)(f * f)), st);
    }
    return fail(CN_ERR_UNSUPPORTED, "ddx: dtype must be FLOAT32 or FLOAT64");
}

} // extern "C"
