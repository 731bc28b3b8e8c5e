// euler.cu -- K2: lab fill fused with WENO5-JS + Rusanov + flux divergence for
// the 3-D compressible Euler equations, and the fused SSP-RK3 stage update.
//
// One CTA owns an 8x8x8 tile of one block.  It stages the tile's cells of all
// five conserved variables into shared memory as primitives (rho, u, v, w, p)
// and, before the sweep of each direction, that direction's two 3-cell halo
// slabs (together the lab of a stencil (-3,4) non-tensorial,
// Block/FieldLab.h:180-224): halo cells inside the block are plain loads,
// cells outside are resolved by cn::lab_value (periodic neighbour, skip rule
// and BC chain of each component's BC vector).  Per direction every face flux
// of the tile is computed exactly once (runs of three faces per thread, each
// cell's WENO5 smoothness indicators shared by its two faces, Rusanov) and
// differenced into per-cell accumulators in shared memory.  The epilogue
// applies the SSP-RK3 (Shu & Osher 1988) convex combination and optionally
// accumulates FP64 conservation sums per CTA (reduced in a fixed order by a
// second kernel, so the sums are deterministic).
//
// The tile's cells of all five components arrive in shared memory by one TMA
// copy (a 5-D tensor map over the state, cuTensorMapEncodeTiled) while the
// threads stage the halo slabs; they are then converted to primitives.
//
// Shared memory per CTA: 5 x 1024 primitives (the tile plus one direction's
// halo slabs, restaged before each sweep; FP32 keeps all three directions'
// slabs) + 5 x 704 accumulators and exchanged face fluxes (the TMA landing
// area of the tile's conservative cells before the sweeps).
#include "cn_internal.h"
#include "cn_tma.cuh"
#include "euler_math.cuh"
#include "euler_stage.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cstring>
#include <mutex>

namespace cn {
namespace euler {

// Dynamic shared memory, from its first 128-byte aligned address: W
// [5][Stg<T>::SV], then A [5][NACC] from a 128-byte aligned offset (the TMA
// destination of the tile's cells); 128 bytes of slack for the alignment.
template <typename T> constexpr size_t acc_offset()
{
    return (5 * Stg<T>::SV * sizeof(T) + 127) / 128 * 128;
}
template <typename T> constexpr size_t stage_smem()
{
    return 128 + acc_offset<T>() + 5 * NACC * sizeof(T);
}

template <typename T>
__global__ void __launch_bounds__(NT, sizeof(T) == 4 ? 4 : 3)
    stage_kernel(StageParams<T> p, CartSrc src, const __grid_constant__ CUtensorMap core)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *base = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
    T *W = reinterpret_cast<T *>(base);                    // [5][Stg<T>::SV]
    T *A = reinterpret_cast<T *>(base + acc_offset<T>()); // [5][NACC]
    __shared__ double red[NT / 32][5];
    __shared__ int snb[29];
    __shared__ TileInfo<T> ts;
    __shared__ __align__(8) uint64_t core_bar;
    if (threadIdx.x == 0) {
        mbar_init(&core_bar, 1);
        fence_mbar_init();
    }
    stage_tile<T, CartSrc, true>(p, src, blockIdx.x, blockIdx.x, W, A, red, snb, &ts, &core, &core_bar);
}

// Fixed-order reduction of per-CTA partials: out[c] = sum_i partials[i][c].
__global__ void __launch_bounds__(256) reduce_partials(const double *partials, int n, double *out)
{
    __shared__ double sh[256];
    for (int c = 0; c < 5; ++c) {
        double s = 0;
        for (int i = threadIdx.x; i < n; i += 256)
            s += partials[(int64_t)i * 5 + c];
        sh[threadIdx.x] = s;
        __syncthreads();
        for (int w = 128; w > 0; w >>= 1) {
            if (threadIdx.x < w)
                sh[threadIdx.x] += sh[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0)
            out[c] = sh[0];
        __syncthreads();
    }
}

// Max over cells of |u_d| + c for each direction (for the CFL time step).
template <typename T>
__global__ void __launch_bounds__(256)
    max_speed_kernel(const T *r, const T *m0, const T *m1, const T *m2, const T *E, int64_t nb,
                     int64_t cells, int64_t bstride, T gamma, T gm1, unsigned long long *out)
{
    double mx[3] = {0, 0, 0};
    const int64_t total = nb * cells;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = i / cells, c = i - b * cells;
        const int64_t o = b * bstride + c;
        T w[5];
        to_primitive<T>(r[o], m0[o], m1[o], m2[o], E[o], gm1, w);
        const double cs = sqrt((double)gamma * (double)w[4] / (double)w[0]);
        for (int d = 0; d < 3; ++d)
            mx[d] = fmax(mx[d], fabs((double)w[1 + d]) + cs);
    }
    for (int d = 0; d < 3; ++d) {
        double v = mx[d];
        for (int off = 16; off > 0; off >>= 1)
            v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
        if ((threadIdx.x & 31) == 0)
            atomicMax(out + d, (unsigned long long)__double_as_longlong(v)); // v >= 0: order-preserving
    }
}

} // namespace euler

using namespace euler;

static cn_status check_euler(const cn_grid *g, int comp0)
{
    if (!g) return fail(CN_ERR_INVALID_ARGUMENT, "grid is NULL");
    if (comp0 < 0 || comp0 + 5 > g->ncomp)
        return fail(CN_ERR_INVALID_ARGUMENT, "Euler state needs 5 components");
    if (g->dtype != CN_FLOAT64 && g->dtype != CN_FLOAT32)
        return fail(CN_ERR_UNSUPPORTED, "Euler kernels need FLOAT32 or FLOAT64 grids");
    if (g->entity != CN_ENTITY_CELL)
        return fail(CN_ERR_UNSUPPORTED, "Euler kernels need cell-centred grids");
    for (int d = 0; d < 3; ++d)
        if (g->n[d] % TB != 0 || g->n[d] < G)
            return fail(CN_ERR_UNSUPPORTED, "Euler kernels need block cells divisible by 8");
    return CN_OK;
}

static bool same_shape(const cn_grid *a, const cn_grid *b)
{
    return a->nblocks == b->nblocks && a->n[0] == b->n[0] && a->n[1] == b->n[1] &&
           a->n[2] == b->n[2] && a->dtype == b->dtype && a->block_stride == b->block_stride;
}

// Tensor map of the five components cs..cs+4 of grid g as the 5-D array
// [comp][block][z][y][x] (innermost first: x, y, z, block, comp), box
// 8 x 8 x 8 x 1 x 5: one TMA copy brings a tile's cells of all components.
// Strides are byte multiples of 16 (block storage is padded to 32 bytes).
static cn_status core_map(const cn_grid *g, int cs, size_t es, CUtensorMap *m)
{
    void *base = static_cast<char *>(g->d_data) + (size_t)cs * g->comp_stride * es;
    const cuuint64_t dims[5] = {(cuuint64_t)g->n[0], (cuuint64_t)g->n[1], (cuuint64_t)g->n[2],
                                (cuuint64_t)g->nblocks, 5};
    const cuuint64_t strides[4] = {(cuuint64_t)g->n[0] * es, (cuuint64_t)g->n[0] * g->n[1] * es,
                                   (cuuint64_t)g->block_stride * es, (cuuint64_t)g->comp_stride * es};
    const cuuint32_t box[5] = {TB, TB, TB, 1, 5};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    for (int i = 0; i < 4; ++i)
        if (strides[i] % 16) return fail(CN_ERR_UNSUPPORTED, "Euler stage: grid strides are not 16-byte multiples");
    // the driver's encoder through the runtime's entry-point query (the
    // library does not link the driver library itself)
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!encode) return fail(CN_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const CUresult r = encode(
        m, es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, base, dims, strides, box,
        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(CN_ERR_CUDA, "cuTensorMapEncodeTiled failed for the Euler tile map");
    return CN_OK;
}

template <typename T>
static cn_status launch_stage(cn_grid *bcsrc, cn_grid *Us, int cs, cn_grid *Un, int cn_,
                              cn_grid *out, int co, int stage, double dt, double gamma,
                              double *partials, cudaStream_t st)
{
    cn_stencil s = {{-G, -G, -G}, {G + 1, G + 1, G + 1}, 0};
    cn_status r = check_lab(Us, &s);
    if (r != CN_OK) return r;
    r = sync_bc(bcsrc, st);
    if (r != CN_OK) return r;
    StageParams<T> p = {};
    CartSrc src;
    src.L = make_geom(Us, &s);
    for (int c = 0; c < 5; ++c) {
        p.U[c] = reinterpret_cast<const T *>(Us->d_data) + (size_t)(cs + c) * Us->comp_stride;
        p.Un[c] = Un ? reinterpret_cast<const T *>(Un->d_data) + (size_t)(cn_ + c) * Un->comp_stride
                     : nullptr;
        p.out[c] = reinterpret_cast<T *>(out->d_data) + (size_t)(co + c) * out->comp_stride;
        src.bc[c] = bc_view(bcsrc, cs + c);
    }
    for (int d = 0; d < 3; ++d) src.ih[d] = 1.0 / Us->h[d];
    p.dt = (T)dt;
    p.gamma = (T)gamma;
    p.gm1 = (T)(gamma - 1.0);
    p.igm1 = (T)(1.0 / (gamma - 1.0));
    p.stage = stage;
    p.partials = partials;
    p.err = Us->d_err;
    CUtensorMap core;
    r = core_map(Us, cs, sizeof(T), &core);
    if (r != CN_OK) return r;
    const size_t smem = stage_smem<T>();
    static DeviceOnce attr_once; // per device (the first call on a device is an eager one)
    r = smem_opt_in(attr_once, stage_kernel<T>, smem);
    if (r != CN_OK) return r;
    const int64_t ctas = (int64_t)Us->nblocks * (Us->n[0] / TB) * (Us->n[1] / TB) * (Us->n[2] / TB);
    stage_kernel<T><<<(unsigned)ctas, NT, smem, st>>>(p, src, core);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

static int64_t stage_ctas(const cn_grid *g)
{
    return (int64_t)g->nblocks * (g->n[0] / TB) * (g->n[1] / TB) * (g->n[2] / TB);
}

static cn_status run_stage(cn_grid *bcsrc, cn_grid *Us, int cs, cn_grid *Un, int cn_, cn_grid *out,
                           int co, int stage, double dt, double gamma, double *partials,
                           cudaStream_t st)
{
    if (Us->dtype == CN_FLOAT64)
        return launch_stage<double>(bcsrc, Us, cs, Un, cn_, out, co, stage, dt, gamma, partials, st);
    return launch_stage<float>(bcsrc, Us, cs, Un, cn_, out, co, stage, dt, gamma, partials, st);
}

} // namespace cn

using namespace cn;

// Scratch of the conservation sums and the wave-speed maximum: per-CTA
// partials and the 5 totals, one set per device, grown on demand.
struct SumScratch {
    double *partials = nullptr;
    double *totals = nullptr;
    int64_t cap = 0;
};
static SumScratch g_sum[64];
static std::mutex g_sum_mu;

static cn_status ensure_sum_scratch(int64_t nctas, SumScratch **out)
{
    int dev = 0;
    CN_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(CN_ERR_UNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lk(g_sum_mu);
    SumScratch &sc = g_sum[dev];
    if (!sc.totals) CN_CUDA_TRY(cudaMalloc(&sc.totals, 5 * sizeof(double)));
    if (nctas > sc.cap) {
        if (sc.partials) cudaFree(sc.partials);
        sc.partials = nullptr;
        sc.cap = 0;
        CN_CUDA_TRY(cudaMalloc(&sc.partials, (size_t)nctas * 5 * sizeof(double)));
        sc.cap = nctas;
    }
    *out = &sc;
    return CN_OK;
}

extern "C" {

cn_status cn_euler_rhs(cn_grid *U, int comp0, double gamma, cn_grid *rhs, int rhs_comp0, void *stream)
{
    cn_status s = check_euler(U, comp0);
    if (s != CN_OK) return s;
    if (!rhs || !same_shape(U, rhs) || rhs_comp0 < 0 || rhs_comp0 + 5 > rhs->ncomp)
        return fail(CN_ERR_SIZE_MISMATCH, "Cartesian: Can not assign two grids of unequal size.");
    return run_stage(U, U, comp0, nullptr, 0, rhs, rhs_comp0, 0, 0.0, gamma, nullptr, as_stream(stream));
}

cn_status cn_euler_rk3_stage(cn_grid *bcsrc, cn_grid *Us, cn_grid *Un, cn_grid *out, int stage,
                             double dt, double gamma, double *sums_out, void *stream)
{
    if (stage < 1 || stage > 3) return fail(CN_ERR_INVALID_ARGUMENT, "stage must be 1, 2 or 3");
    cn_status s = check_euler(Us, 0);
    if (s != CN_OK) return s;
    if (!bcsrc || !out || !same_shape(Us, out) || !same_shape(Us, bcsrc) || bcsrc->ncomp < 5 ||
        out->ncomp < 5 || (stage > 1 && (!Un || !same_shape(Us, Un) || Un->ncomp < 5)))
        return fail(CN_ERR_SIZE_MISMATCH, "Cartesian: Can not assign two grids of unequal size.");
    cudaStream_t st = as_stream(stream);
    double *partials = nullptr;
    SumScratch *sc = nullptr;
    if (sums_out) {
        s = ensure_sum_scratch(stage_ctas(Us), &sc);
        if (s != CN_OK) return s;
        partials = sc->partials;
    }
    s = run_stage(bcsrc, Us, 0, stage > 1 ? Un : nullptr, 0, out, 0, stage, dt, gamma, partials, st);
    if (s != CN_OK) return s;
    if (sums_out) {
        const double vol = Us->h[0] * Us->h[1] * Us->h[2];
        reduce_partials<<<1, 256, 0, st>>>(sc->partials, (int)stage_ctas(Us), sc->totals);
        CN_CUDA_TRY(cudaGetLastError());
        double t[5];
        CN_CUDA_TRY(cudaMemcpyAsync(t, sc->totals, sizeof(t), cudaMemcpyDeviceToHost, st));
        CN_CUDA_TRY(cudaStreamSynchronize(st));
        if ((s = grid_check_error(const_cast<cn_grid *>(Us))) != CN_OK) return s;
        for (int c = 0; c < 5; ++c) sums_out[c] = t[c] * vol;
    }
    return CN_OK;
}

cn_status cn_euler_rk3_step(cn_grid *U, cn_grid *work1, cn_grid *work2, double dt, double gamma,
                            double *sums_out, void *stream)
{
    cn_status s;
    if ((s = cn_euler_rk3_stage(U, U, nullptr, work1, 1, dt, gamma, nullptr, stream)) != CN_OK) return s;
    if ((s = cn_euler_rk3_stage(U, work1, U, work2, 2, dt, gamma, nullptr, stream)) != CN_OK) return s;
    // stage 3 writes U^{n+1} over U^n: each cell reads its own U^n before writing
    return cn_euler_rk3_stage(U, work2, U, U, 3, dt, gamma, sums_out, stream);
}

cn_status cn_euler_max_speed(cn_grid *U, double gamma, double out[3], void *stream)
{
    cn_status s = check_euler(U, 0);
    if (s != CN_OK) return s;
    if (!out) return fail(CN_ERR_INVALID_ARGUMENT, "out is NULL");
    cudaStream_t st = as_stream(stream);
    SumScratch *sc = nullptr;
    s = ensure_sum_scratch(1, &sc);
    if (s != CN_OK) return s;
    unsigned long long *d = reinterpret_cast<unsigned long long *>(sc->totals);
    CN_CUDA_TRY(cudaMemsetAsync(d, 0, 3 * sizeof(unsigned long long), st));
    const int64_t cells = (int64_t)U->n[0] * U->n[1] * U->n[2];
    if (U->dtype == CN_FLOAT64) {
        const double *b = reinterpret_cast<const double *>(U->d_data);
        max_speed_kernel<double><<<148 * 8, 256, 0, st>>>(b, b + U->comp_stride, b + 2 * U->comp_stride,
                                                          b + 3 * U->comp_stride, b + 4 * U->comp_stride,
                                                          U->nblocks, cells, U->block_stride, gamma,
                                                          gamma - 1.0, d);
    } else {
        const float *b = reinterpret_cast<const float *>(U->d_data);
        max_speed_kernel<float><<<148 * 8, 256, 0, st>>>(b, b + U->comp_stride, b + 2 * U->comp_stride,
                                                         b + 3 * U->comp_stride, b + 4 * U->comp_stride,
                                                         U->nblocks, cells, U->block_stride, (float)gamma,
                                                         (float)(gamma - 1.0), d);
    }
    CN_CUDA_TRY(cudaGetLastError());
    unsigned long long h[3];
    CN_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, st));
    CN_CUDA_TRY(cudaStreamSynchronize(st));
    for (int k = 0; k < 3; ++k) {
        double v;
        memcpy(&v, &h[k], sizeof(v));
        out[k] = v;
    }
    return CN_OK;
}

} // extern "C"

// --------------------------------------------------------------------------
// SSP-RK3 stage with conservation sums and no device allocation.
//
// cn_euler_rk3_stage grows its per-CTA partials with cudaMalloc on first use
// and whenever a larger grid arrives.  Some callers cannot allow that: a host
// that runs with a fixed device-memory budget reserved up front (a solver
// sharing the GPU with a pool allocator that owns the rest of the memory), or
// one that must not let a first-time cudaMalloc/cudaFree synchronise the
// device mid-run.  This variant takes its scratch from a fixed file-scope
// device array instead, so a call never allocates; the price is a hard limit
// on the grid size.  Like cn_euler_rk3_stage it copies the sums to the host
// and waits for the stream before it returns.
//
// Size: one 5-double partial per 8^3 tile plus the 5 totals, for at most
// kStaticSumTiles tiles (16.8M cells, e.g. 256^3), 1.25 MiB per device.
// Nothing in the array needs to start at zero: every call writes each
// partial it later reads (one per tile of the grid) and then the totals.
// The array is one per device and the calls share it, so two calls that
// overlap on the same device (two streams, or two host threads) race on it
// and may return each other's sums; callers serialise them.
// Set-up: the first call on a device, with that device current, looks up the
// array's device address with cudaGetSymbolAddress and keeps it.
// BC tables: the stage uploads changed BC vectors of `bcsrc` before its
// launch; if they grew beyond the device table's capacity that upload would
// allocate, so the call is refused (CN_ERR_INVALID_ARGUMENT) and the caller
// runs cn_bc_sync once after changing the BCs, before the no-allocation calls.
// --------------------------------------------------------------------------
static constexpr int64_t kStaticSumTiles = 32768;
static __device__ __align__(256) double g_static_sums[kStaticSumTiles * 5 + 5];
static double *g_static_sums_ptr[64];
static std::mutex g_static_sums_mu;

static cn_status static_sum_scratch(double **out)
{
    int dev = 0;
    CN_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(CN_ERR_UNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lk(g_static_sums_mu);
    if (!g_static_sums_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_sums);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_static_sums)");
        if (!p) return fail(CN_ERR_CUDA, "cudaGetSymbolAddress returned a null address");
        g_static_sums_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_static_sums_ptr[dev];
    return CN_OK;
}

extern "C" cn_status cn_euler_rk3_stage_noalloc(cn_grid *bcsrc, cn_grid *Us, cn_grid *Un, cn_grid *out,
                                                int stage, double dt, double gamma, double *sums_out,
                                                void *stream)
{
    if (stage < 1 || stage > 3) return fail(CN_ERR_INVALID_ARGUMENT, "stage must be 1, 2 or 3");
    if (!sums_out) return fail(CN_ERR_INVALID_ARGUMENT, "sums_out is NULL");
    cn_status s = check_euler(Us, 0);
    if (s != CN_OK) return s;
    if (!bcsrc || !out || !same_shape(Us, out) || !same_shape(Us, bcsrc) || bcsrc->ncomp < 5 ||
        out->ncomp < 5 || (stage > 1 && (!Un || !same_shape(Us, Un) || Un->ncomp < 5)))
        return fail(CN_ERR_SIZE_MISMATCH, "Cartesian: Can not assign two grids of unequal size.");
    const int64_t tiles = stage_ctas(Us);
    if (tiles > kStaticSumTiles)
        return fail(CN_ERR_UNSUPPORTED,
                    "cn_euler_rk3_stage_noalloc: grid has more than 32768 8^3 tiles (16.8M cells), "
                    "the size of its fixed scratch");
    if (sync_bc_would_allocate(bcsrc))
        return fail(CN_ERR_INVALID_ARGUMENT,
                    "cn_euler_rk3_stage_noalloc: the BC vectors grew since the last upload; call cn_bc_sync "
                    "before the no-allocation stage");
    double *scratch = nullptr;
    s = static_sum_scratch(&scratch);
    if (s != CN_OK) return s;
    double *partials = scratch, *totals = scratch + kStaticSumTiles * 5;
    cudaStream_t st = as_stream(stream);
    s = run_stage(bcsrc, Us, 0, stage > 1 ? Un : nullptr, 0, out, 0, stage, dt, gamma, partials, st);
    if (s != CN_OK) return s;
    reduce_partials<<<1, 256, 0, st>>>(partials, (int)tiles, totals);
    CN_CUDA_TRY(cudaGetLastError());
    double t[5];
    CN_CUDA_TRY(cudaMemcpyAsync(t, totals, sizeof(t), cudaMemcpyDeviceToHost, st));
    CN_CUDA_TRY(cudaStreamSynchronize(st));
    if ((s = grid_check_error(const_cast<cn_grid *>(Us))) != CN_OK) return s;
    const double vol = Us->h[0] * Us->h[1] * Us->h[2];
    for (int c = 0; c < 5; ++c) sums_out[c] = t[c] * vol;
    return CN_OK;
}
