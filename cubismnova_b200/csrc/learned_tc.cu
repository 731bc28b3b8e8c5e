// learned_tc.cu -- the learned smoother's 3x3x3 convolutions on the tensor
// cores (tcgen05, sm_100a): BF16 activations and weights, FP32 accumulation
// in tensor memory.
//
// Implicit GEMM without an im2col buffer.  A CTA owns a brick of 16x16x4
// output cells of one block and stages the 18x18x6 input region (brick plus
// a one-cell halo) in shared memory, one row of 16 BF16 channels per region
// cell, rows in region order r = i + 18 (j + 18 k).  An output cell sits at
// row R0 + m with m = x + 18 y + 324 z, and its input at tap (dx, dy, dz) at
// row R0 + m + dx + 18 dy + 324 dz: for every tap the A operand of an
// M = 128 tile is the same run of 128 rows, shifted.  So one M-tile is 27
// MMAs (M = 128, N = 16, K = 16 channels, one per tap) accumulating into the
// same TMEM columns; the A descriptor's start address moves by the tap's row
// offset.  Rows m whose (x, y) fall outside the brick (x or y in 16..17) are
// computed and dropped.  The brick spans m in [0, 1258): 10 M-tiles.
//
// Shared-memory operand layout (unswizzled, K-major): A is two planes (K
// chunks of channels 0-7 and 8-15) of SROWS rows x 16 bytes; core matrices
// are 8 consecutive rows of one plane (SBO = 128 B between 8-row groups,
// LBO = one plane between the two K chunks), so a shift by any number of
// rows is again a valid operand.  B (weights of one tap, N = 16 output
// channels x K = 16 input channels) uses the same form: planes of 16 rows.
//
// Layers: 2 -> 16 (input channels padded with zeros to 16), 16 -> 16, and
// 16 -> 1 (output channels padded to N = 16); ReLU after the first two.  All
// inputs are channels-last BF16, 32 bytes per cell (the features kernel
// writes (x0, x1, 0, ..., 0)), staged with asynchronous 16-byte copies; the
// last layer applies the smoothing update p += omega x0 + y in its epilogue.
// Neighbour cells outside the block are the periodic neighbours of the block
// grid (the activation grids carry no BCs), corners and edges included.
//
// One thread issues the MMAs, commits them to an mbarrier and polls it
// (bounded; on timeout the CTA records an error word, skips its epilogue,
// frees its TMEM and exits) while the other threads wait at the CTA barrier.
#include "cn_internal.h"
#include "cn_tc.cuh"
#include "cn_tma.cuh"
#include "learned_tc.h"
#include "mg_tile.cuh"

#include <cuda_bf16.h>

namespace cn {
namespace nntc {

constexpr int BX = 16, BY = 16, BZ = 4;              // brick of output cells
constexpr int RX = BX + 2, RY = BY + 2, RZ = BZ + 2; // input region 18 x 18 x 6
constexpr int RCELLS = RX * RY * RZ;                 // 1944
constexpr int R0 = 1 + RX + RX * RY;                 // row of output cell (0,0,0): 343
constexpr int MSPAN = (BX - 1) + RX * (BY - 1) + RX * RY * (BZ - 1) + 1; // 1258
constexpr int MT = (MSPAN + 127) / 128;              // 10 M-tiles
// highest row read: R0 + 128 MT - 1 + R0 (tap offsets lie in [-R0, R0])
constexpr int SROWS = ((2 * R0 + 128 * MT + 7) / 8) * 8; // 1968
constexpr int NTHREADS = 256;
constexpr int TMEM_COLS = 256;                       // >= 16 * MT
constexpr uint32_t PLANE = SROWS * 16;               // bytes of one K plane of A
constexpr uint32_t WTAP = 512;                       // bytes of one tap's B (2 planes x 16 rows x 16 B)
constexpr size_t SMEM = 2 * (size_t)PLANE + 27 * WTAP + 16 + 28 * 4;
constexpr uint32_t IDESC = tc::idesc_bf16_f32(128, 16);
static_assert(RCELLS <= SROWS, "region must fit the A rows");
static_assert(16 * MT <= TMEM_COLS, "accumulators must fit the TMEM allocation");

struct Params {
    const uint16_t *act;   // input activations [nblocks][cells][16] BF16
    const float *x;        // mode 2: x0 of the features grid (block stride xbs)
    int64_t xbs;
    const uint16_t *w;     // [27][2][16][8] BF16 B tiles of this layer
    // output: mode 1 writes BF16 activations (optional ReLU); mode 2 updates p
    uint16_t *out;
    float *p;              // mode 2: p (FP32 grid, block stride pbs)
    int64_t pbs;
    float omega;
    int zero_guess;        // mode 2: p starts from zero
    int relu;
    int nb[3], n[3];
    int bricks[3];         // bricks per block along x, y, z
    int *err;
};

__device__ __forceinline__ uint16_t bf16_bits(float v)
{
    return __bfloat16_as_ushort(__float2bfloat16_rn(v));
}

template <int MODE>
__global__ void __launch_bounds__(NTHREADS) conv3_tc_kernel(const __grid_constant__ Params P)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *A = smem;                       // [2][SROWS][16 B]
    unsigned char *Bw = smem + 2 * PLANE;          // [27][2][16][16 B]
    uint64_t *bar = reinterpret_cast<uint64_t *>(Bw + 27 * WTAP);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 1);
    int *snb = reinterpret_cast<int *>(slot + 1);   // 27 periodic neighbour blocks
    int *okf = snb + 27;                            // MMA completion flag

    const int bricks = P.bricks[0] * P.bricks[1] * P.bricks[2];
    const int block = blockIdx.x / bricks;
    int br = blockIdx.x - block * bricks;
    const int ox = (br % P.bricks[0]) * BX;
    br /= P.bricks[0];
    const int oy = (br % P.bricks[1]) * BY;
    const int oz = (br / P.bricks[1]) * BZ;
    const int cells = P.n[0] * P.n[1] * P.n[2];

    // ---- TMEM and barrier set-up (warp 0 allocates)
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    if (threadIdx.x < 32) {
        tc::tmem_alloc(slot, TMEM_COLS);
        tc::tmem_relinquish();
    }
    mg::neighbour_blocks(P.nb, block, snb);
    __syncthreads();

    // ---- weights: 27 taps x 512 B as 16-byte chunks
    for (int i = threadIdx.x; i < 27 * 32; i += NTHREADS)
        reinterpret_cast<uint4 *>(Bw)[i] = __ldg(reinterpret_cast<const uint4 *>(P.w) + i);

    // ---- input region: row u = region cell, two 16-byte chunks (K planes),
    // asynchronous 16-byte copies (many in flight per thread); rows past the
    // region are zero
    for (int t = threadIdx.x; t < 2 * SROWS; t += NTHREADS) {
        const int u = t >> 1, kc = t & 1;
        unsigned char *dst = A + kc * PLANE + u * 16;
        if (u < RCELLS) {
            const int i = u % RX, j = (u / RX) % RY, k = u / (RX * RY);
            const int x = ox + i - 1, y = oy + j - 1, z = oz + k - 1;
            const int r0 = x < 0 ? -1 : (x >= P.n[0] ? 1 : 0), r1 = y < 0 ? -1 : (y >= P.n[1] ? 1 : 0),
                      r2 = z < 0 ? -1 : (z >= P.n[2] ? 1 : 0);
            const int sb = snb[(r0 + 1) + 3 * (r1 + 1) + 9 * (r2 + 1)];
            const int sc = (x - r0 * P.n[0]) + P.n[0] * ((y - r1 * P.n[1]) + P.n[1] * (z - r2 * P.n[2]));
            const uint16_t *src = P.act + ((int64_t)sb * cells + sc) * 16 + kc * 8;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
        } else {
            *reinterpret_cast<uint4 *>(dst) = make_uint4(0u, 0u, 0u, 0u);
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    fence_proxy_async_smem(); // generic-proxy smem writes -> visible to the tensor cores
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = *slot;

    // ---- MMAs: 10 M-tiles x 27 taps, issued by one thread, which then
    // polls the completion barrier (bounded) while the others wait at the
    // CTA barrier.  Descriptor start addresses advance in 16-byte units.
    if (threadIdx.x == 0) {
        const uint64_t da = tc::smem_desc(smem_u32(A), PLANE, 128u);
        const uint64_t db = tc::smem_desc(smem_u32(Bw), 256u, 128u);
#pragma unroll 1
        for (int t = 0; t < MT; ++t) {
#pragma unroll
            for (int q = 0; q < 27; ++q) {
                const int off = (q % 3 - 1) + RX * ((q / 3) % 3 - 1) + RX * RY * (q / 9 - 1);
                tc::mma_bf16(tbase + 16u * t, da + (uint64_t)(R0 + 128 * t + off), db + (uint64_t)(q * (WTAP / 16)),
                             IDESC, q > 0 ? 1u : 0u);
            }
        }
        tc::mma_commit(bar);
        *okf = mbar_wait_bounded(bar, 0) ? 1 : 0;
    }
    __syncthreads();
    const int ok = *okf;
    tc::fence_after_sync();

    // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 of the tiles t = w / 4, w / 4 + 2, ...
    if (ok) {
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const uint32_t lane_base = (uint32_t)(32 * (w & 3)) << 16;
#pragma unroll 1
        for (int t = w >> 2; t < MT; t += 2) {
            float v[16];
            tc::tmem_ld16(tbase + lane_base + 16u * t, v);
            const int m = 128 * t + 32 * (w & 3) + lane;
            const int z = m / (RX * RY), rem = m - z * (RX * RY);
            const int y = rem / RX, x = rem - y * RX;
            if (x >= BX || y >= BY || z >= BZ)
                continue;
            const int c = (ox + x) + P.n[0] * ((oy + y) + P.n[1] * (oz + z));
            if (MODE == 2) {
                const int64_t o = (int64_t)block * P.pbs + c;
                const float x0 = __ldg(P.x + (int64_t)block * P.xbs + c);
                const float pv = P.zero_guess ? 0.f : P.p[o];
                P.p[o] = pv + (P.omega * x0 + v[0]);
            } else {
                uint32_t h[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    float a = v[2 * j], b = v[2 * j + 1];
                    if (P.relu) {
                        a = fmaxf(a, 0.f);
                        b = fmaxf(b, 0.f);
                    }
                    h[j] = (uint32_t)bf16_bits(a) | ((uint32_t)bf16_bits(b) << 16);
                }
                uint4 *dst = reinterpret_cast<uint4 *>(P.out + ((int64_t)block * cells + c) * 16);
                dst[0] = make_uint4(h[0], h[1], h[2], h[3]);
                dst[1] = make_uint4(h[4], h[5], h[6], h[7]);
            }
        }
    } else if (threadIdx.x == 0 && P.err) {
        atomicExch(P.err, kDevErrTimeout);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32)
        tc::tmem_dealloc(tbase, TMEM_COLS);
}

// --------------------------------------------------------------------------
// Persistent, warp-specialised form: one CTA per SM walks the bricks with a
// stride of gridDim.x.  Warps 0-1 (producers) stage brick i into one of two
// A buffers with asynchronous 16-byte copies whose completion arrives on
// full[b]; warp 2 (one thread) waits for full[b], issues the brick's 270 MMAs
// into one of two TMEM accumulators (columns 0 / 256) and commits them to
// empty[b] (A buffer free) and tfull[a] (accumulator ready); warps 4-7
// (epilogue, one TMEM lane quadrant each) drain accumulator a and arrive on
// tempty[a].  So staging of brick i+1 and the epilogue of brick i-1 overlap
// the MMAs of brick i.  Every wait is bounded; a role that gives up records
// an error word and stops, and the others then give up too.
constexpr int PIPE_THREADS = 256;
constexpr int PRODUCERS = 64;                         // warps 0-1
constexpr int MMA_WARP = 2;
constexpr int EPI_WARP0 = 4;                          // warps 4-7
constexpr uint32_t PIPE_TMEM_COLS = 512;              // 2 accumulators x 256 columns
constexpr size_t PIPE_BAR_OFF = 4 * (size_t)PLANE + 27 * WTAP;
constexpr size_t PIPE_SMEM = PIPE_BAR_OFF + 9 * 8 + 8 + 2 * 28 * 4;

__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t *bar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void named_sync(int id, int count)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

struct BrickPos {
    int block, ox, oy, oz;
};
__device__ __forceinline__ BrickPos brick_pos(const Params &P, int i)
{
    const int per = P.bricks[0] * P.bricks[1] * P.bricks[2];
    BrickPos b;
    b.block = i / per;
    int r = i - b.block * per;
    b.ox = (r % P.bricks[0]) * BX;
    r /= P.bricks[0];
    b.oy = (r % P.bricks[1]) * BY;
    b.oz = (r / P.bricks[1]) * BZ;
    return b;
}

template <int MODE>
__global__ void __launch_bounds__(PIPE_THREADS, 1) conv3_tc_pipe(const __grid_constant__ Params P, int nbricks)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *Abuf = smem;                             // [2][2 planes][SROWS][16 B]
    unsigned char *Bw = smem + 4 * PLANE;                   // [27][2][16][16 B]
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + PIPE_BAR_OFF);
    uint64_t *full = bars, *empty = bars + 2, *tfull = bars + 4, *tempty = bars + 6, *fin = bars + 8;
    uint32_t *slot = reinterpret_cast<uint32_t *>(bars + 9);
    int *snb = reinterpret_cast<int *>(slot + 2);           // [2][28]: neighbour blocks per A buffer
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cells = P.n[0] * P.n[1] * P.n[2];

    if (threadIdx.x == 0) {
        for (int b = 0; b < 2; ++b) {
            mbar_init(full + b, PRODUCERS);
            mbar_init(empty + b, 1);
            mbar_init(tfull + b, 1);
            mbar_init(tempty + b, 128);
        }
        mbar_init(fin, 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        tc::tmem_alloc(slot, PIPE_TMEM_COLS);
        tc::tmem_relinquish();
    }
    // weights once; rows past the region stay zero in both A buffers
    for (int i = threadIdx.x; i < 27 * 32; i += PIPE_THREADS)
        reinterpret_cast<uint4 *>(Bw)[i] = __ldg(reinterpret_cast<const uint4 *>(P.w) + i);
    for (int t = threadIdx.x; t < 4 * (SROWS - RCELLS); t += PIPE_THREADS) {
        const int b = t / (2 * (SROWS - RCELLS)), r = t % (2 * (SROWS - RCELLS));
        const int kc = r / (SROWS - RCELLS), u = RCELLS + r % (SROWS - RCELLS);
        *reinterpret_cast<uint4 *>(Abuf + b * 2 * PLANE + kc * PLANE + u * 16) = make_uint4(0u, 0u, 0u, 0u);
    }
    fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = *slot;

    if (warp < 2) {
        // ---------------- producers
        int k = 0;
        for (int i = blockIdx.x; i < nbricks; i += gridDim.x, ++k) {
            const int b = k & 1;
            int *nbt = snb + 28 * b;
            // one thread waits for the buffer; the verdict is shared so that
            // all producers leave together (the named barrier stays matched)
            if (threadIdx.x == 0)
                nbt[27] = (k < 2 || mbar_wait_bounded(empty + b, ((k >> 1) - 1) & 1)) ? 1 : 0;
            named_sync(1, PRODUCERS);
            if (!nbt[27]) {
                if (threadIdx.x == 0 && P.err) atomicExch(P.err, kDevErrTimeout);
                break;
            }
            const BrickPos q = brick_pos(P, i);
            if (threadIdx.x < 27) {
                const int t = threadIdx.x;
                int bx = q.block % P.nb[0] + t % 3 - 1, by = (q.block / P.nb[0]) % P.nb[1] + (t / 3) % 3 - 1,
                    bz = q.block / (P.nb[0] * P.nb[1]) + t / 9 - 1;
                bx = bx < 0 ? bx + P.nb[0] : (bx >= P.nb[0] ? bx - P.nb[0] : bx);
                by = by < 0 ? by + P.nb[1] : (by >= P.nb[1] ? by - P.nb[1] : by);
                bz = bz < 0 ? bz + P.nb[2] : (bz >= P.nb[2] ? bz - P.nb[2] : bz);
                nbt[t] = bx + P.nb[0] * (by + P.nb[1] * bz);
            }
            named_sync(1, PRODUCERS);
            unsigned char *A = Abuf + b * 2 * PLANE;
            for (int t = threadIdx.x; t < 2 * RCELLS; t += PRODUCERS) {
                const int u = t >> 1, kc = t & 1;
                const int ii = u % RX, jj = (u / RX) % RY, kk = u / (RX * RY);
                const int x = q.ox + ii - 1, y = q.oy + jj - 1, z = q.oz + kk - 1;
                const int r0 = x < 0 ? -1 : (x >= P.n[0] ? 1 : 0), r1 = y < 0 ? -1 : (y >= P.n[1] ? 1 : 0),
                          r2 = z < 0 ? -1 : (z >= P.n[2] ? 1 : 0);
                const int sb = nbt[(r0 + 1) + 3 * (r1 + 1) + 9 * (r2 + 1)];
                const int sc = (x - r0 * P.n[0]) + P.n[0] * ((y - r1 * P.n[1]) + P.n[1] * (z - r2 * P.n[2]));
                const uint16_t *src = P.act + ((int64_t)sb * cells + sc) * 16 + kc * 8;
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(A + kc * PLANE + u * 16)),
                             "l"(src)
                             : "memory");
            }
            cp_async_arrive_noinc(full + b);
            named_sync(1, PRODUCERS); // nbt of this buffer stays untouched until the next use
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    } else if (warp == MMA_WARP) {
        // ---------------- MMA issuer
        if (lane == 0) {
            const uint64_t db = tc::smem_desc(smem_u32(Bw), 256u, 128u);
            int k = 0;
            bool issued = false;
            for (int i = blockIdx.x; i < nbricks; i += gridDim.x, ++k) {
                const int b = k & 1;
                if (!mbar_wait_bounded(full + b, (k >> 1) & 1) ||
                    (k >= 2 && !mbar_wait_bounded(tempty + b, ((k >> 1) - 1) & 1))) {
                    if (P.err) atomicExch(P.err, kDevErrTimeout);
                    break;
                }
                fence_proxy_async_smem(); // the producers' copies -> the tensor cores' view
                tc::fence_after_sync();
                const uint64_t da = tc::smem_desc(smem_u32(Abuf + b * 2 * PLANE), PLANE, 128u);
                const uint32_t acc = tbase + 256u * b;
#pragma unroll 1
                for (int t = 0; t < MT; ++t) {
#pragma unroll
                    for (int q = 0; q < 27; ++q) {
                        const int off = (q % 3 - 1) + RX * ((q / 3) % 3 - 1) + RX * RY * (q / 9 - 1);
                        tc::mma_bf16(acc + 16u * t, da + (uint64_t)(R0 + 128 * t + off),
                                     db + (uint64_t)(q * (WTAP / 16)), IDESC, q > 0 ? 1u : 0u);
                    }
                }
                tc::mma_commit(empty + b);
                tc::mma_commit(tfull + b);
                issued = true;
            }
            if (issued) { // everything issued has finished before TMEM is freed
                tc::mma_commit(fin);
                if (!mbar_wait_bounded(fin, 0) && P.err) atomicExch(P.err, kDevErrTimeout);
            }
        }
    } else if (warp >= EPI_WARP0) {
        // ---------------- epilogue
        const int qd = warp - EPI_WARP0;
        const uint32_t lane_base = (uint32_t)(32 * qd) << 16;
        int k = 0;
        for (int i = blockIdx.x; i < nbricks; i += gridDim.x, ++k) {
            const int a = k & 1;
            // warp-uniform verdict: the TMEM loads below are warp-collective
            const int got = __shfl_sync(0xffffffffu, lane == 0 ? (mbar_wait_bounded(tfull + a, (k >> 1) & 1) ? 1 : 0) : 0, 0);
            if (!got) {
                if (lane == 0 && P.err) atomicExch(P.err, kDevErrTimeout);
                break;
            }
            tc::fence_after_sync();
            const BrickPos q = brick_pos(P, i);
#pragma unroll 1
            for (int t = 0; t < MT; ++t) {
                float v[16];
                tc::tmem_ld16(tbase + 256u * a + lane_base + 16u * t, v);
                const int m = 128 * t + 32 * qd + lane;
                const int z = m / (RX * RY), rem = m - z * (RX * RY);
                const int y = rem / RX, x = rem - y * RX;
                if (x >= BX || y >= BY || z >= BZ)
                    continue;
                const int c = (q.ox + x) + P.n[0] * ((q.oy + y) + P.n[1] * (q.oz + z));
                if (MODE == 2) {
                    const int64_t o = (int64_t)q.block * P.pbs + c;
                    const float x0 = __ldg(P.x + (int64_t)q.block * P.xbs + c);
                    const float pv = P.zero_guess ? 0.f : P.p[o];
                    P.p[o] = pv + (P.omega * x0 + v[0]);
                } else {
                    uint32_t h[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        float a0 = v[2 * j], b0 = v[2 * j + 1];
                        if (P.relu) {
                            a0 = fmaxf(a0, 0.f);
                            b0 = fmaxf(b0, 0.f);
                        }
                        h[j] = (uint32_t)bf16_bits(a0) | ((uint32_t)bf16_bits(b0) << 16);
                    }
                    uint4 *dst = reinterpret_cast<uint4 *>(P.out + ((int64_t)q.block * cells + c) * 16);
                    dst[0] = make_uint4(h[0], h[1], h[2], h[3]);
                    dst[1] = make_uint4(h[4], h[5], h[6], h[7]);
                }
            }
            tc::fence_before_sync();
            mbar_arrive(tempty + a);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0)
        tc::tmem_dealloc(tbase, PIPE_TMEM_COLS);
}

// FP32 weights [27][cin][cout] -> BF16 B tiles [27][kc][co][8] (B[co][ci] = W[tap][ci][co])
__global__ void pack_weights_kernel(const float *W, int cin, int cout, uint16_t *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x; // [27][2][16][8]
    if (i >= 27 * 256)
        return;
    const int tap = i / 256, r = i % 256;
    const int kc = r / 128, co = (r / 8) % 16, e = r % 8;
    const int ci = kc * 8 + e;
    const float v = (ci < cin && co < cout) ? W[(tap * cin + ci) * cout + co] : 0.f;
    out[i] = bf16_bits(v);
}

static DeviceOnce attr_set[3], pipe_attr_set[3]; // per mode (1: hidden layer, 2: last layer + update) and device
// kernel form: 1 = persistent warp-specialised pipeline, 0 = one brick per CTA
static int g_conv_form = 1;

template <int MODE>
static cn_status launch(const Params &P, int nblocks, cudaStream_t st)
{
    const int64_t bricks = (int64_t)nblocks * P.bricks[0] * P.bricks[1] * P.bricks[2];
    if (g_conv_form == 1) {
        cn_status s = smem_opt_in(pipe_attr_set[MODE], conv3_tc_pipe<MODE>, PIPE_SMEM);
        if (s != CN_OK) return s;
        int dev = 0, sms = 148;
        CN_CUDA_TRY(cudaGetDevice(&dev));
        CN_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const int64_t grid = bricks < sms ? bricks : sms;
        conv3_tc_pipe<MODE><<<(unsigned)grid, PIPE_THREADS, PIPE_SMEM, st>>>(P, (int)bricks);
        CN_CUDA_TRY(cudaGetLastError());
        return CN_OK;
    }
    cn_status s = smem_opt_in(attr_set[MODE], conv3_tc_kernel<MODE>, SMEM);
    if (s != CN_OK) return s;
    conv3_tc_kernel<MODE><<<(unsigned)bricks, NTHREADS, SMEM, st>>>(P);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

void set_form(int form) { g_conv_form = form ? 1 : 0; }

bool supported(const int n[3])
{
    return n[0] % BX == 0 && n[1] % BY == 0 && n[2] % BZ == 0;
}

cn_status pack_weights(const float *W, int cin, int cout, uint16_t *out, cudaStream_t st)
{
    pack_weights_kernel<<<(27 * 256 + 255) / 256, 256, 0, st>>>(W, cin, cout, out);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

static Params base_params(const int nb[3], const int n[3], int *err)
{
    Params P = {};
    for (int d = 0; d < 3; ++d) {
        P.nb[d] = nb[d];
        P.n[d] = n[d];
    }
    P.bricks[0] = n[0] / BX;
    P.bricks[1] = n[1] / BY;
    P.bricks[2] = n[2] / BZ;
    P.err = err;
    return P;
}

cn_status conv_hidden(const uint16_t *act, const int nb[3], const int n[3], const uint16_t *w, int relu,
                      uint16_t *out, int *err, cudaStream_t st)
{
    Params P = base_params(nb, n, err);
    P.act = act;
    P.w = w;
    P.out = out;
    P.relu = relu;
    return launch<1>(P, nb[0] * nb[1] * nb[2], st);
}

cn_status conv_update(const uint16_t *act, const int nb[3], const int n[3], const uint16_t *w, const float *x0,
                      int64_t xbs, float *p, int64_t pbs, float omega, int zero_guess, int *err, cudaStream_t st)
{
    Params P = base_params(nb, n, err);
    P.act = act;
    P.w = w;
    P.x = x0;
    P.xbs = xbs;
    P.p = p;
    P.pbs = pbs;
    P.omega = omega;
    P.zero_guess = zero_guess;
    return launch<2>(P, nb[0] * nb[1] * nb[2], st);
}

} // namespace nntc
} // namespace cn

using namespace cn;

extern "C" cn_status cn_conv3_bf16(const void *in, void *out, const int nblocks[3], const int block_cells[3],
                                   const float *weights, int relu, void *stream)
{
    if (!in || !out || !nblocks || !block_cells || !weights)
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_conv3_bf16: NULL argument");
    for (int d = 0; d < 3; ++d)
        if (nblocks[d] < 1 || block_cells[d] < 1)
            return fail(CN_ERR_INVALID_ARGUMENT, "cn_conv3_bf16: bad grid shape");
    if (!nntc::supported(block_cells))
        return fail(CN_ERR_UNSUPPORTED, "cn_conv3_bf16: block cells must be multiples of (16, 16, 4)");
    cudaStream_t st = as_stream(stream);
    uint16_t *w = nullptr;
    CN_CUDA_TRY(cudaMallocAsync(&w, 27 * nntc::WTAP, st));
    cn_status s = nntc::pack_weights(weights, 16, 16, w, st);
    if (s == CN_OK)
        s = nntc::conv_hidden(static_cast<const uint16_t *>(in), nblocks, block_cells, w, relu,
                              static_cast<uint16_t *>(out), nullptr, st);
    cudaFreeAsync(w, st);
    return s;
}
