// learned_cc.cu -- the learned smoother's first and last convolutions on the
// CUDA cores, for grid inference beside the tensor-core hidden layer.
//
// The first layer has 2 input channels and the last 1 output channel: on the
// tensor cores (K and N padded to 16) each costs as much as the 16 -> 16
// hidden layer, whose shared-memory operand reads bound it.  Here a CTA owns
// a brick of 16 x 16 x 4 output cells of one block, stages the 18 x 18 x 6
// input region (neighbours across blocks periodic, as on the activation
// grids) in shared memory, and each thread accumulates one (x, y) column of
// 4 cells in FP32: taps outer (the tap's weights loaded once, broadcast from
// shared memory), the column's 4 cells inner.
//   layer 1: in = (x0, x1), the FP32 features grid (two components);
//            out = ReLU, 16 channels, BF16 channels-last.
//   layer 3: in = 16 channels BF16 channels-last; y = sum, then the update
//            p = (zero guess ? 0 : p) + (omega x0 + y).
// Weights FP32 [27][cin][cout] (the network's master copy).
#include "cn_internal.h"
#include "learned_tc.h"
#include "mg_tile.cuh"

#include <cuda_bf16.h>

namespace cn {
namespace nncc {

constexpr int BX = 16, BY = 16, BZ = 4;
constexpr int RX = BX + 2, RY = BY + 2, RZ = BZ + 2;
constexpr int RCELLS = RX * RY * RZ; // 1944
constexpr int NT = BX * BY;          // one column of BZ cells per thread

struct Geo {
    int nb[3], n[3], bricks[3];
};

struct Brick {
    int block, ox, oy, oz;
};

__device__ __forceinline__ Brick brick_of(const Geo &G)
{
    const int per = G.bricks[0] * G.bricks[1] * G.bricks[2];
    Brick b;
    b.block = blockIdx.x / per;
    int r = blockIdx.x - b.block * per;
    b.ox = (r % G.bricks[0]) * BX;
    r /= G.bricks[0];
    b.oy = (r % G.bricks[1]) * BY;
    b.oz = (r / G.bricks[1]) * BZ;
    return b;
}

// block and in-block cell of region cell u (periodic neighbour blocks from snb)
__device__ __forceinline__ int64_t region_src(const Geo &G, const Brick &q, const int *snb, int u, int64_t cells_per)
{
    const int i = u % RX, j = (u / RX) % RY, k = u / (RX * RY);
    const int x = q.ox + i - 1, y = q.oy + j - 1, z = q.oz + k - 1;
    const int r0 = x < 0 ? -1 : (x >= G.n[0] ? 1 : 0), r1 = y < 0 ? -1 : (y >= G.n[1] ? 1 : 0),
              r2 = z < 0 ? -1 : (z >= G.n[2] ? 1 : 0);
    const int sb = snb[(r0 + 1) + 3 * (r1 + 1) + 9 * (r2 + 1)];
    const int sc = (x - r0 * G.n[0]) + G.n[0] * ((y - r1 * G.n[1]) + G.n[1] * (z - r2 * G.n[2]));
    return (int64_t)sb * cells_per + sc;
}

__device__ __forceinline__ uint32_t bf16x2_bits(float a, float b)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b); // a -> low half
    return *reinterpret_cast<const uint32_t *>(&h);
}

// layer 1: 2 -> 16 channels, ReLU, BF16 out
__global__ void __launch_bounds__(NT, 2) layer1_kernel(const Geo G, const float *__restrict__ x0,
                                                       const float *__restrict__ x1, int64_t xbs,
                                                       const float *__restrict__ W, uint16_t *__restrict__ out)
{
    __shared__ __align__(16) float sw[27 * 2 * 16];
    __shared__ float2 sx[RCELLS];
    __shared__ int snb[27];
    const Brick q = brick_of(G);
    for (int i = threadIdx.x; i < 27 * 2 * 16; i += NT) sw[i] = __ldg(W + i);
    mg::neighbour_blocks(G.nb, q.block, snb);
    __syncthreads();
    for (int u = threadIdx.x; u < RCELLS; u += NT) {
        const int64_t o = region_src(G, q, snb, u, xbs); // the features grid: blocks xbs apart
        sx[u] = make_float2(__ldg(x0 + o), __ldg(x1 + o));
    }
    __syncthreads();
    const int cx = threadIdx.x % BX, cy = threadIdx.x / BX;
    float acc[BZ][16];
#pragma unroll
    for (int z = 0; z < BZ; ++z)
#pragma unroll
        for (int c = 0; c < 16; ++c)
            acc[z][c] = 0.f;
#pragma unroll 1
    for (int t = 0; t < 27; ++t) {
        const int dx = t % 3, dy = (t / 3) % 3, dz = t / 9;
        float w0[16], w1[16];
#pragma unroll
        for (int c = 0; c < 16; c += 4) {
            const float4 a = *reinterpret_cast<const float4 *>(sw + t * 32 + c);
            const float4 b = *reinterpret_cast<const float4 *>(sw + t * 32 + 16 + c);
            w0[c] = a.x; w0[c + 1] = a.y; w0[c + 2] = a.z; w0[c + 3] = a.w;
            w1[c] = b.x; w1[c + 1] = b.y; w1[c + 2] = b.z; w1[c + 3] = b.w;
        }
        const float2 *src = sx + (cx + dx) + RX * ((cy + dy) + RY * dz);
#pragma unroll
        for (int z = 0; z < BZ; ++z) {
            const float2 v = src[RX * RY * z];
#pragma unroll
            for (int c = 0; c < 16; ++c)
                acc[z][c] = fmaf(v.x, w0[c], fmaf(v.y, w1[c], acc[z][c]));
        }
    }
    const int64_t cells = (int64_t)G.n[0] * G.n[1] * G.n[2];
#pragma unroll
    for (int z = 0; z < BZ; ++z) {
        const int64_t c = (int64_t)q.block * cells + (q.ox + cx) + G.n[0] * ((q.oy + cy) + (int64_t)G.n[1] * (q.oz + z));
        uint32_t h[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            h[j] = bf16x2_bits(fmaxf(acc[z][2 * j], 0.f), fmaxf(acc[z][2 * j + 1], 0.f));
        uint4 *dst = reinterpret_cast<uint4 *>(out + c * 16);
        dst[0] = make_uint4(h[0], h[1], h[2], h[3]);
        dst[1] = make_uint4(h[4], h[5], h[6], h[7]);
    }
}

// layer 3: 16 -> 1 channel, fused with p = (zero guess ? 0 : p) + (omega x0 + y)
__global__ void __launch_bounds__(NT, 2) layer3_kernel(const Geo G, const uint16_t *__restrict__ act,
                                                       const float *__restrict__ W, const float *__restrict__ x0,
                                                       int64_t xbs, float *__restrict__ p, int64_t pbs, float omega,
                                                       int zero_guess)
{
    __shared__ __align__(16) float sw[27 * 16];
    // channels 0-7 and 8-15 of the region cells in two arrays (consecutive
    // cells 16 bytes apart: conflict-free 16-byte accesses)
    extern __shared__ __align__(16) uint4 sa_dyn[];
    uint4 *sa0 = sa_dyn, *sa1 = sa_dyn + RCELLS;
    __shared__ int snb[27];
    const Brick q = brick_of(G);
    for (int i = threadIdx.x; i < 27 * 16; i += NT) sw[i] = __ldg(W + i);
    mg::neighbour_blocks(G.nb, q.block, snb);
    __syncthreads();
    const int64_t cells = (int64_t)G.n[0] * G.n[1] * G.n[2];
    for (int t = threadIdx.x; t < 2 * RCELLS; t += NT) {
        const int u = t >> 1, half = t & 1;
        const uint16_t *s = act + region_src(G, q, snb, u, cells) * 16 + 8 * half;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32((half ? sa1 : sa0) + u)), "l"(s)
                     : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    const int cx = threadIdx.x % BX, cy = threadIdx.x / BX;
    float acc[BZ] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 1
    for (int t = 0; t < 27; ++t) {
        const int dx = t % 3, dy = (t / 3) % 3, dz = t / 9;
        float w[16];
#pragma unroll
        for (int c = 0; c < 16; c += 4) {
            const float4 a = *reinterpret_cast<const float4 *>(sw + t * 16 + c);
            w[c] = a.x; w[c + 1] = a.y; w[c + 2] = a.z; w[c + 3] = a.w;
        }
        const int u0 = (cx + dx) + RX * ((cy + dy) + RY * dz);
#pragma unroll
        for (int z = 0; z < BZ; ++z) {
            const uint4 a = sa0[u0 + RX * RY * z], b = sa1[u0 + RX * RY * z];
            const uint32_t v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
            float s = acc[z];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                // channel 2j in the low half, 2j+1 in the high half (BF16 = top 16 bits of an FP32)
                s = fmaf(__uint_as_float(v[j] << 16), w[2 * j], s);
                s = fmaf(__uint_as_float(v[j] & 0xFFFF0000u), w[2 * j + 1], s);
            }
            acc[z] = s;
        }
    }
#pragma unroll
    for (int z = 0; z < BZ; ++z) {
        const int64_t c = (q.ox + cx) + G.n[0] * ((q.oy + cy) + (int64_t)G.n[1] * (q.oz + z));
        const int64_t o = (int64_t)q.block * pbs + c;
        const float xv = __ldg(x0 + (int64_t)q.block * xbs + c);
        const float pv = zero_guess ? 0.f : p[o];
        p[o] = pv + (omega * xv + acc[z]);
    }
}

static Geo geo(const int nb[3], const int n[3])
{
    Geo G;
    for (int d = 0; d < 3; ++d) {
        G.nb[d] = nb[d];
        G.n[d] = n[d];
    }
    G.bricks[0] = n[0] / BX;
    G.bricks[1] = n[1] / BY;
    G.bricks[2] = n[2] / BZ;
    return G;
}

static unsigned bricks_of(const Geo &G)
{
    return (unsigned)((int64_t)G.nb[0] * G.nb[1] * G.nb[2] * G.bricks[0] * G.bricks[1] * G.bricks[2]);
}

} // namespace nncc

namespace nntc {

cn_status conv_first_cc(const float *x0, const float *x1, int64_t xbs, const int nb[3], const int n[3],
                        const float *W1, uint16_t *out, cudaStream_t st)
{
    const nncc::Geo G = nncc::geo(nb, n);
    nncc::layer1_kernel<<<nncc::bricks_of(G), nncc::NT, 0, st>>>(G, x0, x1, xbs, W1, out);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

cn_status conv_update_cc(const uint16_t *act, const int nb[3], const int n[3], const float *W3, const float *x0,
                         int64_t xbs, float *p, int64_t pbs, float omega, int zero_guess, cudaStream_t st)
{
    const nncc::Geo G = nncc::geo(nb, n);
    constexpr size_t smem = (size_t)nncc::RCELLS * 2 * sizeof(uint4);
    static DeviceOnce once; // per device
    cn_status s = smem_opt_in(once, nncc::layer3_kernel, smem);
    if (s != CN_OK) return s;
    nncc::layer3_kernel<<<nncc::bricks_of(G), nncc::NT, smem, st>>>(G, act, W3, x0, xbs, p, pbs, omega, zero_guess);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

} // namespace nntc
} // namespace cn
