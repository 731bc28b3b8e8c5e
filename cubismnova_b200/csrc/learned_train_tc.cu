// learned_train_tc.cu -- training of the learned smoother with its hidden
// layer (16 -> 16 channels, 84 % of the network's multiply-adds) on the
// tensor cores (tcgen05, BF16 operands, FP32 accumulation in tensor memory),
// and the first and last layers on the CUDA cores, all on BF16 channels-last
// activations (32 bytes per cell).
//
// Patches are cubes: the input x has side S = P + 8, the activations h1 side
// S1 = S - 2, h2 side S2 = S - 4, the output y side S3 = S - 6 (valid 3x3x3
// convolutions; tap d = (dx, dy, dz) in {0,1,2}^3, index dx + 3 dy + 9 dz).
//
// The hidden layer's three GEMMs:
//   forward        out[q][co] = sum_{t,ci} h1[q + d][ci] W[t][ci][co]
//   backward-data  gin[c][ci] = sum_e gout[c - 2 + e][co] W[26 - e][ci][co],
//                  the forward's form with the source gout, shift -2, taps
//                  flipped and W transposed; the ReLU mask of the layer's
//                  input applied in the epilogue
// run brick-staged (brick_tc_kernel): a brick of output cells with its
// source region in shared memory, each tap's A operand the same rows
// shifted (K-major, M = 128 cells, K = 16 channels, N = 16), 27 MMAs per
// 128-row tile.
//   weight grad    gW[t][ci][co] = sum_q h1[q + d][ci] gout[q][co]
// needs M = (tap, channel), which no shifted descriptor gives (the tap
// offsets are not evenly spaced): wgrad_tc_kernel gathers, for a chunk of
// 128 consecutive output cells (linear over batch and cube), per tap t and
// channel half h a plane of 128 rows x 16 bytes (row r = channels
// 8h..8h+7 of source cell (cell r) + d(t), zero outside the cube; one
// 16-byte cp.async each), reads them MN-major (8 taps = 16 planes per
// M = 128 tile, planes one SBO apart; K = cells, 16 rows per MMA) against
// the chunk's gout rows (MN-major B, N = 16): 4 tiles x 8 MMAs per chunk,
// accumulated over all chunks of a CTA in tensor memory, added to gW with
// atomics at the end.  Rows of taps >= 27 in the last tile read whatever
// the buffer holds; those accumulator rows are never read.  Taps are
// gathered in 4 groups of 8 into two 32 KB buffers, one group ahead of the
// MMAs (issued by one thread, committed to the buffer's mbarrier); lanes 2i
// and 2i+1 copy the two channel halves of one row.  Persistent CTAs, two
// per SM.  Every wait in both kernels is bounded (an error word is set and
// the CTA stops issuing).
#include "cn_internal.h"
#include "cn_tc.cuh"
#include "cn_tma.cuh"
#include "learned_tc.h"

#include <cuda_bf16.h>

#include <type_traits>

namespace cn {
namespace nntr {

constexpr int ROWS = 128;                        // cells per chunk
constexpr int GT = 8;                            // taps per gather group
constexpr int NG = 4;                            // groups per chunk (taps 0-7, 8-15, 16-23, 24-26)
constexpr uint32_t PL = ROWS * 16;               // bytes of one plane
constexpr uint32_t GBUF = 2 * GT * PL;           // one group buffer: 16 planes, 32 KB
constexpr int NT = 2 * ROWS;                     // two threads per row (channel halves)
constexpr uint32_t WBYTES = 27 * 512;            // packed weights of one layer
constexpr uint32_t GOUT_BYTES = 2 * PL;          // gout rows of a chunk (2 planes)
constexpr size_t OFF_G = 2 * (size_t)GBUF;       // two gout buffers
constexpr size_t OFF_BAR = OFF_G + 2 * GOUT_BYTES;
constexpr size_t SMEM = OFF_BAR + 4 * 8 + 16;
constexpr uint32_t IDESC_K = tc::idesc_bf16_f32(128, 16);
// both operands MN-major (bits 15 and 16)
constexpr uint32_t IDESC_MN = tc::idesc_bf16_f32(128, 16) | (1u << 15) | (1u << 16);

enum { FWD = 0, BWD = 1 };

struct Args {
    const uint16_t *src;  // gathered activations [B][Sin^3][16] BF16
    const uint16_t *gout; // weight gradient: [B][Sout^3][16] gradient at the layer's output
    const uint16_t *act;  // backward-data: the layer's input at the output cells (ReLU mask)
    const uint16_t *w;    // forward / backward-data: packed B tiles [27][2][16][8]
    uint16_t *out;        // forward / backward-data: [B][Sout^3][16]
    float *gw;            // weight gradient: [27][16][16] FP32, accumulated
    int Sin, Sout, shift;
    int relu;
    int64_t total;        // B * Sout^3
    int64_t chunks;       // ceil(total / ROWS)
    int *err;
};

__device__ __forceinline__ uint16_t bf16_bits(float v) { return __bfloat16_as_ushort(__float2bfloat16_rn(v)); }

// cell index q of a batch of cubes of side n (n3 = n^3; indices below 2^31,
// checked on the host) -> patch b and (x, y, z); 32-bit divisions
struct CubeIdx {
    int b, x, y, z;
};
__device__ __forceinline__ CubeIdx cube_idx(uint32_t q, uint32_t n, uint32_t n3)
{
    CubeIdx c;
    const uint32_t b = q / n3, rem = q - b * n3, zy = rem / n, z = zy / n;
    c.b = (int)b;
    c.x = (int)(rem - zy * n);
    c.z = (int)z;
    c.y = (int)(zy - z * n);
    return c;
}

// 16-byte asynchronous copy; src_bytes 0 writes zeros (nothing is read)
__device__ __forceinline__ void cp16(void *dst, const void *src, uint32_t src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}

template <int V> using ic = std::integral_constant<int, V>;

__global__ void __launch_bounds__(NT, 2) wgrad_tc_kernel(const __grid_constant__ Args a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *Abuf = smem;                 // [2][16 planes][ROWS][16 B]
    unsigned char *Gbuf = smem + OFF_G;         // [2][2 planes][ROWS][16 B]
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + OFF_BAR);
    uint64_t *empty = bars, *done = bars + 2;   // empty[2]: group buffer free; done: all MMAs complete
    uint32_t *slot = reinterpret_cast<uint32_t *>(bars + 4);
    int *flag = reinterpret_cast<int *>(slot + 1); // [0]: buffer waits, [1]: the final wait
    constexpr uint32_t TCOLS = 64;                 // 4 accumulator tiles x 16 columns
    const int r = threadIdx.x, warp = r >> 5;

    if (r == 0) {
        mbar_init(empty, 1);
        mbar_init(empty + 1, 1);
        mbar_init(done, 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        tc::tmem_alloc(slot, TCOLS);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = *slot;

    const uint32_t so3 = (uint32_t)a.Sout * a.Sout * a.Sout;
    const int64_t si3 = (int64_t)a.Sin * a.Sin * a.Sin, sin1 = a.Sin, sin2 = (int64_t)a.Sin * a.Sin;
    const int nch = (int64_t)blockIdx.x < a.chunks ? (int)((a.chunks - 1 - blockIdx.x) / gridDim.x + 1) : 0;
    const int nitems = NG * nch; // items (chunk j of this CTA, tap group g): i = NG j + g, buffer g & 1
    // gather: thread r copies channel half hh of row rho (a warp: 16 rows =
    // 512 contiguous source bytes where the cells are contiguous)
    const int hh = r & 1, rho = r >> 1;
    int64_t rL = 0, roff = 0; // the row's cell; source element of its tap (0, 0, 0)
    uint32_t mx = 0, my = 0, mz = 0; // per axis: offsets k = 0..2 with the source inside the cube
    auto set_row = [&](int j) {
        rL = (blockIdx.x + (int64_t)j * gridDim.x) * ROWS + rho;
        mx = my = mz = 0;
        if (rL < a.total) {
            const CubeIdx ci = cube_idx((uint32_t)rL, (uint32_t)a.Sout, so3);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                mx |= ((unsigned)(ci.x + k) < (unsigned)a.Sin ? 1u : 0u) << k;
                my |= ((unsigned)(ci.y + k) < (unsigned)a.Sin ? 1u : 0u) << k;
                mz |= ((unsigned)(ci.z + k) < (unsigned)a.Sin ? 1u : 0u) << k;
            }
            roff = (int64_t)ci.b * si3 + ci.x + sin1 * ci.y + sin2 * ci.z;
        }
    };
    auto gather = [&](int j, auto G) {
        constexpr int g = decltype(G)::value;
        if (g == 0) {
            set_row(j);
            // the chunk's gradient rows (buffer j & 1 was last read by chunk j - 2's
            // MMAs, complete before item NG j - 2's)
            const bool v = rL < a.total;
            cp16(Gbuf + (j & 1) * GOUT_BYTES + hh * PL + rho * 16, v ? a.gout + rL * 16 + 8 * hh : a.gout,
                 v ? 16u : 0u);
        }
        unsigned char *A = Abuf + (g & 1) * GBUF;
#pragma unroll
        for (int tl = 0; tl < GT; ++tl) {
            const int t = g * GT + tl;
            if (t < 27) {
                const int dx = t % 3, dy = (t / 3) % 3, dz = t / 9;
                const bool in = ((mx >> dx) & (my >> dy) & (mz >> dz) & 1u) != 0;
                const uint16_t *src = in ? a.src + (roff + dx + sin1 * dy + sin2 * dz) * 16 + 8 * hh : a.src;
                cp16(A + (2 * tl + hh) * PL + rho * 16, src, in ? 16u : 0u);
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    // one item: gather the next (after its buffer's previous MMAs), wait
    // for this item's copies, issue its MMAs.  False when a bounded wait ran
    // out.
    auto item = [&](int j, auto G) -> bool {
        constexpr int g = decltype(G)::value;
        const int i = NG * j + g;
        if (i + 1 < nitems) {
            if (i >= 1) {
                if (r == 0)
                    flag[0] = mbar_wait_bounded(empty + ((g + 1) & 1), (((i + 1) >> 1) - 1) & 1) ? 1 : 0;
                __syncthreads();
                if (!flag[0]) return false;
            }
            if constexpr (g == NG - 1) gather(j + 1, ic<0>{});
            else gather(j, ic<g + 1>{});
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        fence_proxy_async_smem(); // generic-proxy smem writes -> visible to the tensor cores
        tc::fence_before_sync();
        __syncthreads();
        if (r == 0) {
            tc::fence_after_sync();
            const uint32_t A = smem_u32(Abuf + (g & 1) * GBUF), Gs = smem_u32(Gbuf + (j & 1) * GOUT_BYTES);
#pragma unroll
            for (int ks = 0; ks < ROWS / 16; ++ks) {
                const uint64_t da = tc::smem_desc(A + 256u * ks, 128u, PL);
                const uint64_t db = tc::smem_desc(Gs + 256u * ks, 128u, PL);
                tc::mma_bf16(tbase + 16u * g, da, db, IDESC_MN, (j > 0 || ks > 0) ? 1u : 0u);
            }
            tc::mma_commit(empty + (g & 1));
        }
        return true;
    };

    bool ok = true;
    if (nitems > 0) gather(0, ic<0>{});
    for (int j = 0; j < nch && ok; ++j)
        ok = item(j, ic<0>{}) && item(j, ic<1>{}) && item(j, ic<2>{}) && item(j, ic<3>{});
    asm volatile("cp.async.wait_all;" ::: "memory"); // nothing in flight past this point
    // ---- wait for every MMA of this CTA, then add the 4 accumulator tiles
    // (row m = 16 (tap - 8 g) + ci, column co) to gW; warp w reads rows
    // 32 (w % 4) + lane, columns 8 (w / 4) .. + 7
    if (ok && nitems > 0) {
        if (r == 0) {
            tc::mma_commit(done);
            flag[1] = mbar_wait_bounded(done, 0) ? 1 : 0;
        }
        __syncthreads();
        ok = flag[1] != 0;
        if (ok) {
            tc::fence_after_sync();
            const int m = 32 * (warp & 3) + (r & 31), ch = 8 * (warp >> 2);
#pragma unroll 1
            for (int g = 0; g < NG; ++g) {
                float v[8];
                tc::tmem_ld8(tbase + ((uint32_t)(32 * (warp & 3)) << 16) + 16u * g + (uint32_t)ch, v);
                const int t = g * GT + m / 16, ci = m % 16;
                if (t < 27) {
#pragma unroll
                    for (int k = 0; k < 8; ++k) atomicAdd(a.gw + (t * 16 + ci) * 16 + ch + k, v[k]);
                }
            }
        }
    }
    if (!ok && r == 0 && a.err) atomicExch(a.err, kDevErrTimeout);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tbase, TCOLS);
}

// backward-data B tiles: tap e, K = the layer's output channel co, N = its
// input channel ci: B[e][kc][ci][8] = W[26 - e][ci][kc * 8 + j]
__global__ void pack_bwd_kernel(const float *W, uint16_t *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 27 * 256) return;
    const int e = i / 256, rr = i % 256;
    const int kc = rr / 128, ci = (rr / 8) % 16, j = rr % 8;
    out[i] = bf16_bits(W[((26 - e) * 16 + ci) * 16 + kc * 8 + j]);
}

// ------------------------------------------------ brick-staged forward
// The forward and data-gradient GEMMs without im2col, as the grid inference
// kernel does it: a CTA owns a brick of BX x BY x BZ output cells of one
// patch (BX the whole row) and stages the source region around it, (BX+2) x
// (BY+2) x (BZ+2) cells starting at the brick origin + shift, zero outside
// the source cube, one row of 16 channels per region cell (two K planes of
// 16-byte rows).  Output cell (x, y, z) sits at row m = x + RX y + RX RY z
// and its tap e source at row m + e_x + RX e_y + RX RY e_z, so a tap's A
// operand for a 128-row tile is the same run of rows shifted: 27 MMAs (M =
// 128, N = 16, K = 16) per tile into one TMEM accumulator.  Rows whose (x,
// y, z) fall outside the brick or the output cube are computed and dropped.
// One brick per CTA; the wait for the MMAs is bounded (error word, skipped
// epilogue).
struct BrickGeo {
    int BX, BY, BZ;        // brick of output cells
    int RX, RY, RZ;        // source region = brick + 2
    int MT;                // 128-row M tiles covering the brick's rows
    int SROWS;             // staged rows: 128 MT + the largest tap offset (zero past the region)
    int bricks[3];         // bricks per patch along x, y, z
};

constexpr int BRICK_NT = 256;
constexpr int BRICK_MAX_ROWS = 2880;    // 2 planes x 2880 x 16 B = 90 KB: two CTAs per SM
constexpr int BRICK_MAX_MT = 16;        // 256 TMEM columns

template <int MODE>
__global__ void __launch_bounds__(BRICK_NT, 2) brick_tc_kernel(const __grid_constant__ Args a,
                                                                const __grid_constant__ BrickGeo g)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    const uint32_t plane = (uint32_t)g.SROWS * 16u;
    unsigned char *A = smem;                          // [2][SROWS][16 B]
    unsigned char *Wb = smem + 2 * plane;             // [27][2][16][16 B]
    uint64_t *bar = reinterpret_cast<uint64_t *>(Wb + WBYTES);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 1);
    int *okf = reinterpret_cast<int *>(slot + 1);
    const int r = threadIdx.x, warp = r >> 5;
    constexpr uint32_t TCOLS = 256;

    const int per = g.bricks[0] * g.bricks[1] * g.bricks[2];
    const int b = blockIdx.x / per;
    int br = blockIdx.x - b * per;
    const int ox = (br % g.bricks[0]) * g.BX;
    br /= g.bricks[0];
    const int oy = (br % g.bricks[1]) * g.BY;
    const int oz = (br / g.bricks[1]) * g.BZ;

    if (r == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        tc::tmem_alloc(slot, TCOLS);
        tc::tmem_relinquish();
    }
    for (int i = r; i < (int)(WBYTES / 16); i += BRICK_NT)
        reinterpret_cast<uint4 *>(Wb)[i] = __ldg(reinterpret_cast<const uint4 *>(a.w) + i);
    // ---- source region: lanes 2i, 2i+1 copy the two channel halves of a row
    const int64_t si3 = (int64_t)a.Sin * a.Sin * a.Sin;
    const int rrows = g.RX * g.RY * g.RZ;
    for (int t = r; t < 2 * g.SROWS; t += BRICK_NT) {
        const int u = t >> 1, hh = t & 1;
        unsigned char *dst = A + hh * plane + u * 16;
        bool in = false;
        int64_t e = 0;
        if (u < rrows) {
            const int i = u % g.RX, j = (u / g.RX) % g.RY, k = u / (g.RX * g.RY);
            const int sx = ox + i + a.shift, sy = oy + j + a.shift, sz = oz + k + a.shift;
            in = (unsigned)sx < (unsigned)a.Sin && (unsigned)sy < (unsigned)a.Sin && (unsigned)sz < (unsigned)a.Sin;
            if (in) e = (int64_t)b * si3 + sx + (int64_t)a.Sin * (sy + (int64_t)a.Sin * sz);
        }
        cp16(dst, in ? a.src + e * 16 + 8 * hh : a.src, in ? 16u : 0u);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = *slot;

    if (r == 0) {
        const uint32_t a0 = smem_u32(A), b0 = smem_u32(Wb);
        const int sy = g.RX, sz = g.RX * g.RY;
#pragma unroll 1
        for (int t = 0; t < g.MT; ++t) {
#pragma unroll
            for (int q = 0; q < 27; ++q) {
                const int off = q % 3 + sy * ((q / 3) % 3) + sz * (q / 9);
                const uint64_t da = tc::smem_desc(a0 + 16u * (uint32_t)(128 * t + off), plane, 128u);
                const uint64_t db = tc::smem_desc(b0 + 512u * q, 256u, 128u);
                tc::mma_bf16(tbase + 16u * t, da, db, IDESC_K, q > 0 ? 1u : 0u);
            }
        }
        tc::mma_commit(bar);
        *okf = mbar_wait_bounded(bar, 0) ? 1 : 0;
    }
    __syncthreads();
    const int ok = *okf;
    tc::fence_after_sync();
    if (ok) {
        // warp w: TMEM lanes 32 (w % 4) .. + 31 of tiles w / 4, w / 4 + 2, ...
        const uint32_t lanes = (uint32_t)(32 * (warp & 3)) << 16;
        const int64_t so3 = (int64_t)a.Sout * a.Sout * a.Sout;
#pragma unroll 1
        for (int t = warp >> 2; t < g.MT; t += 2) {
            float v[16];
            tc::tmem_ld16(tbase + lanes + 16u * t, v);
            const int m = 128 * t + 32 * (warp & 3) + (r & 31);
            const int z = m / (g.RX * g.RY), rem = m - z * (g.RX * g.RY);
            const int y = rem / g.RX, x = rem - y * g.RX;
            const int X = ox + x, Y = oy + y, Z = oz + z;
            if (x >= g.BX || y >= g.BY || z >= g.BZ || X >= a.Sout || Y >= a.Sout || Z >= a.Sout) continue;
            const int64_t L = (int64_t)b * so3 + X + (int64_t)a.Sout * (Y + (int64_t)a.Sout * Z);
            uint32_t h[8];
            if (MODE == BWD) {
                const uint4 *mk = reinterpret_cast<const uint4 *>(a.act + L * 16);
                const uint4 m0 = mk[0], m1 = mk[1];
                const uint32_t mw[8] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const float lo = __uint_as_float(mw[q] << 16), hi = __uint_as_float(mw[q] & 0xFFFF0000u);
                    h[q] = (uint32_t)bf16_bits(lo > 0.f ? v[2 * q] : 0.f) |
                           ((uint32_t)bf16_bits(hi > 0.f ? v[2 * q + 1] : 0.f) << 16);
                }
            } else {
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    float p = v[2 * q], u = v[2 * q + 1];
                    if (a.relu) {
                        p = fmaxf(p, 0.f);
                        u = fmaxf(u, 0.f);
                    }
                    h[q] = (uint32_t)bf16_bits(p) | ((uint32_t)bf16_bits(u) << 16);
                }
            }
            uint4 *dst = reinterpret_cast<uint4 *>(a.out + L * 16);
            dst[0] = make_uint4(h[0], h[1], h[2], h[3]);
            dst[1] = make_uint4(h[4], h[5], h[6], h[7]);
        }
    } else if (r == 0 && a.err) {
        atomicExch(a.err, kDevErrTimeout);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tbase, TCOLS);
}

// Brick shape for an output cube of side So: whole rows (BX = So, at most
// 64), and the (BY, BZ), BZ <= 4, of least cost while the staged rows fit
// BRICK_MAX_ROWS and the tiles BRICK_MAX_MT; cost = bricks x (tiles + 3),
// a brick's set-up (weights, barrier, TMEM, staging latency) counted as
// three tiles of MMAs.  False if none fits.
static bool brick_geo(int So, BrickGeo &g)
{
    g.BX = So < 64 ? So : 64;
    g.RX = g.BX + 2;
    const int64_t bx = (So + g.BX - 1) / g.BX;
    int64_t best = -1;
    for (int bz = 1; bz <= 4 && bz <= So; ++bz)
        for (int by = 1; by <= So; ++by) {
            const int ry = by + 2, rz = bz + 2;
            const int span = (g.BX - 1) + g.RX * (by - 1) + g.RX * ry * (bz - 1) + 1;
            const int mt = (span + 127) / 128;
            const int offmax = 2 + 2 * g.RX + 2 * g.RX * ry;
            const int srows = ((128 * mt + offmax + 7) / 8) * 8;
            if (mt > BRICK_MAX_MT || srows > BRICK_MAX_ROWS || srows < g.RX * ry * rz) continue;
            const int64_t cost = bx * ((So + by - 1) / by) * ((So + bz - 1) / bz) * (mt + 3);
            if (best < 0 || cost < best) {
                best = cost;
                g.BY = by;
                g.BZ = bz;
                g.RY = ry;
                g.RZ = rz;
                g.MT = mt;
                g.SROWS = srows;
            }
        }
    if (best < 0) return false;
    g.bricks[0] = (int)bx;
    g.bricks[1] = (So + g.BY - 1) / g.BY;
    g.bricks[2] = (So + g.BZ - 1) / g.BZ;
    return true;
}

// ---------------------------------------------------- CUDA-core layers
// layer 1 forward: x [B][2][S^3] FP32 -> h1 [B][(S-2)^3][16] BF16, ReLU
__global__ void __launch_bounds__(128) l1_fwd_cl(const float *__restrict__ x, const float *__restrict__ W1,
                                                  uint16_t *__restrict__ h1, int B, int S)
{
    __shared__ __align__(16) float sw[27 * 2 * 16];
    for (int i = threadIdx.x; i < 27 * 32; i += blockDim.x) sw[i] = W1[i];
    __syncthreads();
    const int So = S - 2;
    const int64_t per = (int64_t)So * So * So, s3 = (int64_t)S * S * S, total = per * B;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const CubeIdx ci = cube_idx((uint32_t)q, (uint32_t)So, (uint32_t)per);
        const int b = ci.b, xx = ci.x, yy = ci.y, zz = ci.z;
        const float *x0 = x + (int64_t)b * 2 * s3, *x1 = x0 + s3;
        float acc[16];
#pragma unroll
        for (int o = 0; o < 16; ++o) acc[o] = 0.f;
#pragma unroll 1
        for (int t = 0; t < 27; ++t) {
            const int64_t e = (xx + t % 3) + (int64_t)S * ((yy + (t / 3) % 3) + (int64_t)S * (zz + t / 9));
            const float v0 = __ldg(x0 + e), v1 = __ldg(x1 + e);
            const float *w = sw + t * 32;
#pragma unroll
            for (int o = 0; o < 16; ++o) acc[o] = fmaf(v0, w[o], fmaf(v1, w[16 + o], acc[o]));
        }
        uint32_t h[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            h[j] = (uint32_t)bf16_bits(fmaxf(acc[2 * j], 0.f)) | ((uint32_t)bf16_bits(fmaxf(acc[2 * j + 1], 0.f)) << 16);
        uint4 *dst = reinterpret_cast<uint4 *>(h1 + q * 16);
        dst[0] = make_uint4(h[0], h[1], h[2], h[3]);
        dst[1] = make_uint4(h[4], h[5], h[6], h[7]);
    }
}

__device__ __forceinline__ void unpack16(const uint16_t *p, float (&v)[16])
{
    const uint4 *s = reinterpret_cast<const uint4 *>(p);
    const uint4 a = __ldg(s), b = __ldg(s + 1);
    const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        v[2 * j] = __uint_as_float(w[j] << 16);
        v[2 * j + 1] = __uint_as_float(w[j] & 0xFFFF0000u);
    }
}

// layer 3 forward: h2 [B][S^3][16] BF16 -> y [B][(S-2)^3] FP32
__global__ void __launch_bounds__(128) l3_fwd_cl(const uint16_t *__restrict__ h2, const float *__restrict__ W3,
                                                  float *__restrict__ y, int B, int S)
{
    __shared__ __align__(16) float sw[27 * 16];
    for (int i = threadIdx.x; i < 27 * 16; i += blockDim.x) sw[i] = W3[i];
    __syncthreads();
    const int So = S - 2;
    const int64_t per = (int64_t)So * So * So, s3 = (int64_t)S * S * S, total = per * B;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const CubeIdx ci = cube_idx((uint32_t)q, (uint32_t)So, (uint32_t)per);
        const int b = ci.b, xx = ci.x, yy = ci.y, zz = ci.z;
        float acc = 0.f;
#pragma unroll 1
        for (int t = 0; t < 27; ++t) {
            const int64_t e = (xx + t % 3) + (int64_t)S * ((yy + (t / 3) % 3) + (int64_t)S * (zz + t / 9));
            float v[16];
            unpack16(h2 + ((int64_t)b * s3 + e) * 16, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) acc = fmaf(v[i], sw[t * 16 + i], acc);
        }
        y[q] = acc;
    }
}

// layer 3 backward-data: gh2[c][ci] = (h2[c][ci] > 0) sum_e gc[c - 2 + e] W3[26 - e][ci]
// for c in S^3 (gc on (S-2)^3, zero outside)
__global__ void __launch_bounds__(128) l3_bwd_data_cl(const float *__restrict__ gc, const float *__restrict__ W3,
                                                       const uint16_t *__restrict__ h2, uint16_t *__restrict__ gh2,
                                                       int B, int S)
{
    __shared__ __align__(16) float sw[27 * 16];
    for (int i = threadIdx.x; i < 27 * 16; i += blockDim.x) sw[i] = W3[i];
    __syncthreads();
    const int So = S - 2;
    const int64_t per = (int64_t)S * S * S, pero = (int64_t)So * So * So, total = per * B;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const CubeIdx ci = cube_idx((uint32_t)q, (uint32_t)S, (uint32_t)per);
        const int b = ci.b, xx = ci.x, yy = ci.y, zz = ci.z;
        float acc[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[i] = 0.f;
#pragma unroll 1
        for (int e = 0; e < 27; ++e) {
            const int ox = xx - 2 + e % 3, oy = yy - 2 + (e / 3) % 3, oz = zz - 2 + e / 9;
            if ((unsigned)ox >= (unsigned)So || (unsigned)oy >= (unsigned)So || (unsigned)oz >= (unsigned)So) continue;
            const float g = __ldg(gc + (int64_t)b * pero + ox + (int64_t)So * (oy + (int64_t)So * oz));
            const float *w = sw + (26 - e) * 16;
#pragma unroll
            for (int i = 0; i < 16; ++i) acc[i] = fmaf(g, w[i], acc[i]);
        }
        float m[16];
        unpack16(h2 + q * 16, m);
        uint32_t h[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            h[j] = (uint32_t)bf16_bits(m[2 * j] > 0.f ? acc[2 * j] : 0.f) |
                   ((uint32_t)bf16_bits(m[2 * j + 1] > 0.f ? acc[2 * j + 1] : 0.f) << 16);
        uint4 *dst = reinterpret_cast<uint4 *>(gh2 + q * 16);
        dst[0] = make_uint4(h[0], h[1], h[2], h[3]);
        dst[1] = make_uint4(h[4], h[5], h[6], h[7]);
    }
}

// warp sum of v[0..N) into lane 0
template <int N> __device__ __forceinline__ void warp_sum(float (&v)[N])
{
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
}

// The weight gradients of the first and last layers: blocks of 27 warps,
// warp w = tap w.  A block walks whole planes (patch b, z) of the output
// cells; the lanes of all 27 warps take the same cells of the plane (index
// y So + x, advanced without divisions), so the per-cell operand (gc or
// gh1) is read from DRAM once and the 27 taps' shifted reads hit L1.
// Per-warp sums, then atomics.
constexpr int WG_THREADS = 27 * 32;

// layer 3: gW3[t][ci] += sum_q h2[q + d(t)][ci] gc[q], q in (S-2)^3, h2 side S
__global__ void __launch_bounds__(WG_THREADS) l3_wgrad_cl(const uint16_t *__restrict__ h2,
                                                           const float *__restrict__ gc, float *__restrict__ gW3,
                                                           int B, int S)
{
    const int t = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int dx = t % 3, dy = (t / 3) % 3, dz = t / 9;
    const int So = S - 2, plane = So * So;
    const int64_t s3 = (int64_t)S * S * S;
    float acc[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) acc[i] = 0.f;
    for (int pz = blockIdx.x; pz < B * So; pz += gridDim.x) {
        const int b = pz / So, zz = pz - b * So;
        const float *gp = gc + (int64_t)pz * plane;
        const uint16_t *hp = h2 + ((int64_t)b * s3 + dx + (int64_t)S * (dy + (int64_t)S * (zz + dz))) * 16;
        int xx = lane, yy = 0;
        for (int idx = lane; idx < plane; idx += 32) {
            while (xx >= So) {
                xx -= So;
                ++yy;
            }
            const float g = __ldg(gp + idx);
            float v[16];
            unpack16(hp + (xx + (int64_t)S * yy) * 16, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) acc[i] = fmaf(v[i], g, acc[i]);
            xx += 32;
        }
    }
    warp_sum(acc);
    if (lane == 0)
#pragma unroll
        for (int i = 0; i < 16; ++i) atomicAdd(gW3 + t * 16 + i, acc[i]);
}

// layer 1: gW1[t][i][o] += sum_q x[i][q + d(t)] gh1[q][o], q in (S-2)^3, x side S
__global__ void __launch_bounds__(WG_THREADS) l1_wgrad_cl(const float *__restrict__ x,
                                                           const uint16_t *__restrict__ gh1, float *__restrict__ gW1,
                                                           int B, int S)
{
    const int t = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int dx = t % 3, dy = (t / 3) % 3, dz = t / 9;
    const int So = S - 2, plane = So * So;
    const int64_t s3 = (int64_t)S * S * S;
    float acc[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) acc[i] = 0.f;
    for (int pz = blockIdx.x; pz < B * So; pz += gridDim.x) {
        const int b = pz / So, zz = pz - b * So;
        const uint16_t *gp = gh1 + (int64_t)pz * plane * 16;
        const float *xp = x + (int64_t)b * 2 * s3 + dx + (int64_t)S * (dy + (int64_t)S * (zz + dz));
        int xx = lane, yy = 0;
        for (int idx = lane; idx < plane; idx += 32) {
            while (xx >= So) {
                xx -= So;
                ++yy;
            }
            const int64_t e = xx + (int64_t)S * yy;
            const float v0 = __ldg(xp + e), v1 = __ldg(xp + e + s3);
            float g[16];
            unpack16(gp + (int64_t)idx * 16, g);
#pragma unroll
            for (int o = 0; o < 16; ++o) {
                acc[o] = fmaf(v0, g[o], acc[o]);
                acc[16 + o] = fmaf(v1, g[o], acc[16 + o]);
            }
            xx += 32;
        }
    }
    warp_sum(acc);
    if (lane == 0)
#pragma unroll
        for (int i = 0; i < 32; ++i) atomicAdd(gW1 + t * 32 + i, acc[i]);
}

static unsigned grid_of(int64_t n, int threads, int64_t cap)
{
    int64_t b = (n + threads - 1) / threads;
    if (b > cap) b = cap;
    return (unsigned)(b < 1 ? 1 : b);
}

static DeviceOnce wgrad_once, brick_once[2];

// weight gradient: persistent CTAs, two per SM
static cn_status launch_wgrad(Args &a, cudaStream_t st)
{
    cn_status s = smem_opt_in(wgrad_once, wgrad_tc_kernel, SMEM);
    if (s != CN_OK) return s;
    int dev = 0, sms = 148;
    CN_CUDA_TRY(cudaGetDevice(&dev));
    CN_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    a.chunks = (a.total + ROWS - 1) / ROWS;
    const int64_t grid = a.chunks < 2LL * sms ? a.chunks : 2LL * sms;
    wgrad_tc_kernel<<<(unsigned)grid, NT, SMEM, st>>>(a);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

// forward / backward-data: one CTA per brick
template <int MODE>
static cn_status launch_conv(Args &a, int B, cudaStream_t st)
{
    BrickGeo g;
    if (!brick_geo(a.Sout, g)) return fail(CN_ERR_INVALID_ARGUMENT, "learned smoother training: empty patch");
    const size_t smem = 2 * (size_t)g.SROWS * 16 + WBYTES + 16;
    // one opt-in per device, at the largest brick any patch size can take
    constexpr size_t smem_max = 2 * (size_t)BRICK_MAX_ROWS * 16 + WBYTES + 16;
    cn_status s = smem_opt_in(brick_once[MODE], brick_tc_kernel<MODE>, smem_max);
    if (s != CN_OK) return s;
    const int64_t ctas = (int64_t)B * g.bricks[0] * g.bricks[1] * g.bricks[2];
    brick_tc_kernel<MODE><<<(unsigned)ctas, BRICK_NT, smem, st>>>(a, g);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

} // namespace nntr

namespace nntc {

cn_status train_forward_tc(const TrainBufs &T, const float *x, const float *W, int B, int P, cudaStream_t st)
{
    using namespace nntr;
    const int S = P + 8, S1 = S - 2, S2 = S - 4, S3 = S - 6;
    const float *W1 = W, *W2 = W + 27 * 2 * 16, *W3 = W + 27 * 2 * 16 + 27 * 16 * 16;
    if ((int64_t)B * S * S * S >= (int64_t)1 << 31)
        return fail(CN_ERR_UNSUPPORTED, "learned smoother training: batch too large for 32-bit cell indices");
    cn_status s;
    // packed B tiles of the hidden layer: forward, backward-data
    if ((s = pack_weights(W2, 16, 16, T.wfwd, st)) != CN_OK) return s;
    pack_bwd_kernel<<<27, 256, 0, st>>>(W2, T.wbwd);
    l1_fwd_cl<<<grid_of((int64_t)B * S1 * S1 * S1, 128, 148 * 64), 128, 0, st>>>(x, W1, T.h1, B, S);
    CN_CUDA_TRY(cudaGetLastError());
    Args a = {};
    a.src = T.h1;
    a.w = T.wfwd;
    a.out = T.h2;
    a.Sin = S1;
    a.Sout = S2;
    a.shift = 0;
    a.relu = 1;
    a.total = (int64_t)B * S2 * S2 * S2;
    a.err = T.err;
    if ((s = launch_conv<FWD>(a, B, st)) != CN_OK) return s;
    l3_fwd_cl<<<grid_of((int64_t)B * S3 * S3 * S3, 128, 148 * 64), 128, 0, st>>>(T.h2, W3, T.y, B, S2);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

cn_status train_backward_tc(const TrainBufs &T, const float *x, const float *W, float *gW, int B, int P,
                            cudaStream_t st)
{
    using namespace nntr;
    const int S = P + 8, S1 = S - 2, S2 = S - 4, S3 = S - 6;
    const float *W3 = W + 27 * 2 * 16 + 27 * 16 * 16;
    float *gW1 = gW, *gW2 = gW + 27 * 2 * 16, *gW3 = gW + 27 * 2 * 16 + 27 * 16 * 16;
    cn_status s;
    CN_CUDA_TRY(cudaMemsetAsync(gW, 0, sizeof(float) * (27 * 2 * 16 + 27 * 16 * 16 + 27 * 16), st));
    int dev = 0, sms = 148;
    CN_CUDA_TRY(cudaGetDevice(&dev));
    CN_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    l3_wgrad_cl<<<grid_of((int64_t)B * S3, 1, sms), WG_THREADS, 0, st>>>(T.h2, T.gc, gW3, B, S2);
    l3_bwd_data_cl<<<grid_of((int64_t)B * S2 * S2 * S2, 128, 148 * 64), 128, 0, st>>>(T.gc, W3, T.h2, T.gh2, B, S2);
    CN_CUDA_TRY(cudaGetLastError());
    Args w = {};
    w.src = T.h1;
    w.gout = T.gh2;
    w.gw = gW2;
    w.Sin = S1;
    w.Sout = S2;
    w.shift = 0;
    w.total = (int64_t)B * S2 * S2 * S2;
    w.err = T.err;
    if ((s = launch_wgrad(w, st)) != CN_OK) return s;
    Args d = {};
    d.src = T.gh2;
    d.act = T.h1;
    d.w = T.wbwd;
    d.out = T.gh1;
    d.Sin = S2;
    d.Sout = S1;
    d.shift = -2;
    d.total = (int64_t)B * S1 * S1 * S1;
    d.err = T.err;
    if ((s = launch_conv<BWD>(d, B, st)) != CN_OK) return s;
    l1_wgrad_cl<<<grid_of((int64_t)B * S1, 1, sms), WG_THREADS, 0, st>>>(x, T.gh1, gW1, B, S);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

} // namespace nntc
} // namespace cn
