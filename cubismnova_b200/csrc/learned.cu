// learned.cu -- a learned 3-D convolutional smoother for the multigrid solver.
//
// Network (no biases, so it is positively homogeneous in the residual):
//   x  = (x0, x1),  x0 = (L p - f) / D = -r / D  (the Jacobi correction of
//        L p = f, whose diagonal is -D),  x1 = x0 * ln k
//   h1 = relu(conv3(W1, x))   2 -> 16 channels, 3x3x3 taps
//   h2 = relu(conv3(W2, h1)) 16 -> 16
//   y  = conv3(W3, h2)       16 -> 1
//   smoothing step:  p <- p + omega * x0 + y        (Jacobi plus a learned term)
// Weights are stored [tap][cin][cout], tap = dx+1 + 3*(dy+1) + 9*(dz+1).
//
// Training (all on the device): samples are block-sized patches of
// residuals r taken from the plain V-cycle (before pre-smoothing and after the
// coarse-grid correction) with the coefficients k; the loss is the residual
// left after one smoothing step, normalised per sample,
//   loss = (1/B) sum_b  || r_b - A c_b ||^2 / || r_b ||^2 ,  c = omega x0 + y,
// evaluated on the patch interior (A = the variable-coefficient operator).
// Patches carry a 4-cell halo: three valid convolutions and A each shrink the
// region by one cell.  Backward: the adjoint of A (gather form), transposed
// convolutions masked by the ReLU, weight gradients reduced per tap, Adam.
// The network's forward and backward run either on the tensor cores with
// BF16 activations (learned_train_tc.cu, the default) or in FP32 on the CUDA
// cores (the patch kernels below; cn_nn_set_training); the loss, its
// adjoint and Adam are shared.
//
// Inference on the grid runs layer by layer on grids of 16 channels, each
// convolution reading its input through the lab of a (-1,2) tensorial stencil
// (periodic block neighbours and BCs), so the network sees exactly the
// neighbourhood a FieldLab would give it.
#include "cn_internal.h"
#include "learned_tc.h"
#include "mg_tile.cuh"
#include "mg_internal.h"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

namespace cn {
namespace nn {

constexpr int CI = 2, CH = 16;

__device__ __forceinline__ int tap_of(int dx, int dy, int dz) { return (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1); }

// ------------------------------------------------------------------ patches
// Valid 3x3x3 convolution of a batch of cubes: in [B][Cin][S^3] -> out
// [B][Cout][(S-2)^3], optional ReLU.  One thread per output cell.
template <int Cin, int Cout, bool RELU>
__global__ void __launch_bounds__(128) conv_fwd_patch(const float *__restrict__ in, const float *__restrict__ W,
                                                      float *__restrict__ out, int B, int S)
{
    extern __shared__ float sw[];
    for (int i = threadIdx.x; i < 27 * Cin * Cout; i += blockDim.x) sw[i] = W[i];
    __syncthreads();
    const int So = S - 2;
    const int64_t per = (int64_t)So * So * So;
    const int64_t total = per * B;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(t / per);
        int64_t c = t - b * per;
        const int x = (int)(c % So), y = (int)((c / So) % So), z = (int)(c / ((int64_t)So * So));
        float acc[Cout];
#pragma unroll
        for (int o = 0; o < Cout; ++o) acc[o] = 0.f;
        const float *ib = in + (int64_t)b * Cin * S * S * S;
        for (int dz = 0; dz < 3; ++dz)
            for (int dy = 0; dy < 3; ++dy)
                for (int dx = 0; dx < 3; ++dx) {
                    const int tap = dx + 3 * dy + 9 * dz;
                    const int64_t off = (x + dx) + (int64_t)S * ((y + dy) + (int64_t)S * (z + dz));
#pragma unroll
                    for (int i = 0; i < Cin; ++i) {
                        const float v = ib[(int64_t)i * S * S * S + off];
                        const float *w = sw + (tap * Cin + i) * Cout;
#pragma unroll
                        for (int o = 0; o < Cout; ++o) acc[o] = fmaf(v, w[o], acc[o]);
                    }
                }
        float *ob = out + (int64_t)b * Cout * per;
#pragma unroll
        for (int o = 0; o < Cout; ++o) ob[(int64_t)o * per + c] = RELU ? fmaxf(acc[o], 0.f) : acc[o];
    }
}

// Transposed convolution: gin [B][Cin][S^3] = sum over taps of W^T gout
// [B][Cout][(S-2)^3], then multiplied by (act > 0) if act (the ReLU output
// that fed this convolution) is given.
template <int Cin, int Cout>
__global__ void __launch_bounds__(128) conv_bwd_data_patch(const float *__restrict__ gout, const float *__restrict__ W,
                                                           const float *__restrict__ act, float *__restrict__ gin,
                                                           int B, int S)
{
    extern __shared__ float sw[];
    for (int i = threadIdx.x; i < 27 * Cin * Cout; i += blockDim.x) sw[i] = W[i];
    __syncthreads();
    const int So = S - 2;
    const int64_t per = (int64_t)S * S * S, pero = (int64_t)So * So * So;
    const int64_t total = per * B;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(t / per);
        int64_t c = t - b * per;
        const int x = (int)(c % S), y = (int)((c / S) % S), z = (int)(c / ((int64_t)S * S));
        float acc[Cin];
#pragma unroll
        for (int i = 0; i < Cin; ++i) acc[i] = 0.f;
        const float *gb = gout + (int64_t)b * Cout * pero;
        for (int dz = 0; dz < 3; ++dz) {
            const int oz = z - dz;
            if (oz < 0 || oz >= So) continue;
            for (int dy = 0; dy < 3; ++dy) {
                const int oy = y - dy;
                if (oy < 0 || oy >= So) continue;
                for (int dx = 0; dx < 3; ++dx) {
                    const int ox = x - dx;
                    if (ox < 0 || ox >= So) continue;
                    const int tap = dx + 3 * dy + 9 * dz;
                    const int64_t off = ox + (int64_t)So * (oy + (int64_t)So * oz);
                    for (int o = 0; o < Cout; ++o) {
                        const float g = gb[(int64_t)o * pero + off];
#pragma unroll
                        for (int i = 0; i < Cin; ++i) acc[i] = fmaf(g, sw[(tap * Cin + i) * Cout + o], acc[i]);
                    }
                }
            }
        }
        float *ob = gin + (int64_t)b * Cin * per;
#pragma unroll
        for (int i = 0; i < Cin; ++i) {
            float v = acc[i];
            if (act && !(act[(int64_t)b * Cin * per + (int64_t)i * per + c] > 0.f)) v = 0.f;
            ob[(int64_t)i * per + c] = v;
        }
    }
}

// Weight gradient: gW[tap][i][o] += sum_{b,q} in[b][i][q + tap] * gout[b][o][q].
// Grid: blockIdx.y = tap, blockIdx.x = chunk of output positions; threads own
// (i, o) pairs and reduce over a staged chunk of positions.
template <int Cin, int Cout>
__global__ void __launch_bounds__(256) conv_bwd_weight_patch(const float *__restrict__ in, const float *__restrict__ gout,
                                                             float *__restrict__ gW, int B, int S)
{
    constexpr int CHUNK = 64;
    __shared__ float si[CHUNK][Cin];
    __shared__ float sg[CHUNK][Cout];
    const int tap = blockIdx.y;
    const int dx = tap % 3, dy = (tap / 3) % 3, dz = tap / 9;
    const int So = S - 2;
    const int64_t pero = (int64_t)So * So * So, per = (int64_t)S * S * S;
    const int64_t total = pero * B;
    const int pair = threadIdx.x;
    const int pi = pair / Cout, po = pair % Cout;
    float acc = 0.f;
    for (int64_t base = (int64_t)blockIdx.x * CHUNK; base < total; base += (int64_t)gridDim.x * CHUNK) {
        __syncthreads();
        for (int e = threadIdx.x; e < CHUNK * (Cin + Cout); e += blockDim.x) {
            const int q = e % CHUNK, ch = e / CHUNK;
            const int64_t t = base + q;
            float v = 0.f;
            if (t < total) {
                const int b = (int)(t / pero);
                const int64_t c = t - b * pero;
                const int x = (int)(c % So), y = (int)((c / So) % So), z = (int)(c / ((int64_t)So * So));
                if (ch < Cin) {
                    v = in[(int64_t)b * Cin * per + (int64_t)ch * per + (x + dx) + (int64_t)S * ((y + dy) + (int64_t)S * (z + dz))];
                } else {
                    v = gout[(int64_t)b * Cout * pero + (int64_t)(ch - Cin) * pero + c];
                }
            }
            if (ch < Cin) si[q][ch] = v;
            else sg[q][ch - Cin] = v;
        }
        __syncthreads();
        if (pair < Cin * Cout) {
#pragma unroll 8
            for (int q = 0; q < CHUNK; ++q) acc = fmaf(si[q][pi], sg[q][po], acc);
        }
    }
    if (pair < Cin * Cout) atomicAdd(gW + (tap * Cin + pi) * Cout + po, acc);
}

__device__ __forceinline__ float harmf(float a, float b)
{
    const float t = a * b;
    return (t + t) / (a + b);
}

// c = omega*x0 + y on the region R1 (P+2)^3; Ac on the interior P^3 with k on
// R1; per-sample sums of r^2 and (r - Ac)^2; g = d loss / d(Ac) written for
// the adjoint.  x is [B][2][(P+8)^3], y [B][1][(P+2)^3], k [B][(P+2)^3],
// r [B][P^3].
__global__ void __launch_bounds__(256) loss_fwd(const float *x, const float *y, float omega, int B, int P,
                                                float *c_out)
{
    const int S = P + 8, R = P + 2;
    const int64_t perR = (int64_t)R * R * R, perS = (int64_t)S * S * S;
    // c on R1
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < perR * B; t += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(t / perR);
        const int64_t cc = t - b * perR;
        const int X = (int)(cc % R), Y = (int)((cc / R) % R), Z = (int)(cc / (R * R));
        const float x0 = x[(int64_t)b * 2 * perS + (X + 3) + (int64_t)S * ((Y + 3) + (int64_t)S * (Z + 3))];
        c_out[t] = omega * x0 + y[t];
    }
}

// Grid (chunks, B): blockIdx.y is the sample; per-sample sums reduced in the
// block (warp shuffles, then one warp) before one atomic pair per block.
__global__ void __launch_bounds__(256) loss_res(const float *c, const float *k, const float *r, float ih2, int B, int P,
                                                float *res_out, double *sums)
{
    const int R = P + 2;
    const int64_t perR = (int64_t)R * R * R, perP = (int64_t)P * P * P;
    const int b = blockIdx.y;
    const float *cb = c + b * perR, *kb = k + b * perR;
    double srr = 0.0, see = 0.0;
    for (int64_t cc = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; cc < perP; cc += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(cc % P) + 1, y = (int)((cc / P) % P) + 1, z = (int)(cc / (P * P)) + 1;
        const int64_t i = x + (int64_t)R * (y + (int64_t)R * z);
        const float pc = cb[i], kc = kb[i];
        const int64_t st[3] = {1, R, (int64_t)R * R};
        float f[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const float kp = harmf(kc, kb[i + st[d]]), km = harmf(kb[i - st[d]], kc);
            f[d] = kp * (cb[i + st[d]] - pc) - km * (pc - cb[i - st[d]]);
        }
        const float Ac = ih2 * ((f[0] + f[1]) + f[2]);
        const int64_t t = b * perP + cc;
        const float rv = r[t];
        const float e = rv - Ac;
        res_out[t] = e;
        srr += (double)rv * rv;
        see += (double)e * e;
    }
    __shared__ double part[2][8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        srr += __shfl_xor_sync(0xffffffffu, srr, o);
        see += __shfl_xor_sync(0xffffffffu, see, o);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        part[0][w] = srr;
        part[1][w] = see;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, e2 = 0.0;
        for (int j = 0; j < (int)(blockDim.x >> 5); ++j) {
            a += part[0][j];
            e2 += part[1][j];
        }
        atomicAdd(sums + 2 * b, a);
        atomicAdd(sums + 2 * b + 1, e2);
    }
}

// gc on R1 = adjoint of (c -> Ac on the interior) applied to g = -2 w_b (r - Ac) / B
__global__ void __launch_bounds__(256) loss_adjoint(const float *res, const float *k, const double *sums, float ih2,
                                                    int B, int P, float *gc)
{
    const int R = P + 2;
    const int64_t perR = (int64_t)R * R * R, perP = (int64_t)P * P * P;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < perR * B; t += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(t / perR);
        const int64_t cc = t - b * perR;
        const int X = (int)(cc % R), Y = (int)((cc / R) % R), Z = (int)(cc / (R * R));
        const double rr = sums[2 * b];
        const float w = rr > 0 ? (float)(-2.0 / (rr * B)) : 0.f;
        const float *kb = k + b * perR;
        const float *eb = res + b * perP;
        auto interior = [&](int a, int bb, int c2) { return a >= 1 && a <= P && bb >= 1 && bb <= P && c2 >= 1 && c2 <= P; };
        auto gidx = [&](int a, int bb, int c2) { return (int64_t)(a - 1) + P * ((int64_t)(bb - 1) + (int64_t)P * (c2 - 1)); };
        const int64_t i = X + (int64_t)R * (Y + (int64_t)R * Z);
        const float kc = kb[i];
        float acc = 0.f;
        // own row: d(Ac)_j / dc_j = -ih2 * sum kf
        if (interior(X, Y, Z)) {
            float s = 0.f;
            const int64_t st[3] = {1, R, (int64_t)R * R};
            for (int d = 0; d < 3; ++d) s += harmf(kc, kb[i + st[d]]) + harmf(kb[i - st[d]], kc);
            acc += -ih2 * s * eb[gidx(X, Y, Z)];
        }
        const int dxs[6] = {1, -1, 0, 0, 0, 0}, dys[6] = {0, 0, 1, -1, 0, 0}, dzs[6] = {0, 0, 0, 0, 1, -1};
        for (int m = 0; m < 6; ++m) {
            const int a = X + dxs[m], bb = Y + dys[m], c2 = Z + dzs[m];
            if (!interior(a, bb, c2)) continue;
            const float kn = kb[a + (int64_t)R * (bb + (int64_t)R * c2)];
            acc += ih2 * harmf(kn, kc) * eb[gidx(a, bb, c2)];
        }
        gc[t] = w * acc;
    }
}

__global__ void adam_kernel(float *p, const float *g, float *m, float *v, int n, float lr, float b1, float b2,
                            float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// ------------------------------------------------------------ grid layers
// The network applied to grids in block layout: neighbours through the lab of
// a (-1,2) tensorial stencil.
template <typename T>
__device__ __forceinline__ T gfetch(const T *comp, const LabGeom &L, const BcView &bc, int block, int x, int y, int z)
{
    return lab_fetch<T>(comp, L, bc, block, x, y, z);
}

struct GridIO {
    const float *in;   // Cin components, cstride apart
    int64_t in_cs;
    BcView in_bc[CH];
    float *out;
    int64_t out_cs;
    LabGeom L;         // tensorial (-1,2)
    int nblocks;
};

template <int Cin, int Cout, bool RELU>
__global__ void __launch_bounds__(128) conv_grid(const __grid_constant__ GridIO g, const float *__restrict__ W)
{
    extern __shared__ float sw[];
    for (int i = threadIdx.x; i < 27 * Cin * Cout; i += blockDim.x) sw[i] = W[i];
    __syncthreads();
    const LabGeom &L = g.L;
    const int64_t cells = (int64_t)L.n[0] * L.n[1] * L.n[2];
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < cells * g.nblocks;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int block = (int)(t / cells);
        const int64_t c = t - block * cells;
        const int x = (int)(c % L.n[0]), y = (int)((c / L.n[0]) % L.n[1]), z = (int)(c / ((int64_t)L.n[0] * L.n[1]));
        const bool inner = x > 0 && y > 0 && z > 0 && x < L.n[0] - 1 && y < L.n[1] - 1 && z < L.n[2] - 1;
        float acc[Cout];
#pragma unroll
        for (int o = 0; o < Cout; ++o) acc[o] = 0.f;
        const int64_t base = (int64_t)block * L.bstride;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int tap = tap_of(dx, dy, dz);
                    const int64_t off = base + (x + dx) + (int64_t)L.n[0] * ((y + dy) + (int64_t)L.n[1] * (z + dz));
#pragma unroll
                    for (int i = 0; i < Cin; ++i) {
                        const float *ci = g.in + (int64_t)i * g.in_cs;
                        const float v = inner ? __ldg(ci + off) : gfetch<float>(ci, L, g.in_bc[i], block, x + dx, y + dy, z + dz);
                        const float *w = sw + (tap * Cin + i) * Cout;
#pragma unroll
                        for (int o = 0; o < Cout; ++o) acc[o] = fmaf(v, w[o], acc[o]);
                    }
                }
#pragma unroll
        for (int o = 0; o < Cout; ++o)
            g.out[(int64_t)o * g.out_cs + base + c] = RELU ? fmaxf(acc[o], 0.f) : acc[o];
    }
}

} // namespace nn
} // namespace cn

// ----------------------------------------------------------- grid features
namespace cn {
namespace nn {

// x0 = (L p - f) / D = -r / D (the Jacobi correction; L has diagonal -D),
// x1 = x0 ln k, with r = f - L p (p == NULL: p = 0), and r itself; with
// `packed`, also the BF16 channels-last input of the tensor-core layers,
// (x0, x1, 0, ..., 0) per cell.  One CTA per tile of a block: p and k with a
// one-cell halo staged in shared memory (mg_tile.cuh).
struct FeatArgs {
    LabGeom L;
    BcView pbc, kbc;
    const float *p, *k, *f;
    const float *coef; // level coefficients of the multigrid, 8 per cell
    float ih2;
    float *x0, *x1, *rout;
    uint16_t *packed;
};

__global__ void __launch_bounds__(mg::kTileThreads, mg::kTileMinCtas) features_tile(const __grid_constant__ FeatArgs A,
                                                                  const __grid_constant__ mg::Tile T)
{
    __shared__ __align__(16) float sp[mg::kRegionMax];
    __shared__ int snb[27];
    const LabGeom &L = A.L;
    mg::TilePos q = mg::tile_pos(T);
    mg::region_layout<float>(q, L);
    mg::neighbour_blocks(L.nb, q.block, snb);
    __syncthreads();
    if (A.p)
        mg::stage_region<float>(A.p, L, A.pbc, q, false, snb, sp);
    else
        for (int u = threadIdx.x; u < q.rs * q.ey * q.ez; u += mg::kTileThreads) sp[u] = 0.f;
    mg::cp_async_wait_all();
    __syncthreads();
    const int cells = T.t[0] * T.t[1] * T.t[2];
    const int64_t bcells = (int64_t)L.n[0] * L.n[1] * L.n[2];
    const int st[3] = {1, q.rs, q.rs * q.ey};
    for (int c = threadIdx.x; c < cells; c += mg::kTileThreads) {
        int x, y, z;
        mg::tile_cell(T, c, x, y, z);
        const int64_t lc = (q.x0 + x) + (int64_t)L.n[0] * ((q.y0 + y) + (int64_t)L.n[1] * (q.z0 + z));
        const int64_t o = (int64_t)q.block * L.bstride + lc;
        float Lp, D, pc;
        mg::op7_coef<float, float>(sp, mg::ridx(q, x, y, z), st, A.coef + ((int64_t)q.block * bcells + lc) * mg::kCoefPerCell,
                                   A.ih2, Lp, D, pc);
        const float fc = __ldg(A.f + o);
        const float r = fc - Lp;
        const float a = (Lp - fc) / D;
        const float b = a * logf(__ldg(A.k + o));
        A.x0[o] = a;
        A.x1[o] = b;
        if (A.rout) A.rout[o] = r;
        if (A.packed) {
            const uint32_t w0 = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(a)) |
                                ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(b)) << 16);
            uint4 *dst = reinterpret_cast<uint4 *>(A.packed + ((int64_t)q.block * bcells + lc) * 16);
            dst[0] = make_uint4(w0, 0u, 0u, 0u);
            dst[1] = make_uint4(0u, 0u, 0u, 0u);
        }
    }
}

// p += omega * x0 + y
__global__ void __launch_bounds__(256) smooth_update(float *p, const float *x0, const float *y, float omega, int64_t n,
                                                     int zero_guess)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = (zero_guess ? 0.f : p[i]) + (omega * x0[i] + y[i]);
}

// Patch extraction around block b: out[c][X][Y][Z] for X,Y,Z in [-h, n+h).
__global__ void __launch_bounds__(256) extract_patch(const float *comp, const __grid_constant__ LabGeom L,
                                                     const __grid_constant__ BcView bc, const int *blocks, int np,
                                                     int halo, float *out, int64_t out_stride)
{
    const int E = L.n[0] + 2 * halo;
    const int64_t per = (int64_t)E * E * E;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < per * np; t += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(t / per);
        const int64_t c = t - j * per;
        const int X = (int)(c % E) - halo, Y = (int)((c / E) % E) - halo, Z = (int)(c / ((int64_t)E * E)) - halo;
        out[(int64_t)j * out_stride + c] = gfetch<float>(comp, L, bc, blocks[j], X, Y, Z);
    }
}

__global__ void gather_batch(const float *src, int64_t per, const int *idx, int B, float *dst)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < per * B; t += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(t / per);
        dst[t] = src[(int64_t)idx[b] * per + (t - (int64_t)b * per)];
    }
}

} // namespace nn
} // namespace cn

using namespace cn;
using namespace cn::nn;

struct cn_nn {
    float *w = nullptr; // W1 | W2 | W3 (FP32 master)
    float *m = nullptr, *v = nullptr;
    float *g = nullptr;
    int step = 0;
    double omega = 0.8;
    // work buffers for a batch
    int wB = 0, wP = 0;
    float *h1 = nullptr, *h2 = nullptr, *y = nullptr, *c = nullptr, *res = nullptr, *gc = nullptr, *gh2 = nullptr,
          *gh1 = nullptr;
    double *sums = nullptr;
    // grid inference: 1 = BF16 tensor cores (tcgen05) where the block shape
    // allows, 0 = FP32 CUDA cores; packed BF16 weights of the three layers
    int inference = 1;
    uint16_t *wpack = nullptr;
    // training: 1 = hidden layer on the tensor cores with BF16 channels-last
    // activations (learned_train_tc.cu), 0 = FP32 CUDA cores throughout
    int training = 1;
    uint16_t *bh1 = nullptr, *bh2 = nullptr, *bgh1 = nullptr, *bgh2 = nullptr, *bw = nullptr;
    int *d_err = nullptr; // device error word of the tensor-core training kernels
};

static constexpr int NW1 = 27 * CI * CH, NW2 = 27 * CH * CH, NW3 = 27 * CH;
static constexpr int NWT = NW1 + NW2 + NW3;

static unsigned nblk(int64_t n)
{
    int64_t b = (n + 255) / 256;
    if (b > 148 * 32) b = 148 * 32;
    return (unsigned)(b < 1 ? 1 : b);
}

static void free_work(cn_nn *nn)
{
    float *bufs[] = {nn->h1, nn->h2, nn->y, nn->c, nn->res, nn->gc, nn->gh2, nn->gh1};
    for (float *b : bufs)
        if (b) cudaFree(b);
    uint16_t *hb[] = {nn->bh1, nn->bh2, nn->bgh1, nn->bgh2};
    for (uint16_t *b : hb)
        if (b) cudaFree(b);
    if (nn->sums) cudaFree(nn->sums);
    nn->h1 = nn->h2 = nn->y = nn->c = nn->res = nn->gc = nn->gh2 = nn->gh1 = nullptr;
    nn->bh1 = nn->bh2 = nn->bgh1 = nn->bgh2 = nullptr;
    nn->sums = nullptr;
    nn->wB = nn->wP = 0;
}

// work buffers for batches of B patches of P^3 cells in the current training mode
static cn_status nn_work(cn_nn *nn, int B, int P)
{
    const bool have = nn->training == 1 ? nn->bh1 != nullptr : nn->h1 != nullptr;
    if (nn->wB >= B && nn->wP == P && have) return CN_OK;
    free_work(nn);
    const int64_t s6 = (int64_t)(P + 6) * (P + 6) * (P + 6), s4 = (int64_t)(P + 4) * (P + 4) * (P + 4),
                  s2 = (int64_t)(P + 2) * (P + 2) * (P + 2), s0 = (int64_t)P * P * P;
    if (nn->training == 1) {
        CN_CUDA_TRY(cudaMalloc(&nn->bh1, sizeof(uint16_t) * B * CH * s6));
        CN_CUDA_TRY(cudaMalloc(&nn->bgh1, sizeof(uint16_t) * B * CH * s6));
        CN_CUDA_TRY(cudaMalloc(&nn->bh2, sizeof(uint16_t) * B * CH * s4));
        CN_CUDA_TRY(cudaMalloc(&nn->bgh2, sizeof(uint16_t) * B * CH * s4));
        if (!nn->bw) CN_CUDA_TRY(cudaMalloc(&nn->bw, 2 * nntc::kPackedWeightBytes));
        if (!nn->d_err) {
            CN_CUDA_TRY(cudaMalloc(&nn->d_err, sizeof(int)));
            CN_CUDA_TRY(cudaMemset(nn->d_err, 0, sizeof(int)));
        }
    } else {
        CN_CUDA_TRY(cudaMalloc(&nn->h1, sizeof(float) * B * CH * s6));
        CN_CUDA_TRY(cudaMalloc(&nn->gh1, sizeof(float) * B * CH * s6));
        CN_CUDA_TRY(cudaMalloc(&nn->h2, sizeof(float) * B * CH * s4));
        CN_CUDA_TRY(cudaMalloc(&nn->gh2, sizeof(float) * B * CH * s4));
    }
    CN_CUDA_TRY(cudaMalloc(&nn->y, sizeof(float) * B * s2));
    CN_CUDA_TRY(cudaMalloc(&nn->c, sizeof(float) * B * s2));
    CN_CUDA_TRY(cudaMalloc(&nn->gc, sizeof(float) * B * s2));
    CN_CUDA_TRY(cudaMalloc(&nn->res, sizeof(float) * B * s0));
    CN_CUDA_TRY(cudaMalloc(&nn->sums, sizeof(double) * 2 * B));
    nn->wB = B;
    nn->wP = P;
    return CN_OK;
}

// the tensor-core training kernels' error word (set when a bounded wait ran
// out); read after a synchronisation, cleared when set
static cn_status nn_check_error(cn_nn *nn)
{
    if (!nn->d_err) return CN_OK;
    int e = 0;
    CN_CUDA_TRY(cudaMemcpy(&e, nn->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e == 0) return CN_OK;
    CN_CUDA_TRY(cudaMemset(nn->d_err, 0, sizeof(int)));
    return fail(CN_ERR_DEVICE, "learned smoother training: a tensor-core kernel gave up waiting (error word " +
                                    std::to_string(e) + ")");
}

template <int Cin, int Cout, bool RELU>
static void fwd_patch(const float *in, const float *W, float *out, int B, int S, cudaStream_t st)
{
    const int64_t n = (int64_t)B * (S - 2) * (S - 2) * (S - 2);
    int64_t b = (n + 127) / 128;
    if (b > 148 * 64) b = 148 * 64;
    conv_fwd_patch<Cin, Cout, RELU><<<(unsigned)b, 128, sizeof(float) * 27 * Cin * Cout, st>>>(in, W, out, B, S);
}

template <int Cin, int Cout>
static void bwd_patch(const float *in, const float *gout, const float *W, const float *act, float *gin, float *gW, int B,
                      int S, cudaStream_t st)
{
    conv_bwd_weight_patch<Cin, Cout><<<dim3(96, 27), 256, 0, st>>>(in, gout, gW, B, S);
    if (gin) {
        const int64_t n = (int64_t)B * S * S * S;
        int64_t b = (n + 127) / 128;
        if (b > 148 * 64) b = 148 * 64;
        conv_bwd_data_patch<Cin, Cout><<<(unsigned)b, 128, sizeof(float) * 27 * Cin * Cout, st>>>(gout, W, act, gin, B, S);
    }
}

extern "C" {

cn_status cn_nn_create(uint64_t seed, double omega, double init_scale, cn_nn **out)
{
    if (!out) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    cn_nn *nn = new cn_nn();
    nn->omega = omega;
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    std::vector<float> w(NWT);
    // He-style scales for the two hidden layers, a small last layer so the
    // untrained smoother starts as weighted Jacobi
    for (int i = 0; i < NW1; ++i) w[i] = nd(rng) * std::sqrt(2.f / (27 * CI));
    for (int i = 0; i < NW2; ++i) w[NW1 + i] = nd(rng) * std::sqrt(2.f / (27 * CH));
    for (int i = 0; i < NW3; ++i) w[NW1 + NW2 + i] = nd(rng) * (float)init_scale;
    cudaError_t e = cudaMalloc(&nn->w, sizeof(float) * NWT);
    if (e == cudaSuccess) e = cudaMalloc(&nn->m, sizeof(float) * NWT);
    if (e == cudaSuccess) e = cudaMalloc(&nn->v, sizeof(float) * NWT);
    if (e == cudaSuccess) e = cudaMalloc(&nn->g, sizeof(float) * NWT);
    if (e == cudaSuccess) e = cudaMemcpy(nn->w, w.data(), sizeof(float) * NWT, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(nn->m, 0, sizeof(float) * NWT);
    if (e == cudaSuccess) e = cudaMemset(nn->v, 0, sizeof(float) * NWT);
    if (e != cudaSuccess) {
        extern cn_status cn_nn_destroy(cn_nn *);
        cn_nn_destroy(nn);
        return cuda_fail(e, "cn_nn_create");
    }
    *out = nn;
    return CN_OK;
}

cn_status cn_nn_set_inference(cn_nn *nn, int mode)
{
    if (!nn || mode < 0 || mode > 1) return fail(CN_ERR_INVALID_ARGUMENT, "cn_nn_set_inference: bad argument");
    nn->inference = mode;
    return CN_OK;
}

cn_status cn_nn_set_training(cn_nn *nn, int mode)
{
    if (!nn || mode < 0 || mode > 1) return fail(CN_ERR_INVALID_ARGUMENT, "cn_nn_set_training: bad argument");
    nn->training = mode;
    return CN_OK;
}

cn_status cn_nn_destroy(cn_nn *nn)
{
    if (!nn) return CN_OK;
    free_work(nn);
    float *bufs[] = {nn->w, nn->m, nn->v, nn->g};
    for (float *b : bufs)
        if (b) cudaFree(b);
    if (nn->wpack) cudaFree(nn->wpack);
    if (nn->bw) cudaFree(nn->bw);
    if (nn->d_err) cudaFree(nn->d_err);
    delete nn;
    return CN_OK;
}

cn_status cn_nn_get_weights(const cn_nn *nn, float *host)
{
    if (!nn || !host) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    CN_CUDA_TRY(cudaMemcpy(host, nn->w, sizeof(float) * NWT, cudaMemcpyDeviceToHost));
    return CN_OK;
}

cn_status cn_nn_set_weights(cn_nn *nn, const float *host)
{
    if (!nn || !host) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    CN_CUDA_TRY(cudaMemcpy(nn->w, host, sizeof(float) * NWT, cudaMemcpyHostToDevice));
    return CN_OK;
}

int cn_nn_weight_count(void) { return NWT; }

// Loss and gradient (into the internal gradient buffer, also copied to
// grad_out if given: device or host pointer of NWT floats) for a batch of
// patches on the device: x [B][2][(P+8)^3], k [B][(P+2)^3], r [B][P^3].
cn_status cn_nn_loss_grad(cn_nn *nn, const float *x, const float *k, const float *r, int B, int P, double ih2,
                          double *loss, float *grad_out, void *stream)
{
    if (!nn || !x || !k || !r || B < 1 || P < 1) return fail(CN_ERR_INVALID_ARGUMENT, "cn_nn_loss_grad: bad argument");
    cudaStream_t st = as_stream(stream);
    cn_status s = nn_work(nn, B, P);
    if (s != CN_OK) return s;
    const float *W1 = nn->w, *W2 = nn->w + NW1, *W3 = nn->w + NW1 + NW2;
    const int S = P + 8;
    const nntc::TrainBufs T = {nn->bh1,  nn->bh2, nn->bgh1, nn->bgh2, nn->bw, nn->bw + nntc::kPackedWeightBytes / 2,
                               nn->y,    nn->gc,  nn->d_err};
    if (nn->training == 1) {
        if ((s = nntc::train_forward_tc(T, x, nn->w, B, P, st)) != CN_OK) return s;
    } else {
        fwd_patch<CI, CH, true>(x, W1, nn->h1, B, S, st);
        fwd_patch<CH, CH, true>(nn->h1, W2, nn->h2, B, S - 2, st);
        fwd_patch<CH, 1, false>(nn->h2, W3, nn->y, B, S - 4, st);
    }
    const int64_t s2 = (int64_t)(P + 2) * (P + 2) * (P + 2), s0 = (int64_t)P * P * P;
    loss_fwd<<<nblk(B * s2), 256, 0, st>>>(x, nn->y, (float)nn->omega, B, P, nn->c);
    CN_CUDA_TRY(cudaMemsetAsync(nn->sums, 0, sizeof(double) * 2 * B, st));
    {
        int64_t gx = (s0 + 255) / 256;
        if (gx > 64) gx = 64;
        loss_res<<<dim3((unsigned)gx, (unsigned)B), 256, 0, st>>>(nn->c, k, r, (float)ih2, B, P, nn->res, nn->sums);
    }
    loss_adjoint<<<nblk(B * s2), 256, 0, st>>>(nn->res, k, nn->sums, (float)ih2, B, P, nn->gc);
    if (nn->training == 1) {
        if ((s = nntc::train_backward_tc(T, x, nn->w, nn->g, B, P, st)) != CN_OK) return s;
    } else {
        CN_CUDA_TRY(cudaMemsetAsync(nn->g, 0, sizeof(float) * NWT, st));
        bwd_patch<CH, 1>(nn->h2, nn->gc, W3, nn->h2, nn->gh2, nn->g + NW1 + NW2, B, S - 4, st);
        bwd_patch<CH, CH>(nn->h1, nn->gh2, W2, nn->h1, nn->gh1, nn->g + NW1, B, S - 2, st);
        bwd_patch<CI, CH>(x, nn->gh1, W1, nullptr, nullptr, nn->g, B, S, st);
    }
    CN_CUDA_TRY(cudaGetLastError());
    if (grad_out) CN_CUDA_TRY(cudaMemcpyAsync(grad_out, nn->g, sizeof(float) * NWT, cudaMemcpyDefault, st));
    if (loss) {
        std::vector<double> h(2 * B);
        CN_CUDA_TRY(cudaMemcpyAsync(h.data(), nn->sums, sizeof(double) * 2 * B, cudaMemcpyDeviceToHost, st));
        CN_CUDA_TRY(cudaStreamSynchronize(st));
        if ((s = nn_check_error(nn)) != CN_OK) return s;
        double l = 0;
        for (int b = 0; b < B; ++b) l += h[2 * b] > 0 ? h[2 * b + 1] / h[2 * b] : 0.0;
        *loss = l / B;
    }
    return CN_OK;
}

cn_status cn_nn_adam_step(cn_nn *nn, double lr, void *stream)
{
    if (!nn) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    nn->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)nn->step), c2 = 1.f - std::pow(b2, (float)nn->step);
    adam_kernel<<<(NWT + 255) / 256, 256, 0, as_stream(stream)>>>(nn->w, nn->g, nn->m, nn->v, NWT, (float)lr, b1, b2,
                                                                   1e-8f, c1, c2);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

// Training on npatches device-resident patches: `epochs` passes of shuffled
// minibatches of `batch`, Adam with learning rate lr.  Returns the mean loss
// of the last epoch.
cn_status cn_nn_train(cn_nn *nn, const float *x, const float *k, const float *r, int npatches, int P, double ih2,
                      int epochs, int batch, double lr, uint64_t seed, double *last_loss, void *stream)
{
    if (!nn || !x || !k || !r || npatches < 1 || batch < 1) return fail(CN_ERR_INVALID_ARGUMENT, "cn_nn_train: bad argument");
    cudaStream_t st = as_stream(stream);
    if (batch > npatches) batch = npatches;
    const int64_t px = 2LL * (P + 8) * (P + 8) * (P + 8), pk = (int64_t)(P + 2) * (P + 2) * (P + 2), pr = (int64_t)P * P * P;
    float *bx = nullptr, *bk = nullptr, *br = nullptr;
    int *bidx = nullptr;
    CN_CUDA_TRY(cudaMalloc(&bx, sizeof(float) * batch * px));
    CN_CUDA_TRY(cudaMalloc(&bk, sizeof(float) * batch * pk));
    CN_CUDA_TRY(cudaMalloc(&br, sizeof(float) * batch * pr));
    CN_CUDA_TRY(cudaMalloc(&bidx, sizeof(int) * batch));
    std::mt19937_64 rng(seed);
    std::vector<int> order(npatches);
    for (int i = 0; i < npatches; ++i) order[i] = i;
    double ep_loss = 0;
    cn_status s = CN_OK;
    for (int e = 0; e < epochs && s == CN_OK; ++e) {
        std::shuffle(order.begin(), order.end(), rng);
        ep_loss = 0;
        int nb = 0;
        for (int i0 = 0; i0 + batch <= npatches && s == CN_OK; i0 += batch) {
            CN_CUDA_TRY(cudaMemcpyAsync(bidx, order.data() + i0, sizeof(int) * batch, cudaMemcpyHostToDevice, st));
            gather_batch<<<nblk(batch * px), 256, 0, st>>>(x, px, bidx, batch, bx);
            gather_batch<<<nblk(batch * pk), 256, 0, st>>>(k, pk, bidx, batch, bk);
            gather_batch<<<nblk(batch * pr), 256, 0, st>>>(r, pr, bidx, batch, br);
            double l = 0;
            s = cn_nn_loss_grad(nn, bx, bk, br, batch, P, ih2, &l, nullptr, st);
            if (s == CN_OK) s = cn_nn_adam_step(nn, lr, st);
            ep_loss += l;
            ++nb;
        }
        ep_loss /= (nb > 0 ? nb : 1);
    }
    cudaStreamSynchronize(st);
    if (s == CN_OK) s = nn_check_error(nn);
    cudaFree(bx);
    cudaFree(bk);
    cudaFree(br);
    cudaFree(bidx);
    if (last_loss) *last_loss = ep_loss;
    return s;
}

} // extern "C"

// ------------------------------------------------- multigrid integration
static cn_status level_bufs(cn_mg *m, int l)
{
    if ((int)m->nn_bufs.size() < 4 * m->nlevels) m->nn_bufs.resize(4 * m->nlevels, nullptr);
    if (m->nn_bufs[4 * l]) return CN_OK;
    cn_grid *g = m->p[l];
    const int nc[4] = {2, CH, CH, 1};
    for (int i = 0; i < 4; ++i) {
        cn_status s = cn_grid_create(g->nb, g->n, nc[i], CN_FLOAT32, g->begin, g->end, &m->nn_bufs[4 * l + i]);
        if (s != CN_OK) return s;
        s = sync_bc(m->nn_bufs[4 * l + i], nullptr);
        if (s != CN_OK) return s;
    }
    return CN_OK;
}

static GridIO gio(cn_grid *in, cn_grid *out, const LabGeom &Lt)
{
    GridIO g;
    g.in = reinterpret_cast<const float *>(in->d_data);
    g.in_cs = in->comp_stride;
    for (int c = 0; c < CH; ++c) g.in_bc[c] = bc_view(in, c < in->ncomp ? c : 0);
    g.out = reinterpret_cast<float *>(out->d_data);
    g.out_cs = out->comp_stride;
    g.L = Lt;
    g.nblocks = in->nblocks;
    return g;
}

template <int Cin, int Cout, bool RELU>
static cn_status conv_on_grid(cn_grid *in, cn_grid *out, const float *W, const LabGeom &Lt, cudaStream_t st)
{
    const int64_t n = (int64_t)in->nblocks * in->n[0] * in->n[1] * in->n[2];
    int64_t b = (n + 127) / 128;
    if (b > 148 * 64) b = 148 * 64;
    conv_grid<Cin, Cout, RELU><<<(unsigned)b, 128, sizeof(float) * 27 * Cin * Cout, st>>>(gio(in, out, Lt), W);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

static cn_status features(cn_mg *m, int l, const float *p, const float *f, float *rout, cudaStream_t st,
                          uint16_t *packed = nullptr)
{
    cn_grid *X = m->nn_bufs[4 * l];
    FeatArgs A;
    A.L = make_geom(m->p[l], &kS1);
    A.pbc = bc_view(m->p[l], 0);
    A.kbc = bc_view(m->k[l], 0);
    A.p = p;
    A.k = fptr(m->k[l]);
    A.f = f;
    A.coef = m->coef[l];
    A.ih2 = (float)(1.0 / (m->p[l]->h[0] * m->p[l]->h[0]));
    A.x0 = reinterpret_cast<float *>(X->d_data);
    A.x1 = A.x0 + X->comp_stride;
    A.rout = rout;
    A.packed = packed;
    const mg::Tile T = mg::tile_of(m->p[l]->n);
    features_tile<<<(unsigned)(m->p[l]->nblocks * T.count), mg::kTileThreads, 0, st>>>(A, T);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

// Grid inference with the hidden layer on the tensor cores: features (FP32)
// -> first layer on the CUDA cores (2 -> 16, BF16 out) -> hidden layer on the
// tensor cores (tcgen05, 16 -> 16) -> last layer on the CUDA cores fused with
// the update of p.  (The first and last layers' 2 input / 1 output channels
// would be padded to 16 on the tensor cores.)
static cn_status nn_smooth_tc(cn_mg *m, int l, int apps, bool zero_guess, cudaStream_t st)
{
    cn_grid *P = m->p[l], *X = m->nn_bufs[4 * l];
    if ((int)m->nn_act.size() < 2 * m->nlevels) m->nn_act.resize(2 * m->nlevels, nullptr);
    const size_t abytes = (size_t)P->nblocks * P->n[0] * P->n[1] * P->n[2] * 16 * sizeof(uint16_t);
    for (int i = 0; i < 2; ++i)
        if (!m->nn_act[2 * l + i]) CN_CUDA_TRY(cudaMalloc(&m->nn_act[2 * l + i], abytes));
    cn_nn *nn = m->nn;
    if (!nn->wpack) CN_CUDA_TRY(cudaMalloc(&nn->wpack, nntc::kPackedWeightBytes));
    uint16_t *w2 = nn->wpack;
    cn_status s;
    if ((s = nntc::pack_weights(nn->w + NW1, CH, CH, w2, st)) != CN_OK) return s;
    uint16_t *h1 = static_cast<uint16_t *>(m->nn_act[2 * l]), *h2 = static_cast<uint16_t *>(m->nn_act[2 * l + 1]);
    const float *x = reinterpret_cast<const float *>(X->d_data);
    for (int a = 0; a < apps; ++a) {
        const bool zg = zero_guess && a == 0;
        if ((s = features(m, l, zg ? nullptr : fptr(P), fptr(m->f[l]), nullptr, st)) != CN_OK) return s;
        if ((s = nntc::conv_first_cc(x, x + X->comp_stride, X->block_stride, P->nb, P->n, nn->w, h1, st)) != CN_OK)
            return s;
        if ((s = nntc::conv_hidden(h1, P->nb, P->n, w2, 1, h2, P->d_err, st)) != CN_OK) return s;
        if ((s = nntc::conv_update_cc(h2, P->nb, P->n, nn->w + NW1 + NW2, x, X->block_stride, fptr(P),
                                      P->block_stride, (float)nn->omega, zg ? 1 : 0, st)) != CN_OK)
            return s;
    }
    return CN_OK;
}

cn_status nn_smooth(cn_mg *m, int l, int apps, bool zero_guess, cudaStream_t st)
{
    cn_status s = level_bufs(m, l);
    if (s != CN_OK) return s;
    if (m->nn->inference == 1 && nntc::supported(m->p[l]->n) && apps > 0) return nn_smooth_tc(m, l, apps, zero_guess, st);
    cn_grid *X = m->nn_bufs[4 * l], *H1 = m->nn_bufs[4 * l + 1], *H2 = m->nn_bufs[4 * l + 2], *Y = m->nn_bufs[4 * l + 3];
    const LabGeom Lt = make_geom(m->p[l], &kS1t);
    const float *W1 = m->nn->w, *W2 = m->nn->w + NW1, *W3 = m->nn->w + NW1 + NW2;
    const int64_t n = m->p[l]->comp_stride;
    if (apps == 0 && zero_guess) CN_CUDA_TRY(cudaMemsetAsync(m->p[l]->d_data, 0, sizeof(float) * n, st));
    for (int a = 0; a < apps; ++a) {
        const bool zg = zero_guess && a == 0;
        if ((s = features(m, l, zg ? nullptr : fptr(m->p[l]), fptr(m->f[l]), nullptr, st)) != CN_OK) return s;
        if ((s = conv_on_grid<CI, CH, true>(X, H1, W1, Lt, st)) != CN_OK) return s;
        if ((s = conv_on_grid<CH, CH, true>(H1, H2, W2, Lt, st)) != CN_OK) return s;
        if ((s = conv_on_grid<CH, 1, false>(H2, Y, W3, Lt, st)) != CN_OK) return s;
        smooth_update<<<nblk(n), 256, 0, st>>>(fptr(m->p[l]), reinterpret_cast<const float *>(X->d_data),
                                                reinterpret_cast<const float *>(Y->d_data), (float)m->nn->omega, n,
                                                zg ? 1 : 0);
        CN_CUDA_TRY(cudaGetLastError());
    }
    return CN_OK;
}

// patch collection state used by the capture hook
struct Collect {
    float *x, *k, *r;
    int max, n, per;
    std::mt19937_64 *rng;
    int *d_blocks;
};

static cn_status take_patches(cn_mg *m, Collect *c, const float *p, cudaStream_t st)
{
    if (c->n >= c->max) return CN_OK;
    cn_status s = level_bufs(m, 0);
    if (s != CN_OK) return s;
    cn_grid *X = m->nn_bufs[0], *Y = m->nn_bufs[3];
    // r goes to the Y buffer (1 component)
    if ((s = features(m, 0, p, fptr(m->f[0]), fptr(Y), st)) != CN_OK) return s;
    const int take = std::min(c->per, c->max - c->n);
    std::vector<int> blocks(take);
    std::uniform_int_distribution<int> ud(0, m->p[0]->nblocks - 1);
    for (int i = 0; i < take; ++i) blocks[i] = ud(*c->rng);
    CN_CUDA_TRY(cudaMemcpyAsync(c->d_blocks, blocks.data(), sizeof(int) * take, cudaMemcpyHostToDevice, st));
    const int P = m->p[0]->n[0];
    const int64_t sx = (int64_t)(P + 8) * (P + 8) * (P + 8), sk = (int64_t)(P + 2) * (P + 2) * (P + 2),
                  sr = (int64_t)P * P * P;
    const cn_stencil s4 = {{-4, -4, -4}, {5, 5, 5}, 1};
    const LabGeom L4 = make_geom(X, &s4), L1 = make_geom(m->k[0], &kS1t);
    const cn_stencil s0 = {{0, 0, 0}, {1, 1, 1}, 0};
    const LabGeom L0 = make_geom(Y, &s0);
    for (int ch = 0; ch < 2; ++ch)
        extract_patch<<<nblk(take * sx), 256, 0, st>>>(reinterpret_cast<const float *>(X->d_data) + ch * X->comp_stride,
                                                       L4, bc_view(X, ch), c->d_blocks, take, 4,
                                                       c->x + (int64_t)c->n * 2 * sx + ch * sx, 2 * sx);
    extract_patch<<<nblk(take * sk), 256, 0, st>>>(fptr(m->k[0]), L1, bc_view(m->k[0], 0), c->d_blocks, take, 1,
                                                   c->k + (int64_t)c->n * sk, sk);
    extract_patch<<<nblk(take * sr), 256, 0, st>>>(fptr(Y), L0, bc_view(Y, 0), c->d_blocks, take, 0,
                                                   c->r + (int64_t)c->n * sr, sr);
    CN_CUDA_TRY(cudaGetLastError());
    c->n += take;
    return CN_OK;
}

static cn_status capture_hook(cn_mg *m, cudaStream_t st)
{
    return take_patches(m, reinterpret_cast<Collect *>(m->capture_ctx), fptr(m->p[0]), st);
}

extern "C" {

// Training samples from plain V-cycles solving L p = f: for each of `cycles`
// outer cycles, `per_snapshot` random blocks of the finest residual before
// pre-smoothing and after the coarse-grid correction.  Outputs (device
// pointers): x [max][2][(P+8)^3], k [max][(P+2)^3], r [max][P^3], P = block
// cells of the finest level (cubic blocks).
cn_status cn_mg_collect_patches(cn_mg *m, const cn_grid *f, int cycles, int per_snapshot, uint64_t seed, float *x,
                                float *k, float *r, int max_patches, int *count, void *stream)
{
    if (!m || !f || !x || !k || !r || !count) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    cn_grid *g0 = m->p[0];
    if (g0->n[0] != g0->n[1] || g0->n[0] != g0->n[2] || g0->n[0] < 4)
        return fail(CN_ERR_UNSUPPORTED, "patch collection needs cubic blocks of at least 4 cells");
    cudaStream_t st = as_stream(stream);
    cn_grid *p64 = nullptr;
    cn_status s = cn_grid_create(g0->nb, g0->n, 1, CN_FLOAT64, g0->begin, g0->end, &p64);
    if (s != CN_OK) return s;
    std::mt19937_64 rng(seed);
    Collect c{x, k, r, max_patches, 0, per_snapshot, &rng, nullptr};
    if (cudaMalloc(&c.d_blocks, sizeof(int) * (per_snapshot > 0 ? per_snapshot : 1)) != cudaSuccess) {
        cn_grid_destroy(p64);
        return fail(CN_ERR_OUT_OF_MEMORY, "cn_mg_collect_patches");
    }
    cn_nn *saved = m->nn;
    m->nn = nullptr; // plain V-cycles
    CN_CUDA_TRY(cudaMemsetAsync(p64->d_data, 0, sizeof(double) * p64->comp_stride, st));
    for (int cyc = 0; cyc < cycles && s == CN_OK; ++cyc) {
        s = cn_mg_residual(m, p64, f, m->f[0], nullptr, nullptr, stream);
        if (s == CN_OK) s = take_patches(m, &c, nullptr, st);
        m->capture = capture_hook;
        m->capture_ctx = &c;
        if (s == CN_OK) s = vcycle(m, 0, st);
        m->capture = nullptr;
        m->capture_ctx = nullptr;
        if (s == CN_OK) s = cn_mg_accumulate(m, p64, stream);
    }
    m->nn = saved;
    cudaStreamSynchronize(st);
    cudaFree(c.d_blocks);
    cn_grid_destroy(p64);
    *count = c.n;
    return s;
}

// Smoother selection: nn == NULL restores weighted Jacobi everywhere; else the
// network replaces Jacobi on the levels whose bit is set in level_mask.
cn_status cn_mg_set_smoother_phases(cn_mg *m, cn_nn *nn, unsigned pre_mask, unsigned post_mask, int pre_apps,
                                    int post_apps)
{
    if (!m) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    m->nn = nn;
    m->nn_levels = nn ? pre_mask : 0;
    m->nn_post_levels = nn ? post_mask : 0;
    m->nn_pre_apps = pre_apps;
    m->nn_post_apps = post_apps;
    if (nn) {
        for (int l = 0; l < m->nlevels - 1; ++l)
            if (((pre_mask | post_mask) >> l) & 1) {
                cn_status s = level_bufs(m, l);
                if (s != CN_OK) return s;
            }
    }
    return CN_OK;
}

cn_status cn_mg_set_smoother(cn_mg *m, cn_nn *nn, unsigned level_mask)
{
    return cn_mg_set_smoother_phases(m, nn, level_mask, level_mask, -1, -1);
}

} // extern "C"
