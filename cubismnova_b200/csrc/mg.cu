// mg.cu -- geometric multigrid for div(k grad p) = f on a periodic block grid.
//
// The reference announces "integrated multigrid solvers" (README.rst:43-44)
// without code; this is the standard cell-centred method on the lab/stencil
// machinery of this library:
//   operator  (L p)_i = ih2 * sum_d [ kf(i,i+e_d)(p_{i+e_d} - p_i) - kf(i-e_d,i)(p_i - p_{i-e_d}) ]
//             kf(a, b) = (a*b + a*b) / (a + b)        (harmonic face mean)
//   smoother  weighted Jacobi  p <- p + omega (L p - f) / D,  D = ih2 * sum of the 6 kf
//   restrict  f_c = (sum of the 8 children's residuals) / 8, k_c = mean of 8 k
//   prolong   trilinear cell-centred weights (3/4, 1/4 per direction)
//   coarsest  conjugate gradients in FP64 in one CTA (mean-zero projection)
// Levels keep the block count and halve the cells per block (32^3 -> 16^3 ->
// ... -> 1^3), so fine block b maps onto coarse block b.  V-cycle fields are
// FP32; the outer defect correction keeps the fine solution, its residual and
// the residual norm in FP64, because an FP32 solution cannot be represented
// accurately enough for a 1e-8 relative residual.  Neighbour values come from
// the same lab resolution as every other stencil (periodic block wrap, and the
// grid's BCs if any); halo cells inside a block are plain cached loads.
#include "cn_internal.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace cn {
namespace mg {

struct Geo {
    LabGeom L;       // stencil (-1,2) non-tensorial, geometry of the solution p
    LabGeom Lk;      // the same for the FP32 grids (k, f, r): block strides may differ
    BcView bc;       // BCs of p
    int nblocks;
};

// Cell t of a level in block order (32-bit arithmetic: cn_mg_create checks
// that the finest level has fewer than 2^31 cells).
__device__ __forceinline__ void cell_of(int64_t t, const LabGeom &L, int &block, int &x, int &y,
                                        int &z)
{
    const unsigned n0 = (unsigned)L.n[0], n1 = (unsigned)L.n[1];
    const unsigned cells = n0 * n1 * (unsigned)L.n[2];
    const unsigned tt = (unsigned)t;
    const unsigned b = tt / cells;
    const unsigned c = tt - b * cells;
    const unsigned yz = c / n0;
    const unsigned zz = yz / n1;
    block = (int)b;
    x = (int)(c - yz * n0);
    y = (int)(yz - zz * n1);
    z = (int)zz;
}

// neighbour values: cn::lab_fetch (plain loads inside the block and for
// periodic neighbours of blocks without BCs, the lab otherwise)
template <typename T>
__device__ __forceinline__ T fetch(const T *comp, const LabGeom &L, const BcView &bc, int block, int x, int y,
                                   int z)
{
    return lab_fetch<T>(comp, L, bc, block, x, y, z);
}

template <typename T> __device__ __forceinline__ T harm(T a, T b)
{
    const T t = a * b;
    return (t + t) / (a + b);
}

// The 13 values of the 7-point operator at one cell: v[0] = p, v[1] = k,
// then per direction d: p(+e_d), p(-e_d), k(+e_d), k(-e_d); p == NULL reads
// as zero.  Cells interior to their block take plain loads.
template <typename TP>
__device__ __forceinline__ void load7(const TP *p, const float *k, const Geo &G, const BcView &kbc, int block,
                                      int x, int y, int z, TP (&v)[14])
{
    const LabGeom &L = G.L, &Lk = G.Lk;
    if (x > 0 && y > 0 && z > 0 && x < L.n[0] - 1 && y < L.n[1] - 1 && z < L.n[2] - 1) {
        const int64_t cell = x + (int64_t)L.n[0] * (y + (int64_t)L.n[1] * z);
        const TP *pb = p ? p + (int64_t)block * L.bstride + cell : nullptr;
        const float *kb = k + (int64_t)block * Lk.bstride + cell;
        const int64_t st[3] = {1, L.n[0], (int64_t)L.n[0] * L.n[1]};
        v[0] = pb ? __ldg(pb) : TP(0);
        v[1] = (TP)__ldg(kb);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v[2 + 4 * d] = pb ? __ldg(pb + st[d]) : TP(0);
            v[3 + 4 * d] = pb ? __ldg(pb - st[d]) : TP(0);
            v[4 + 4 * d] = (TP)__ldg(kb + st[d]);
            v[5 + 4 * d] = (TP)__ldg(kb - st[d]);
        }
    } else {
        v[0] = p ? fetch<TP>(p, L, G.bc, block, x, y, z) : TP(0);
        v[1] = (TP)fetch<float>(k, Lk, kbc, block, x, y, z);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int ox = d == 0, oy = d == 1, oz = d == 2;
            v[2 + 4 * d] = p ? fetch<TP>(p, L, G.bc, block, x + ox, y + oy, z + oz) : TP(0);
            v[3 + 4 * d] = p ? fetch<TP>(p, L, G.bc, block, x - ox, y - oy, z - oz) : TP(0);
            v[4 + 4 * d] = (TP)fetch<float>(k, Lk, kbc, block, x + ox, y + oy, z + oz);
            v[5 + 4 * d] = (TP)fetch<float>(k, Lk, kbc, block, x - ox, y - oy, z - oz);
        }
    }
}

// L p and the diagonal D at one cell from its 13 values; TP is the solution
// type (float in the V-cycle, double in the outer residual), k is FP32.
template <typename TP>
__device__ __forceinline__ void op7_math(const TP (&v)[14], TP ih2, TP &Lp, TP &D, TP &pc)
{
    pc = v[0];
    const TP kc = v[1];
    TP f[3], s[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const TP pp = v[2 + 4 * d], pm = v[3 + 4 * d];
        const TP kp = harm<TP>(kc, v[4 + 4 * d]);
        const TP km = harm<TP>(v[5 + 4 * d], kc);
        f[d] = kp * (pp - pc) - km * (pc - pm);
        s[d] = kp + km;
    }
    Lp = ih2 * ((f[0] + f[1]) + f[2]);
    D = ih2 * ((s[0] + s[1]) + s[2]);
}

template <typename TP>
__device__ __forceinline__ void op7(const TP *p, const float *k, const Geo &G, const BcView &kbc,
                                    int block, int x, int y, int z, TP ih2, TP &Lp, TP &D, TP &pc)
{
    TP v[14];
    load7<TP>(p, k, G, kbc, block, x, y, z, v);
    op7_math<TP>(v, ih2, Lp, D, pc);
}

struct KArgs {
    Geo G;
    BcView kbc;
    const float *k;
    float ih2;
    double ih2d;
};

// weighted Jacobi sweep: pout = pin + omega (L pin - f) / D  (pin == NULL: zero guess)
__global__ void __launch_bounds__(256) jacobi_kernel(const __grid_constant__ KArgs a, const float *pin,
                                                     const float *f, float *pout, float omega)
{
    const LabGeom &L = a.G.L;
    const int64_t total = (int64_t)a.G.nblocks * L.n[0] * L.n[1] * L.n[2];
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        int block, x, y, z;
        cell_of(t, L, block, x, y, z);
        const int64_t o = (int64_t)block * L.bstride + x + (int64_t)L.n[0] * (y + (int64_t)L.n[1] * z);
        const float fc = __ldg(f + o);
        float Lp, D, pc;
        op7<float>(pin, a.k, a.G, a.kbc, block, x, y, z, a.ih2, Lp, D, pc);
        // zero guess (pin == NULL): L 0 = 0, only the diagonal is used
        pout[o] = pin ? pc + omega * ((Lp - fc) / D) : 0.0f + omega * ((0.0f - fc) / D);
    }
}

// residual of the fine level restricted onto the coarse right-hand side:
// one thread per coarse cell, fc = (sum of its 8 children's f - L p) / 8
__global__ void __launch_bounds__(256) resid_restrict_kernel(const __grid_constant__ KArgs a, const float *p,
                                                             const float *f,
                                                             LabGeom Lc, float *fc)
{
    const LabGeom &L = a.G.L;
    const int64_t total = (int64_t)a.G.nblocks * Lc.n[0] * Lc.n[1] * Lc.n[2];
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        int block, X, Y, Z;
        cell_of(t, Lc, block, X, Y, Z);
        float r[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int x = 2 * X + (c & 1), y = 2 * Y + ((c >> 1) & 1), z = 2 * Z + (c >> 2);
            const int64_t o = (int64_t)block * L.bstride + x + (int64_t)L.n[0] * (y + (int64_t)L.n[1] * z);
            float Lp, D, pc;
            op7<float>(p, a.k, a.G, a.kbc, block, x, y, z, a.ih2, Lp, D, pc);
            r[c] = __ldg(f + o) - Lp;
        }
        const float s = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        fc[(int64_t)block * Lc.bstride + X + (int64_t)Lc.n[0] * (Y + (int64_t)Lc.n[1] * Z)] = s * 0.125f;
    }
}

// coarse k = mean of the 8 children
__global__ void __launch_bounds__(256) restrict_mean_kernel(LabGeom L, const float *kf, LabGeom Lc,
                                                            float *kc, int nblocks)
{
    const int64_t total = (int64_t)nblocks * Lc.n[0] * Lc.n[1] * Lc.n[2];
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        int block, X, Y, Z;
        cell_of(t, Lc, block, X, Y, Z);
        float v[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int x = 2 * X + (c & 1), y = 2 * Y + ((c >> 1) & 1), z = 2 * Z + (c >> 2);
            v[c] = kf[(int64_t)block * L.bstride + x + (int64_t)L.n[0] * (y + (int64_t)L.n[1] * z)];
        }
        const float s = ((v[0] + v[1]) + (v[2] + v[3])) + ((v[4] + v[5]) + (v[6] + v[7]));
        kc[(int64_t)block * Lc.bstride + X + (int64_t)Lc.n[0] * (Y + (int64_t)Lc.n[1] * Z)] = s * 0.125f;
    }
}

// p_fine += trilinear interpolation of the coarse correction e
__global__ void __launch_bounds__(256) prolong_kernel(const __grid_constant__ LabGeom L, float *p,
                                                      const __grid_constant__ LabGeom Lct,
                                                      const __grid_constant__ BcView cbc, const float *e,
                                                      int nblocks)
{
    const int64_t total = (int64_t)nblocks * L.n[0] * L.n[1] * L.n[2];
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        int block, x, y, z;
        cell_of(t, L, block, x, y, z);
        const int X = x >> 1, Y = y >> 1, Z = z >> 1;
        const int sx = (x & 1) ? 1 : -1, sy = (y & 1) ? 1 : -1, sz = (z & 1) ? 1 : -1;
        float v[8];
        if ((unsigned)(X + sx) < (unsigned)Lct.n[0] && (unsigned)(Y + sy) < (unsigned)Lct.n[1] &&
            (unsigned)(Z + sz) < (unsigned)Lct.n[2]) {
            const float *eb = e + (int64_t)block * Lct.bstride + X + (int64_t)Lct.n[0] * (Y + (int64_t)Lct.n[1] * Z);
            const int64_t ox = sx, oy = (int64_t)sy * Lct.n[0], oz = (int64_t)sz * Lct.n[0] * Lct.n[1];
            v[0] = __ldg(eb);
            v[1] = __ldg(eb + ox);
            v[2] = __ldg(eb + oy);
            v[3] = __ldg(eb + ox + oy);
            v[4] = __ldg(eb + oz);
            v[5] = __ldg(eb + ox + oz);
            v[6] = __ldg(eb + oy + oz);
            v[7] = __ldg(eb + ox + oy + oz);
        } else {
            v[0] = fetch<float>(e, Lct, cbc, block, X, Y, Z);
            v[1] = fetch<float>(e, Lct, cbc, block, X + sx, Y, Z);
            v[2] = fetch<float>(e, Lct, cbc, block, X, Y + sy, Z);
            v[3] = fetch<float>(e, Lct, cbc, block, X + sx, Y + sy, Z);
            v[4] = fetch<float>(e, Lct, cbc, block, X, Y, Z + sz);
            v[5] = fetch<float>(e, Lct, cbc, block, X + sx, Y, Z + sz);
            v[6] = fetch<float>(e, Lct, cbc, block, X, Y + sy, Z + sz);
            v[7] = fetch<float>(e, Lct, cbc, block, X + sx, Y + sy, Z + sz);
        }
        const float a0 = 0.75f * v[0] + 0.25f * v[1];
        const float a1 = 0.75f * v[2] + 0.25f * v[3];
        const float a2 = 0.75f * v[4] + 0.25f * v[5];
        const float a3 = 0.75f * v[6] + 0.25f * v[7];
        const float b0 = 0.75f * a0 + 0.25f * a1;
        const float b1 = 0.75f * a2 + 0.25f * a3;
        const float val = 0.75f * b0 + 0.25f * b1;
        const int64_t o = (int64_t)block * L.bstride + x + (int64_t)L.n[0] * (y + (int64_t)L.n[1] * z);
        p[o] = p[o] + val;
    }
}

// FP64 residual of the outer iteration: r = f - L p64 (p64 += e first if e),
// r32 = (float) r, per-CTA FP64 partial sums of r^2 (and f^2).
__global__ void __launch_bounds__(256) resid64_kernel(const __grid_constant__ KArgs a, const double *p64,
                                                      const float *f,
                                                      float *r32, double *partials)
{
    __shared__ double sh[2][8];
    const LabGeom &L = a.G.L;
    const int64_t total = (int64_t)a.G.nblocks * L.n[0] * L.n[1] * L.n[2];
    double rr = 0, ff = 0;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        int block, x, y, z;
        cell_of(t, L, block, x, y, z);
        const LabGeom &Lk = a.G.Lk;
        const int64_t o = (int64_t)block * Lk.bstride + x + (int64_t)Lk.n[0] * (y + (int64_t)Lk.n[1] * z);
        double Lp, D, pc;
        op7<double>(p64, a.k, a.G, a.kbc, block, x, y, z, a.ih2d, Lp, D, pc);
        const double fc = (double)__ldg(f + o);
        const double r = fc - Lp;
        if (r32) r32[o] = (float)r;
        rr += r * r;
        ff += fc * fc;
    }
    for (int off = 16; off > 0; off >>= 1) {
        rr += __shfl_down_sync(0xffffffffu, rr, off);
        ff += __shfl_down_sync(0xffffffffu, ff, off);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        sh[0][w] = rr;
        sh[1][w] = ff;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0, s1 = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            s0 += sh[0][i];
            s1 += sh[1][i];
        }
        partials[2 * blockIdx.x] = s0;
        partials[2 * blockIdx.x + 1] = s1;
    }
}

__global__ void __launch_bounds__(256) sum_pairs_kernel(const double *partials, int n, double *out)
{
    __shared__ double sh[2][256];
    double a = 0, b = 0;
    for (int i = threadIdx.x; i < n; i += 256) {
        a += partials[2 * i];
        b += partials[2 * i + 1];
    }
    sh[0][threadIdx.x] = a;
    sh[1][threadIdx.x] = b;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + s];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sh[0][0];
        out[1] = sh[1][0];
    }
}

// p64 += e (block layouts with their own strides)
__global__ void __launch_bounds__(256) axpy64_kernel(double *p64, int64_t s64, const float *e, int64_t s32,
                                                     int64_t cells, int nblocks)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cells * nblocks;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = i / cells, c = i - b * cells;
        p64[b * s64 + c] += (double)e[b * s32 + c];
    }
}

// Coarsest level: CG in FP64 on -L x = -f, one CTA, cells <= 4096, periodic
// grid of global extent (GX, GY, GZ); block layout in and out.
constexpr int kCoarseMax = 4096;
constexpr int kCoarseThreads = 1024;

__global__ void __launch_bounds__(kCoarseThreads)
    coarsest_cg_kernel(LabGeom L, const float *f, const float *k, float *p, double ih2, int max_iter,
                       double rtol, int *iters_out)
{
    extern __shared__ double sm[];
    const int GX = L.nb[0] * L.n[0], GY = L.nb[1] * L.n[1], GZ = L.nb[2] * L.n[2];
    const int N = GX * GY * GZ;
    double *kk = sm;            // k
    double *d = kk + N;         // search direction
    double *red = d + N;        // 32 reduction slots
    constexpr int PER = kCoarseMax / kCoarseThreads;
    double x[PER], r[PER], q[PER];
    auto gidx = [&](int i, int &blk, int64_t &o) {
        const int gx = i % GX, gy = (i / GX) % GY, gz = i / (GX * GY);
        const int bx = gx / L.n[0], by = gy / L.n[1], bz = gz / L.n[2];
        blk = bx + L.nb[0] * (by + L.nb[1] * bz);
        o = (int64_t)blk * L.bstride + (gx % L.n[0]) + (int64_t)L.n[0] * ((gy % L.n[1]) + (int64_t)L.n[1] * (gz % L.n[2]));
    };
    auto block_sum = [&](double v) -> double {
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
        __syncthreads();
        double s = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
        return s;
    };
    // load, b = -f with its mean removed
    double bsum = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int i = threadIdx.x + j * kCoarseThreads;
        x[j] = 0;
        r[j] = 0;
        if (i < N) {
            int blk;
            int64_t o;
            gidx(i, blk, o);
            kk[i] = (double)k[o];
            r[j] = -(double)f[o];
            bsum += r[j];
        }
    }
    const double mean = block_sum(bsum) / N;
    double rr = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int i = threadIdx.x + j * kCoarseThreads;
        if (i < N) {
            r[j] -= mean;
            d[i] = r[j];
            rr += r[j] * r[j];
        }
    }
    rr = block_sum(rr);
    const double stop = rtol * rtol * rr;
    int it = 0;
    for (; it < max_iter && rr > stop && rr > 0; ++it) {
        __syncthreads();
        double dq = 0;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const int i = threadIdx.x + j * kCoarseThreads;
            q[j] = 0;
            if (i < N) {
                const int gx = i % GX, gy = (i / GX) % GY, gz = i / (GX * GY);
                const int nbr[6] = {((gx + 1) % GX) + GX * (gy + GY * gz), ((gx + GX - 1) % GX) + GX * (gy + GY * gz),
                                    gx + GX * (((gy + 1) % GY) + GY * gz), gx + GX * (((gy + GY - 1) % GY) + GY * gz),
                                    gx + GX * (gy + GY * ((gz + 1) % GZ)), gx + GX * (gy + GY * ((gz + GZ - 1) % GZ))};
                double s = 0;
                const double kc = kk[i];
#pragma unroll
                for (int m = 0; m < 6; ++m) {
                    const double kn = kk[nbr[m]];
                    const double t = kc * kn;
                    s += ((t + t) / (kc + kn)) * (d[i] - d[nbr[m]]);
                }
                q[j] = ih2 * s; // (-L d)_i
                dq += d[i] * q[j];
            }
        }
        dq = block_sum(dq);
        const double alpha = rr / dq;
        double rn = 0;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const int i = threadIdx.x + j * kCoarseThreads;
            if (i < N) {
                x[j] += alpha * d[i];
                r[j] -= alpha * q[j];
                rn += r[j] * r[j];
            }
        }
        rn = block_sum(rn);
        const double beta = rn / rr;
        rr = rn;
        __syncthreads();
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const int i = threadIdx.x + j * kCoarseThreads;
            if (i < N) d[i] = r[j] + beta * d[i];
        }
    }
    // mean-zero solution back to the block layout
    double xs = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int i = threadIdx.x + j * kCoarseThreads;
        if (i < N) xs += x[j];
    }
    const double xm = block_sum(xs) / N;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int i = threadIdx.x + j * kCoarseThreads;
        if (i < N) {
            int blk;
            int64_t o;
            gidx(i, blk, o);
            p[o] = (float)(x[j] - xm);
        }
    }
    if (threadIdx.x == 0 && iters_out) *iters_out = it;
}

} // namespace mg
} // namespace cn

// ---------------------------------------------------------------- host side
using namespace cn;
using namespace cn::mg;

#include "mg_internal.h"

const cn_stencil kS1 = {{-1, -1, -1}, {2, 2, 2}, 0};
const cn_stencil kS1t = {{-1, -1, -1}, {2, 2, 2}, 1};

KArgs kargs(cn_mg *m, int l)
{
    KArgs a;
    a.G.L = make_geom(m->p[l], &kS1);
    a.G.Lk = a.G.L;
    a.G.bc = bc_view(m->p[l], 0);
    a.G.nblocks = m->p[l]->nblocks;
    a.kbc = bc_view(m->k[l], 0);
    a.k = reinterpret_cast<const float *>(m->k[l]->d_data);
    a.ih2d = 1.0 / (m->p[l]->h[0] * m->p[l]->h[0]);
    a.ih2 = (float)a.ih2d;
    return a;
}

unsigned grid_for(int64_t n)
{
    int64_t b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return (unsigned)(b < 1 ? 1 : b);
}

float *fptr(cn_grid *g) { return reinterpret_cast<float *>(g->d_data); }

// weighted Jacobi sweeps on level l (p = 0 on entry if zero_guess)
static cn_status smooth(cn_mg *m, int l, int sweeps, bool zero_guess, cudaStream_t st)
{
    KArgs a = kargs(m, l);
    const int64_t cells = (int64_t)m->p[l]->nblocks * m->p[l]->n[0] * m->p[l]->n[1] * m->p[l]->n[2];
    for (int s = 0; s < sweeps; ++s) {
        const bool zg = zero_guess && s == 0;
        // ping-pong so that the result of the last sweep lands in p
        float *src = fptr(m->p[l]), *dst = fptr(m->pt[l]);
        jacobi_kernel<<<grid_for(cells), 256, 0, st>>>(a, zg ? nullptr : src, fptr(m->f[l]), dst,
                                                        (float)m->omega);
        CN_CUDA_TRY(cudaGetLastError());
        std::swap(m->p[l], m->pt[l]);
    }
    if (sweeps == 0 && zero_guess)
        CN_CUDA_TRY(cudaMemsetAsync(m->p[l]->d_data, 0, (size_t)m->p[l]->comp_stride * 4, st));
    return CN_OK;
}

static cn_status coarsest(cn_mg *m, int l, cudaStream_t st)
{
    cn_grid *g = m->p[l];
    const LabGeom L = make_geom(g, &kS1);
    const int N = g->nblocks * g->n[0] * g->n[1] * g->n[2];
    const size_t smem = (size_t)(2 * N + 32) * sizeof(double);
    CN_CUDA_TRY(cudaFuncSetAttribute(coarsest_cg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    coarsest_cg_kernel<<<1, kCoarseThreads, smem, st>>>(L, fptr(m->f[l]), fptr(m->k[l]), fptr(g),
                                                         1.0 / (g->h[0] * g->h[0]), m->coarse_iters_max,
                                                         1e-13, m->iters);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}


static cn_status smooth_any(cn_mg *m, int l, int sweeps, bool zero_guess, cudaStream_t st)
{
    if (m->nn && ((m->nn_levels >> l) & 1)) return nn_smooth(m, l, sweeps, zero_guess, st);
    return smooth(m, l, sweeps, zero_guess, st);
}

cn_status vcycle(cn_mg *m, int l, cudaStream_t st)
{
    if (l == m->nlevels - 1) return coarsest(m, l, st);
    cn_status s = smooth_any(m, l, m->nu1, true, st);
    if (s != CN_OK) return s;
    KArgs a = kargs(m, l);
    const LabGeom Lc = make_geom(m->p[l + 1], &kS1);
    const int64_t ccells = (int64_t)m->p[l + 1]->nblocks * Lc.n[0] * Lc.n[1] * Lc.n[2];
    resid_restrict_kernel<<<grid_for(ccells), 256, 0, st>>>(a, fptr(m->p[l]), fptr(m->f[l]), Lc,
                                                             fptr(m->f[l + 1]));
    CN_CUDA_TRY(cudaGetLastError());
    s = vcycle(m, l + 1, st);
    if (s != CN_OK) return s;
    const LabGeom Lf = make_geom(m->p[l], &kS1);
    const LabGeom Lct = make_geom(m->p[l + 1], &kS1t);
    const int64_t fcells = (int64_t)m->p[l]->nblocks * Lf.n[0] * Lf.n[1] * Lf.n[2];
    prolong_kernel<<<grid_for(fcells), 256, 0, st>>>(Lf, fptr(m->p[l]), Lct, bc_view(m->p[l + 1], 0),
                                                      fptr(m->p[l + 1]), m->p[l]->nblocks);
    CN_CUDA_TRY(cudaGetLastError());
    if (l == 0 && m->capture) {
        s = m->capture(m, st);
        if (s != CN_OK) return s;
    }
    return smooth_any(m, l, m->nu2, false, st);
}

extern "C" {

cn_status cn_mg_create(cn_grid *k, int nu1, int nu2, double omega, int max_levels, cn_mg **out)
{
    if (!k || !out) return fail(CN_ERR_INVALID_ARGUMENT, "cn_mg_create: NULL argument");
    *out = nullptr;
    if (k->dtype != CN_FLOAT32 || k->ncomp < 1)
        return fail(CN_ERR_UNSUPPORTED, "cn_mg_create: the coefficient grid must be FLOAT32");
    if (k->h[0] != k->h[1] || k->h[0] != k->h[2])
        return fail(CN_ERR_UNSUPPORTED, "cn_mg_create: cubic cells are required");
    if (nu1 < 0 || nu2 < 0 || omega <= 0 || omega >= 2)
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_mg_create: bad smoothing parameters");
    if ((int64_t)k->nblocks * k->n[0] * k->n[1] * k->n[2] >= ((int64_t)1 << 31))
        return fail(CN_ERR_UNSUPPORTED, "cn_mg_create: at most 2^31 - 1 cells");
    cn_mg *m = new cn_mg();
    m->nu1 = nu1;
    m->nu2 = nu2;
    m->omega = omega;
    // levels: halve cells per block while all extents are even
    int n[3] = {k->n[0], k->n[1], k->n[2]};
    int levels = 1;
    while (n[0] % 2 == 0 && n[1] % 2 == 0 && n[2] % 2 == 0 && (max_levels <= 0 || levels < max_levels)) {
        n[0] /= 2;
        n[1] /= 2;
        n[2] /= 2;
        ++levels;
    }
    const int coarse_cells = k->nblocks * n[0] * n[1] * n[2];
    if (coarse_cells > kCoarseMax) {
        delete m;
        return fail(CN_ERR_UNSUPPORTED, "cn_mg_create: coarsest level has more than 4096 cells");
    }
    m->nlevels = levels;
    m->coarse_iters_max = 4 * coarse_cells + 100;
    cn_status s = CN_OK;
    const double b0[3] = {k->begin[0], k->begin[1], k->begin[2]};
    const double e0[3] = {k->end[0], k->end[1], k->end[2]};
    int cells[3] = {k->n[0], k->n[1], k->n[2]};
    for (int l = 0; l < levels && s == CN_OK; ++l) {
        cn_grid *gp = nullptr, *gt = nullptr, *gf = nullptr, *gk = nullptr;
        s = cn_grid_create(k->nb, cells, 1, CN_FLOAT32, b0, e0, &gp);
        if (s == CN_OK) s = cn_grid_create(k->nb, cells, 1, CN_FLOAT32, b0, e0, &gt);
        if (s == CN_OK) s = cn_grid_create(k->nb, cells, 1, CN_FLOAT32, b0, e0, &gf);
        if (s == CN_OK && l > 0) s = cn_grid_create(k->nb, cells, 1, CN_FLOAT32, b0, e0, &gk);
        m->p.push_back(gp);
        m->pt.push_back(gt);
        m->f.push_back(gf);
        m->k.push_back(l == 0 ? k : gk);
        for (int d = 0; d < 3; ++d) cells[d] /= 2;
    }
    if (s == CN_OK) s = cn_grid_create(k->nb, k->n, 1, CN_FLOAT32, b0, e0, &m->r32);
    const int64_t fine = (int64_t)k->nblocks * k->n[0] * k->n[1] * k->n[2];
    m->nparts = (int)grid_for(fine);
    if (s == CN_OK && cudaMalloc(&m->partials, sizeof(double) * 2 * m->nparts) != cudaSuccess)
        s = fail(CN_ERR_OUT_OF_MEMORY, "cn_mg_create: partials");
    if (s == CN_OK && cudaMalloc(&m->sums, sizeof(double) * 2) != cudaSuccess)
        s = fail(CN_ERR_OUT_OF_MEMORY, "cn_mg_create: sums");
    if (s == CN_OK && cudaMalloc(&m->iters, sizeof(int)) != cudaSuccess)
        s = fail(CN_ERR_OUT_OF_MEMORY, "cn_mg_create: iters");
    // coarse coefficients
    for (int l = 1; l < levels && s == CN_OK; ++l) {
        s = sync_bc(m->p[l], nullptr);
        if (s != CN_OK) break;
        s = sync_bc(m->k[l], nullptr);
        const LabGeom Lf = make_geom(m->k[l - 1], &kS1), Lc = make_geom(m->k[l], &kS1);
        const int64_t cc = (int64_t)k->nblocks * Lc.n[0] * Lc.n[1] * Lc.n[2];
        restrict_mean_kernel<<<grid_for(cc), 256>>>(Lf, fptr(m->k[l - 1]), Lc, fptr(m->k[l]), k->nblocks);
        if (cudaGetLastError() != cudaSuccess) s = fail(CN_ERR_CUDA, "restrict_mean_kernel launch");
    }
    if (s == CN_OK) s = sync_bc(m->p[0], nullptr);
    if (s == CN_OK) s = sync_bc(k, nullptr);
    if (s == CN_OK && cudaDeviceSynchronize() != cudaSuccess) s = fail(CN_ERR_CUDA, "cn_mg_create");
    if (s != CN_OK) {
        extern cn_status cn_mg_destroy(cn_mg *);
        cn_mg_destroy(m);
        return s;
    }
    *out = m;
    return CN_OK;
}

cn_status cn_mg_destroy(cn_mg *m)
{
    if (!m) return CN_OK;
    for (int l = 0; l < (int)m->p.size(); ++l) {
        cn_grid_destroy(m->p[l]);
        cn_grid_destroy(m->pt[l]);
        cn_grid_destroy(m->f[l]);
        if (l > 0) cn_grid_destroy(m->k[l]);
    }
    cn_grid_destroy(m->r32);
    for (cn_grid *g : m->nn_bufs) cn_grid_destroy(g);
    for (void *a : m->nn_act)
        if (a) cudaFree(a);
    if (m->partials) cudaFree(m->partials);
    if (m->sums) cudaFree(m->sums);
    if (m->iters) cudaFree(m->iters);
    delete m;
    return CN_OK;
}

cn_status cn_mg_levels(const cn_mg *m, int *nlevels, int *coarsest_cells)
{
    if (!m || !nlevels) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    *nlevels = m->nlevels;
    if (coarsest_cells) {
        const cn_grid *g = m->p[m->nlevels - 1];
        *coarsest_cells = g->nblocks * g->n[0] * g->n[1] * g->n[2];
    }
    return CN_OK;
}

// One V-cycle for L e = rhs from e = 0 (FP32), result in e.
cn_status cn_mg_vcycle(cn_mg *m, const cn_grid *rhs, cn_grid *e, void *stream)
{
    if (!m || !rhs || !e) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    cn_grid *g0 = m->p[0];
    if (rhs->comp_stride != g0->comp_stride || e->comp_stride != g0->comp_stride ||
        rhs->dtype != CN_FLOAT32 || e->dtype != CN_FLOAT32)
        return fail(CN_ERR_SIZE_MISMATCH, "Cartesian: Can not assign two grids of unequal size.");
    cudaStream_t st = as_stream(stream);
    CN_CUDA_TRY(cudaMemcpyAsync(m->f[0]->d_data, rhs->d_data, (size_t)g0->comp_stride * 4,
                                cudaMemcpyDeviceToDevice, st));
    cn_status s = vcycle(m, 0, st);
    if (s != CN_OK) return s;
    CN_CUDA_TRY(cudaMemcpyAsync(e->d_data, m->p[0]->d_data, (size_t)g0->comp_stride * 4,
                                cudaMemcpyDeviceToDevice, st));
    return CN_OK;
}

// FP64 residual r = f - L p64 of the finest level; returns ||r||^2 and ||f||^2
// (waits for the stream).  r32 (optional) receives (float) r.
cn_status cn_mg_residual(cn_mg *m, const cn_grid *p64, const cn_grid *f, cn_grid *r32, double *rr,
                         double *ff, void *stream)
{
    if (!m || !p64 || !f) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    if (p64->dtype != CN_FLOAT64 || f->dtype != CN_FLOAT32 || p64->nblocks != m->p[0]->nblocks ||
        p64->n[0] != m->p[0]->n[0] || f->comp_stride != m->p[0]->comp_stride)
        return fail(CN_ERR_SIZE_MISMATCH, "Cartesian: Can not assign two grids of unequal size.");
    cudaStream_t st = as_stream(stream);
    cn_status s = sync_bc(const_cast<cn_grid *>(p64), st);
    if (s != CN_OK) return s;
    KArgs a = kargs(m, 0);
    a.G.L.bstride = p64->block_stride;
    a.G.bc = bc_view(p64, 0);
    resid64_kernel<<<m->nparts, 256, 0, st>>>(a, reinterpret_cast<const double *>(p64->d_data),
                                               reinterpret_cast<const float *>(f->d_data),
                                               r32 ? fptr(r32) : nullptr, m->partials);
    CN_CUDA_TRY(cudaGetLastError());
    sum_pairs_kernel<<<1, 256, 0, st>>>(m->partials, m->nparts, m->sums);
    CN_CUDA_TRY(cudaGetLastError());
    double h[2];
    CN_CUDA_TRY(cudaMemcpyAsync(h, m->sums, sizeof(h), cudaMemcpyDeviceToHost, st));
    CN_CUDA_TRY(cudaStreamSynchronize(st));
    if (rr) *rr = h[0];
    if (ff) *ff = h[1];
    return CN_OK;
}

// Solve L p = f to ||f - L p|| <= rtol ||f||: p (FP64) is zeroed, then
// each cycle r = f - L p (FP64), e = V-cycle(r) (FP32), p += e.
cn_status cn_mg_solve(cn_mg *m, const cn_grid *f, cn_grid *p64, double rtol, int max_cycles,
                      int *cycles, double *relres, void *stream)
{
    if (!m || !f || !p64) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaStream_t st = as_stream(stream);
    CN_CUDA_TRY(cudaMemsetAsync(p64->d_data, 0, (size_t)p64->comp_stride * 8, st));
    double rr = 0, ff = 0;
    cn_status s = cn_mg_residual(m, p64, f, m->f[0], &rr, &ff, stream);
    if (s != CN_OK) return s;
    const double fn = std::sqrt(ff);
    double rel = fn > 0 ? std::sqrt(rr) / fn : 0.0;
    int c = 0;
    while (c < max_cycles && rel > rtol) {
        s = vcycle(m, 0, st);
        if (s != CN_OK) return s;
        s = cn_mg_accumulate(m, p64, stream);
        if (s != CN_OK) return s;
        s = cn_mg_residual(m, p64, f, m->f[0], &rr, nullptr, stream);
        if (s != CN_OK) return s;
        rel = std::sqrt(rr) / fn;
        ++c;
    }
    if (cycles) *cycles = c;
    if (relres) *relres = rel;
    return CN_OK;
}

// p64 += finest-level correction (the result of the last V-cycle)
cn_status cn_mg_accumulate(cn_mg *m, cn_grid *p64, void *stream)
{
    if (!m || !p64) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    const cn_grid *g = m->p[0];
    if (p64->dtype != CN_FLOAT64 || p64->nblocks != g->nblocks || p64->n[0] != g->n[0] || p64->n[1] != g->n[1] ||
        p64->n[2] != g->n[2])
        return fail(CN_ERR_SIZE_MISMATCH, "Cartesian: Can not assign two grids of unequal size.");
    const int64_t cells = (int64_t)g->n[0] * g->n[1] * g->n[2];
    axpy64_kernel<<<grid_for(cells * g->nblocks), 256, 0, as_stream(stream)>>>(
        reinterpret_cast<double *>(p64->d_data), p64->block_stride, fptr(m->p[0]), g->block_stride, cells, g->nblocks);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

// Single operators on the finest level, for tests: one Jacobi sweep
// pout = pin + omega (L pin - f)/D, and residual-restriction onto level 1.
cn_status cn_mg_jacobi(cn_mg *m, const cn_grid *pin, const cn_grid *f, cn_grid *pout, void *stream)
{
    if (!m || !pin || !f || !pout) return fail(CN_ERR_INVALID_ARGUMENT, "NULL argument");
    KArgs a = kargs(m, 0);
    const int64_t cells = (int64_t)pin->nblocks * pin->n[0] * pin->n[1] * pin->n[2];
    jacobi_kernel<<<grid_for(cells), 256, 0, as_stream(stream)>>>(
        a, reinterpret_cast<const float *>(pin->d_data), reinterpret_cast<const float *>(f->d_data),
        fptr(pout), (float)m->omega);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

cn_status cn_mg_restrict_residual(cn_mg *m, const cn_grid *p, const cn_grid *f, cn_grid *fc, void *stream)
{
    if (!m || !p || !f || !fc || m->nlevels < 2) return fail(CN_ERR_INVALID_ARGUMENT, "bad argument");
    KArgs a = kargs(m, 0);
    const LabGeom Lc = make_geom(fc, &kS1);
    const int64_t cc = (int64_t)fc->nblocks * Lc.n[0] * Lc.n[1] * Lc.n[2];
    resid_restrict_kernel<<<grid_for(cc), 256, 0, as_stream(stream)>>>(
        a, reinterpret_cast<const float *>(p->d_data), reinterpret_cast<const float *>(f->d_data), Lc, fptr(fc));
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

cn_status cn_mg_prolong(cn_mg *m, const cn_grid *ec, cn_grid *p, void *stream)
{
    if (!m || !ec || !p) return fail(CN_ERR_INVALID_ARGUMENT, "bad argument");
    cn_status s = sync_bc(const_cast<cn_grid *>(ec), as_stream(stream));
    if (s != CN_OK) return s;
    const LabGeom Lf = make_geom(p, &kS1), Lct = make_geom(ec, &kS1t);
    const int64_t fc = (int64_t)p->nblocks * Lf.n[0] * Lf.n[1] * Lf.n[2];
    prolong_kernel<<<grid_for(fc), 256, 0, as_stream(stream)>>>(Lf, fptr(p), Lct, bc_view(ec, 0),
                                                                 reinterpret_cast<const float *>(ec->d_data),
                                                                 p->nblocks);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

// Coarse coefficient grid of level l (read-only view for tests).
cn_status cn_mg_level_grid(cn_mg *m, int level, int which, cn_grid **out)
{
    if (!m || !out || level < 0 || level >= m->nlevels) return fail(CN_ERR_INVALID_ARGUMENT, "bad level");
    *out = which == 0 ? m->p[level] : (which == 1 ? m->f[level] : m->k[level]);
    return CN_OK;
}

} // extern "C"
