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
#include "mg_tile.cuh"

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

struct KArgs {
    Geo G;
    BcView kbc;
    const float *k;
    const float *coef; // level coefficients, 8 per cell (see op7_coef)
    float ih2;
    double ih2d;
};

// dense index of tile cell (x, y, z) in its block
__device__ __forceinline__ int64_t dense_cell(const LabGeom &L, const TilePos &q, int x, int y, int z)
{
    return (q.x0 + x) + (int64_t)L.n[0] * ((q.y0 + y) + (int64_t)L.n[1] * (q.z0 + z));
}

// Coefficients of one level (see op7_coef) in precision TC (float for the
// V-cycle; resid64_kernel forms the FP64 means itself with the same
// operations): k staged per tile with its one-cell halo, then per cell the
// operations of op7_math in TC.
template <typename TC>
__global__ void __launch_bounds__(kTileThreads, kTileMinCtas) coef_kernel(const __grid_constant__ KArgs a,
                                                                          const __grid_constant__ Tile T, TC ih2,
                                                                          TC *coef)
{
    __shared__ __align__(16) float sk[kRegionMax];
    __shared__ int snb[27];
    const LabGeom &L = a.G.L;
    TilePos q = tile_pos(T);
    region_layout<float>(q, a.G.Lk);
    neighbour_blocks(L.nb, q.block, snb);
    __syncthreads();
    stage_region<float>(a.k, a.G.Lk, a.kbc, q, false, snb, sk);
    cp_async_wait_all();
    __syncthreads();
    int x, y, z0, zl;
    if (!column_run(T, x, y, z0, zl)) return;
    const int st[3] = {1, q.rs, q.rs * q.ey};
    const int64_t cells = (int64_t)L.n[0] * L.n[1] * L.n[2];
    for (int z = z0; z < z0 + zl; ++z) {
        TC *cv = coef + ((int64_t)q.block * cells + dense_cell(L, q, x, y, z)) * kCoefPerCell;
        const int u = ridx(q, x, y, z);
        const TC kc = (TC)sk[u];
        TC sd[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const TC kp = harm<TC>(kc, (TC)sk[u + st[d]]);
            const TC km = harm<TC>((TC)sk[u - st[d]], kc);
            cv[d] = kp;
            cv[3 + d] = km;
            sd[d] = kp + km;
        }
        cv[6] = ih2 * ((sd[0] + sd[1]) + sd[2]);
        cv[7] = TC(0);
    }
}

// FP64 harmonic face means of the finest level, each face once: per block
// the x faces ((n0 + 1) n1 n2, face i between cells i - 1 and i), then the y
// and z faces, x fastest.  A cell writes its +d faces, and cells on the
// block's lower side also their -d face, with the operations of coef_kernel:
// harm(kc, k(+e_d)) and harm(k(-e_d), kc), which are the same bits since
// harm is symmetric.  Boundary faces use this block's lab of k.
__host__ __device__ inline int64_t face_count(const int n[3])
{
    return (int64_t)(n[0] + 1) * n[1] * n[2] + (int64_t)n[0] * (n[1] + 1) * n[2] + (int64_t)n[0] * n[1] * (n[2] + 1);
}

__device__ __forceinline__ int64_t face_index(const int n[3], int d, int x, int y, int z)
{
    if (d == 0) return x + (int64_t)(n[0] + 1) * (y + (int64_t)n[1] * z);
    const int64_t fx = (int64_t)(n[0] + 1) * n[1] * n[2];
    if (d == 1) return fx + x + (int64_t)n[0] * (y + (int64_t)(n[1] + 1) * z);
    return fx + (int64_t)n[0] * (n[1] + 1) * n[2] + x + (int64_t)n[0] * (y + (int64_t)n[1] * z);
}

__global__ void __launch_bounds__(kTileThreads, kTileMinCtas) face64_kernel(const __grid_constant__ KArgs a,
                                                                            const __grid_constant__ Tile T,
                                                                            double *faces)
{
    __shared__ __align__(16) float sk[kRegionMax];
    __shared__ int snb[27];
    const LabGeom &L = a.G.Lk;
    TilePos q = tile_pos(T);
    region_layout<float>(q, L);
    neighbour_blocks(L.nb, q.block, snb);
    __syncthreads();
    stage_region<float>(a.k, L, a.kbc, q, false, snb, sk);
    cp_async_wait_all();
    __syncthreads();
    int x, y, z0, zl;
    if (!column_run(T, x, y, z0, zl)) return;
    const int st[3] = {1, q.rs, q.rs * q.ey};
    double *fb = faces + (int64_t)q.block * face_count(L.n);
    for (int z = z0; z < z0 + zl; ++z) {
        const int u = ridx(q, x, y, z);
        const double kc = (double)sk[u];
        const int g[3] = {q.x0 + x, q.y0 + y, q.z0 + z};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int ex = d == 0, ey = d == 1, ez = d == 2;
            fb[face_index(L.n, d, g[0] + ex, g[1] + ey, g[2] + ez)] = harm<double>(kc, (double)sk[u + st[d]]);
            if (g[d] == 0)
                fb[face_index(L.n, d, g[0], g[1], g[2])] = harm<double>((double)sk[u - st[d]], kc);
        }
    }
}

// weighted Jacobi sweep: pout = pin + omega (L pin - f) / D  (pin == NULL: zero guess)
__global__ void __launch_bounds__(kTileThreads, kTileMinCtas) jacobi_kernel(const __grid_constant__ KArgs a,
                                                              const __grid_constant__ Tile T, const float *pin,
                                                              const float *f, float *pout, float omega)
{
    __shared__ __align__(16) float sp[kRegionMax];
    __shared__ int snb[27];
    const LabGeom &L = a.G.L;
    TilePos q = tile_pos(T);
    region_layout<float>(q, L);
    if (pin) {
        neighbour_blocks(L.nb, q.block, snb);
        __syncthreads();
        stage_region<float>(pin, L, a.G.bc, q, false, snb, sp);
        cp_async_wait_all();
        __syncthreads();
    }
    int x, y, z0, zl;
    if (!column_run(T, x, y, z0, zl)) return;
    const int st[3] = {1, q.rs, q.rs * q.ey};
    const int64_t cells = (int64_t)L.n[0] * L.n[1] * L.n[2];
    const int64_t oz = (int64_t)L.n[0] * L.n[1];
    int64_t c = dense_cell(L, q, x, y, z0);
    int u = ridx(q, x, y, z0);
    const float4 *cv = reinterpret_cast<const float4 *>(a.coef + ((int64_t)q.block * cells + c) * kCoefPerCell);
    const int64_t cvz = oz * kCoefPerCell / 4;
    int64_t o = (int64_t)q.block * L.bstride + c;
    // the next cell's loads go out before this cell's store
    float4 ca = __ldg(cv), cb = __ldg(cv + 1);
    float fc = __ldg(f + o);
    for (int k = 0; k < zl; ++k, u += st[2]) {
        float4 na = ca, nb = cb;
        float nf = fc;
        if (k + 1 < zl) {
            na = __ldg(cv + cvz);
            nb = __ldg(cv + cvz + 1);
            nf = __ldg(f + o + oz);
        }
        if (pin) {
            const float cc[8] = {ca.x, ca.y, ca.z, ca.w, cb.x, cb.y, cb.z, cb.w};
            const float pc = sp[u];
            float fl[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const float kp = cc[d], km = cc[3 + d];
                fl[d] = kp * (sp[u + st[d]] - pc) - km * (pc - sp[u - st[d]]);
            }
            const float Lp = a.ih2 * ((fl[0] + fl[1]) + fl[2]);
            pout[o] = pc + omega * ((Lp - fc) / cb.z);
        } else {
            pout[o] = 0.0f + omega * ((0.0f - fc) / cb.z);
        }
        ca = na;
        cb = nb;
        fc = nf;
        cv += cvz;
        o += oz;
    }
}

// residual of the fine level restricted onto the coarse right-hand side:
// fc = (sum of its 8 children's f - L p) / 8, children summed in the order
// ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)), child c = dx | dy<<1 | dz<<2.
// Compiled for 4 CTAs per SM (64 registers): at the tile kernels' 6 it
// spills 188 bytes per thread and the solve takes 1 % longer.
__global__ void __launch_bounds__(kTileThreads, 4) resid_restrict_kernel(const __grid_constant__ KArgs a,
                                                                      const __grid_constant__ Tile T,
                                                                      const float *p, const float *f,
                                                                      const __grid_constant__ LabGeom Lc, float *fc)
{
    __shared__ __align__(16) float sp[kRegionMax];
    __shared__ float sr[32 * 8 * 4];
    __shared__ int snb[27];
    const LabGeom &L = a.G.L;
    TilePos q = tile_pos(T);
    region_layout<float>(q, L);
    neighbour_blocks(L.nb, q.block, snb);
    __syncthreads();
    stage_region<float>(p, L, a.G.bc, q, false, snb, sp);
    cp_async_wait_all();
    __syncthreads();
    {
        int x, y, z0, zl;
        if (column_run(T, x, y, z0, zl)) {
            const int st[3] = {1, q.rs, q.rs * q.ey};
            const int64_t cells = (int64_t)L.n[0] * L.n[1] * L.n[2];
            const int64_t oz = (int64_t)L.n[0] * L.n[1];
            int64_t c = dense_cell(L, q, x, y, z0);
            int u = ridx(q, x, y, z0);
            int ct = x + T.t[0] * (y + T.t[1] * z0);
            for (int k = 0; k < zl; ++k, c += oz, u += st[2], ct += T.t[0] * T.t[1]) {
                float Lp, D, pc;
                op7_coef<float, float>(sp, u, st, a.coef + ((int64_t)q.block * cells + c) * kCoefPerCell, a.ih2, Lp,
                                       D, pc);
                sr[ct] = __ldg(f + (int64_t)q.block * L.bstride + c) - Lp;
            }
        }
    }
    __syncthreads();
    const int hx = T.t[0] / 2, hy = T.t[1] / 2, hz = T.t[2] / 2;
    for (int c = threadIdx.x; c < hx * hy * hz; c += kTileThreads) {
        const int X = c % hx, Y = (c / hx) % hy, Z = c / (hx * hy);
        float r[8];
#pragma unroll
        for (int ch = 0; ch < 8; ++ch) {
            const int x = 2 * X + (ch & 1), y = 2 * Y + ((ch >> 1) & 1), z = 2 * Z + (ch >> 2);
            r[ch] = sr[x + T.t[0] * (y + T.t[1] * z)];
        }
        const float s = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        const int gx = q.x0 / 2 + X, gy = q.y0 / 2 + Y, gz = q.z0 / 2 + Z;
        fc[(int64_t)q.block * Lc.bstride + gx + (int64_t)Lc.n[0] * (gy + (int64_t)Lc.n[1] * gz)] = s * 0.125f;
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

// p_fine += trilinear interpolation of the coarse correction e: the fine
// tile's coarse cells plus a one-cell halo (edges and corners included) are
// staged, then each fine cell combines its 8 coarse values.
__global__ void __launch_bounds__(kTileThreads, kTileMinCtas) prolong_kernel(const __grid_constant__ LabGeom L,
                                                               const __grid_constant__ Tile T, float *p,
                                                               const __grid_constant__ LabGeom Lct,
                                                               const __grid_constant__ BcView cbc, const float *e)
{
    __shared__ __align__(16) float se[(16 + 8) * (4 + 2) * (2 + 2)];
    __shared__ int snb[27];
    const TilePos qf = tile_pos(T);
    neighbour_blocks(Lct.nb, qf.block, snb);
    __syncthreads();
    TilePos qc = qf;
    qc.x0 = qf.x0 / 2;
    qc.y0 = qf.y0 / 2;
    qc.z0 = qf.z0 / 2;
    qc.ex = T.t[0] / 2 + 2;
    qc.ey = T.t[1] / 2 + 2;
    qc.ez = T.t[2] / 2 + 2;
    qc.xo = 1;
    qc.rs = qc.ex;
    region_layout<float>(qc, Lct);
    stage_region<float>(e, Lct, cbc, qc, true, snb, se);
    cp_async_wait_all();
    __syncthreads();
    const int cells = T.t[0] * T.t[1] * T.t[2];
    for (int c = threadIdx.x; c < cells; c += kTileThreads) {
        int x, y, z;
        tile_cell(T, c, x, y, z);
        const int X = x >> 1, Y = y >> 1, Z = z >> 1;
        const int sx = (x & 1) ? 1 : -1, sy = (y & 1) ? 1 : -1, sz = (z & 1) ? 1 : -1;
        const int u = ridx(qc, X, Y, Z);
        const int ox = sx, oy = sy * qc.rs, oz = sz * qc.rs * qc.ey;
        const float v0 = se[u], v1 = se[u + ox], v2 = se[u + oy], v3 = se[u + ox + oy];
        const float v4 = se[u + oz], v5 = se[u + ox + oz], v6 = se[u + oy + oz], v7 = se[u + ox + oy + oz];
        const float a0 = 0.75f * v0 + 0.25f * v1;
        const float a1 = 0.75f * v2 + 0.25f * v3;
        const float a2 = 0.75f * v4 + 0.25f * v5;
        const float a3 = 0.75f * v6 + 0.25f * v7;
        const float b0 = 0.75f * a0 + 0.25f * a1;
        const float b1 = 0.75f * a2 + 0.25f * a3;
        const float val = 0.75f * b0 + 0.25f * b1;
        const int64_t o = (int64_t)qf.block * L.bstride + (qf.x0 + x) + (int64_t)L.n[0] * ((qf.y0 + y) + (int64_t)L.n[1] * (qf.z0 + z));
        p[o] = p[o] + val;
    }
}

// FP64 residual of the outer iteration: r = f - L p64, r32 = (float) r,
// per-CTA FP64 partial sums of r^2 and f^2.  The tile's p64 is staged with
// its one-cell halo; the six face means of a cell come from the FP64 face
// arrays (face64_kernel) and are applied in op7_coef's order, so L p64 is
// bit for bit the operator of the per-cell coefficients.
__global__ void __launch_bounds__(kTileThreads, 4) resid64_kernel(const __grid_constant__ KArgs a,
                                                               const __grid_constant__ Tile T, const double *p64,
                                                               const float *f, float *r32, double *partials,
                                                               const double *faces)
{
    __shared__ __align__(16) double sp[kRegionMax];
    __shared__ double sh[2][kTileThreads / 32];
    __shared__ int snb[27];
    const LabGeom &L = a.G.L, &Lk = a.G.Lk;
    TilePos q = tile_pos(T);
    region_layout<double>(q, L);
    neighbour_blocks(L.nb, q.block, snb);
    __syncthreads();
    stage_region<double>(p64, L, a.G.bc, q, false, snb, sp);
    cp_async_wait_all();
    __syncthreads();
    double rr = 0, ff = 0;
    int x, y, z0, zl;
    if (column_run(T, x, y, z0, zl)) {
        const int st[3] = {1, q.rs, q.rs * q.ey};
        const double *fb = faces + (int64_t)q.block * face_count(Lk.n);
        // the six face indices of the column's first cell; along z they
        // advance by each face array's plane size, and the next cell's
        // loads go out before this cell's arithmetic
        const int gx = q.x0 + x, gy = q.y0 + y, gz = q.z0 + z0;
        const int64_t dz[3] = {(int64_t)(Lk.n[0] + 1) * Lk.n[1], (int64_t)Lk.n[0] * (Lk.n[1] + 1),
                               (int64_t)Lk.n[0] * Lk.n[1]};
        int64_t im[3], ip[3];
        im[0] = face_index(Lk.n, 0, gx, gy, gz);
        ip[0] = im[0] + 1;
        im[1] = face_index(Lk.n, 1, gx, gy, gz);
        ip[1] = im[1] + Lk.n[0];
        im[2] = face_index(Lk.n, 2, gx, gy, gz);
        ip[2] = im[2] + dz[2];
        int64_t o = (int64_t)q.block * Lk.bstride + dense_cell(Lk, q, x, y, z0); // FP32 fields (f, r32)
        const int64_t oz = (int64_t)Lk.n[0] * Lk.n[1];
        double km[3], kp[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            km[d] = __ldg(fb + im[d]);
            kp[d] = __ldg(fb + ip[d]);
        }
        float fcf = __ldg(f + o);
        int u = ridx(q, x, y, z0);
        for (int k = 0; k < zl; ++k, u += st[2], o += oz) {
            double nkm[3], nkp[3];
            float nf = fcf;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                nkm[d] = km[d];
                nkp[d] = kp[d];
            }
            if (k + 1 < zl) {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    im[d] += dz[d];
                    ip[d] += dz[d];
                    nkm[d] = __ldg(fb + im[d]);
                    nkp[d] = __ldg(fb + ip[d]);
                }
                nf = __ldg(f + o + oz);
            }
            const double pc = sp[u];
            double fd[3];
#pragma unroll
            for (int d = 0; d < 3; ++d)
                fd[d] = kp[d] * (sp[u + st[d]] - pc) - km[d] * (pc - sp[u - st[d]]);
            const double Lp = a.ih2d * ((fd[0] + fd[1]) + fd[2]);
            const double fc = (double)fcf;
            const double r = fc - Lp;
            if (r32) r32[o] = (float)r;
            rr += r * r;
            ff += fc * fc;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                km[d] = nkm[d];
                kp[d] = nkp[d];
            }
            fcf = nf;
        }
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
        for (int i = 0; i < kTileThreads / 32; ++i) {
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

// Coarsest levels of at most kCoarseDenseMax cells are solved directly: the
// operator A = -L (harmonic face means, as coarsest_cg_kernel applies it) is
// singular on the periodic grid with the constants as null space, so the
// set-up inverts A' = A + (s/N) 1 1^T (s: the mean diagonal), which is SPD
// and maps every mean-zero b to the mean-zero solution of A x = b.  Per
// V-cycle this kernel forms b = -f with its mean removed, as the CG does,
// and x = A'^-1 b: each CTA takes 32 rows (one per lane), its 8 warps split
// the columns, and the symmetric inverse is read column-wise (coalesced).
constexpr int kCoarseDenseMax = 512;
constexpr int kDenseRows = 32, kDenseThreads = 256;

__global__ void __launch_bounds__(kDenseThreads)
    coarsest_dense_kernel(LabGeom L, const float *f, float *p, const double *inv, int N)
{
    __shared__ double b[kCoarseDenseMax];
    __shared__ double red[kDenseThreads / 32][kDenseRows];
    __shared__ double wsum[kDenseThreads / 32];
    const int GX = L.nb[0] * L.n[0], GY = L.nb[1] * L.n[1];
    auto offset = [&](int i) {
        const int gx = i % GX, gy = (i / GX) % GY, gz = i / (GX * GY);
        const int bx = gx / L.n[0], by = gy / L.n[1], bz = gz / L.n[2];
        const int blk = bx + L.nb[0] * (by + L.nb[1] * bz);
        return (int64_t)blk * L.bstride + (gx % L.n[0]) +
               (int64_t)L.n[0] * ((gy % L.n[1]) + (int64_t)L.n[1] * (gz % L.n[2]));
    };
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double s = 0;
    for (int i = threadIdx.x; i < N; i += kDenseThreads) {
        b[i] = -(double)f[offset(i)];
        s += b[i];
    }
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (lane == 0) wsum[warp] = s;
    __syncthreads();
    double tot = 0;
    for (int w = 0; w < kDenseThreads / 32; ++w) tot += wsum[w];
    const double mean = tot / N;
    for (int i = threadIdx.x; i < N; i += kDenseThreads) b[i] -= mean;
    __syncthreads();
    const int row = blockIdx.x * kDenseRows + lane;
    const int per = (N + kDenseThreads / 32 - 1) / (kDenseThreads / 32);
    const int j0 = warp * per, j1 = min(N, j0 + per);
    double acc = 0;
    if (row < N)
        for (int j = j0; j < j1; ++j) acc += inv[(int64_t)j * N + row] * b[j];
    red[warp][lane] = acc;
    __syncthreads();
    if (warp == 0 && row < N) {
        double x = 0;
        for (int w = 0; w < kDenseThreads / 32; ++w) x += red[w][lane];
        p[offset(row)] = (float)x;
    }
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
    a.coef = (int)m->coef.size() > l ? m->coef[l] : nullptr;
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
    const Tile T = tile_of(m->p[l]->n);
    for (int s = 0; s < sweeps; ++s) {
        const bool zg = zero_guess && s == 0;
        // ping-pong so that the result of the last sweep lands in p
        float *src = fptr(m->p[l]), *dst = fptr(m->pt[l]);
        jacobi_kernel<<<(unsigned)(m->p[l]->nblocks * T.count), kTileThreads, 0, st>>>(
            a, T, zg ? nullptr : src, fptr(m->f[l]), dst, (float)m->omega);
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
    if (m->coarse_inv) {
        const LabGeom L = make_geom(g, &kS1);
        coarsest_dense_kernel<<<(unsigned)((m->coarse_n + kDenseRows - 1) / kDenseRows), kDenseThreads, 0, st>>>(
            L, fptr(m->f[l]), fptr(g), m->coarse_inv, m->coarse_n);
        CN_CUDA_TRY(cudaGetLastError());
        return CN_OK;
    }
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


// pre-smoothing (post = false, from a zero guess) or post-smoothing of level
// l: the learned smoother where its level masks select it, else Jacobi
static cn_status smooth_any(cn_mg *m, int l, bool post, cudaStream_t st)
{
    const int sweeps = post ? m->nu2 : m->nu1;
    const unsigned mask = post ? m->nn_post_levels : m->nn_levels;
    if (m->nn && ((mask >> l) & 1)) {
        const int apps = post ? m->nn_post_apps : m->nn_pre_apps;
        return nn_smooth(m, l, apps >= 0 ? apps : sweeps, !post, st);
    }
    return smooth(m, l, sweeps, !post, st);
}

cn_status vcycle(cn_mg *m, int l, cudaStream_t st)
{
    if (l == m->nlevels - 1) return coarsest(m, l, st);
    cn_status s = smooth_any(m, l, false, st);
    if (s != CN_OK) return s;
    KArgs a = kargs(m, l);
    const LabGeom Lc = make_geom(m->p[l + 1], &kS1);
    const Tile T = tile_of(m->p[l]->n);
    resid_restrict_kernel<<<(unsigned)(m->p[l]->nblocks * T.count), kTileThreads, 0, st>>>(
        a, T, fptr(m->p[l]), fptr(m->f[l]), Lc, fptr(m->f[l + 1]));
    CN_CUDA_TRY(cudaGetLastError());
    s = vcycle(m, l + 1, st);
    if (s != CN_OK) return s;
    const LabGeom Lf = make_geom(m->p[l], &kS1);
    const LabGeom Lct = make_geom(m->p[l + 1], &kS1t);
    prolong_kernel<<<(unsigned)(m->p[l]->nblocks * T.count), kTileThreads, 0, st>>>(
        Lf, T, fptr(m->p[l]), Lct, bc_view(m->p[l + 1], 0), fptr(m->p[l + 1]));
    CN_CUDA_TRY(cudaGetLastError());
    if (l == 0 && m->capture) {
        s = m->capture(m, st);
        if (s != CN_OK) return s;
    }
    return smooth_any(m, l, true, st);
}

// Inverse of the regularised coarsest operator (see coarsest_dense_kernel),
// built on the host in FP64 from the coarsest level's k: Cholesky A' = C C^T,
// C^-1 by forward substitution, A'^-1 = C^-T C^-1.
static cn_status coarse_inverse(cn_mg *m)
{
    const int l = m->nlevels - 1;
    const cn_grid *g = m->p[l];
    const int GX = g->nb[0] * g->n[0], GY = g->nb[1] * g->n[1], GZ = g->nb[2] * g->n[2];
    const int N = GX * GY * GZ;
    std::vector<float> kb((size_t)m->k[l]->comp_stride);
    CN_CUDA_TRY(cudaMemcpy(kb.data(), m->k[l]->d_data, kb.size() * sizeof(float), cudaMemcpyDeviceToHost));
    std::vector<double> kk(N);
    for (int i = 0; i < N; ++i) {
        const int gx = i % GX, gy = (i / GX) % GY, gz = i / (GX * GY);
        const int blk = gx / g->n[0] + g->nb[0] * (gy / g->n[1] + g->nb[1] * (gz / g->n[2]));
        kk[i] = (double)kb[(size_t)blk * m->k[l]->block_stride + (gx % g->n[0]) +
                           (size_t)g->n[0] * ((gy % g->n[1]) + (size_t)g->n[1] * (gz % g->n[2]))];
    }
    const double ih2 = 1.0 / (g->h[0] * g->h[0]);
    std::vector<double> A((size_t)N * N, 0.0);
    for (int i = 0; i < N; ++i) {
        const int gx = i % GX, gy = (i / GX) % GY, gz = i / (GX * GY);
        const int nbr[6] = {((gx + 1) % GX) + GX * (gy + GY * gz), ((gx + GX - 1) % GX) + GX * (gy + GY * gz),
                            gx + GX * (((gy + 1) % GY) + GY * gz), gx + GX * (((gy + GY - 1) % GY) + GY * gz),
                            gx + GX * (gy + GY * ((gz + 1) % GZ)), gx + GX * (gy + GY * ((gz + GZ - 1) % GZ))};
        for (int q = 0; q < 6; ++q) {
            const double t = kk[i] * kk[nbr[q]];
            const double kf = ih2 * ((t + t) / (kk[i] + kk[nbr[q]]));
            A[(size_t)i * N + i] += kf;
            A[(size_t)i * N + nbr[q]] -= kf;
        }
    }
    double sd = 0;
    for (int i = 0; i < N; ++i) sd += A[(size_t)i * N + i];
    if (!(sd > 0)) return CN_OK; // a one-cell level: the CG keeps it (x = 0)
    const double reg = sd / N / N;
    for (size_t e = 0; e < A.size(); ++e) A[e] += reg;
    // Cholesky, lower factor in A
    for (int j = 0; j < N; ++j) {
        double d = A[(size_t)j * N + j];
        for (int q = 0; q < j; ++q) d -= A[(size_t)j * N + q] * A[(size_t)j * N + q];
        if (!(d > 0)) return CN_OK; // not numerically definite: the CG keeps the level
        const double c = std::sqrt(d);
        A[(size_t)j * N + j] = c;
        for (int i = j + 1; i < N; ++i) {
            double v = A[(size_t)i * N + j];
            for (int q = 0; q < j; ++q) v -= A[(size_t)i * N + q] * A[(size_t)j * N + q];
            A[(size_t)i * N + j] = v / c;
        }
    }
    // Ci = C^-1 (lower), column by column
    std::vector<double> Ci((size_t)N * N, 0.0);
    for (int c = 0; c < N; ++c) {
        Ci[(size_t)c * N + c] = 1.0 / A[(size_t)c * N + c];
        for (int i = c + 1; i < N; ++i) {
            double v = 0;
            for (int q = c; q < i; ++q) v -= A[(size_t)i * N + q] * Ci[(size_t)q * N + c];
            Ci[(size_t)i * N + c] = v / A[(size_t)i * N + i];
        }
    }
    // inverse = Ci^T Ci (symmetric)
    std::vector<double> inv((size_t)N * N, 0.0);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j <= i; ++j) {
            double v = 0;
            for (int q = i; q < N; ++q) v += Ci[(size_t)q * N + i] * Ci[(size_t)q * N + j];
            inv[(size_t)i * N + j] = v;
            inv[(size_t)j * N + i] = v;
        }
    if (cudaMalloc(&m->coarse_inv, inv.size() * sizeof(double)) != cudaSuccess)
        return fail(CN_ERR_OUT_OF_MEMORY, "cn_mg_create: coarsest inverse");
    CN_CUDA_TRY(cudaMemcpy(m->coarse_inv, inv.data(), inv.size() * sizeof(double), cudaMemcpyHostToDevice));
    m->coarse_n = N;
    return CN_OK;
}

extern "C" {

cn_status cn_mg_create(cn_grid *k, int nu1, int nu2, double omega, int max_levels, cn_mg **out)
{
    if (!k || !out) return fail(CN_ERR_INVALID_ARGUMENT, "cn_mg_create: NULL argument");
    *out = nullptr;
    if (k->dtype != CN_FLOAT32 || k->ncomp < 1)
        return fail(CN_ERR_UNSUPPORTED, "cn_mg_create: the coefficient grid must be FLOAT32");
    if (k->entity != CN_ENTITY_CELL)
        return fail(CN_ERR_UNSUPPORTED, "cn_mg_create: cell-centred grids only");
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
    m->nparts = k->nblocks * tile_of(k->n).count;
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
    // operator coefficients of every level (k is fixed from here on): 8 FP32
    // values per cell for the V-cycle, FP64 face means of the finest level for
    // the outer residual
    for (int l = 0; l < levels && s == CN_OK; ++l) {
        const int64_t cells = (int64_t)k->nblocks * m->p[l]->n[0] * m->p[l]->n[1] * m->p[l]->n[2];
        float *c = nullptr;
        if (cudaMalloc(&c, sizeof(float) * kCoefPerCell * cells) != cudaSuccess) {
            s = fail(CN_ERR_OUT_OF_MEMORY, "cn_mg_create: coefficients");
            break;
        }
        m->coef.push_back(c);
        const KArgs a = kargs(m, l);
        const Tile T = tile_of(m->p[l]->n);
        coef_kernel<float><<<(unsigned)(m->p[l]->nblocks * T.count), kTileThreads>>>(a, T, a.ih2, c);
        if (cudaGetLastError() != cudaSuccess) s = fail(CN_ERR_CUDA, "coef_kernel launch");
    }
    if (s == CN_OK) {
        if (cudaMalloc(&m->face64, sizeof(double) * face_count(k->n) * k->nblocks) != cudaSuccess) {
            s = fail(CN_ERR_OUT_OF_MEMORY, "cn_mg_create: face means");
        } else {
            const KArgs a = kargs(m, 0);
            const Tile T = tile_of(k->n);
            face64_kernel<<<(unsigned)(k->nblocks * T.count), kTileThreads>>>(a, T, m->face64);
            if (cudaGetLastError() != cudaSuccess) s = fail(CN_ERR_CUDA, "face64_kernel launch");
        }
    }
    if (s == CN_OK && cudaDeviceSynchronize() != cudaSuccess) s = fail(CN_ERR_CUDA, "cn_mg_create");
    if (s == CN_OK && coarse_cells <= kCoarseDenseMax) s = coarse_inverse(m);
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
    if (m->face64) cudaFree(m->face64);
    for (float *c : m->coef)
        if (c) cudaFree(c);
    if (m->coarse_inv) cudaFree(m->coarse_inv);
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
    resid64_kernel<<<m->nparts, kTileThreads, 0, st>>>(
        a, tile_of(p64->n), reinterpret_cast<const double *>(p64->d_data), reinterpret_cast<const float *>(f->d_data),
        r32 ? fptr(r32) : nullptr, m->partials, m->face64);
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
    // the learned smoother's tensor-core layers record bounded-wait failures
    // in the level grids' error words (cn_mg_residual has synchronised)
    for (int l = 0; l < m->nlevels; ++l)
        if ((s = grid_check_error(m->p[l])) != CN_OK) return s;
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
    const Tile T = tile_of(pin->n);
    jacobi_kernel<<<(unsigned)(pin->nblocks * T.count), kTileThreads, 0, as_stream(stream)>>>(
        a, T, reinterpret_cast<const float *>(pin->d_data), reinterpret_cast<const float *>(f->d_data),
        fptr(pout), (float)m->omega);
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

cn_status cn_mg_restrict_residual(cn_mg *m, const cn_grid *p, const cn_grid *f, cn_grid *fc, void *stream)
{
    if (!m || !p || !f || !fc || m->nlevels < 2) return fail(CN_ERR_INVALID_ARGUMENT, "bad argument");
    KArgs a = kargs(m, 0);
    const LabGeom Lc = make_geom(fc, &kS1);
    const Tile T = tile_of(p->n);
    resid_restrict_kernel<<<(unsigned)(p->nblocks * T.count), kTileThreads, 0, as_stream(stream)>>>(
        a, T, reinterpret_cast<const float *>(p->d_data), reinterpret_cast<const float *>(f->d_data), Lc, fptr(fc));
    CN_CUDA_TRY(cudaGetLastError());
    return CN_OK;
}

cn_status cn_mg_prolong(cn_mg *m, const cn_grid *ec, cn_grid *p, void *stream)
{
    if (!m || !ec || !p) return fail(CN_ERR_INVALID_ARGUMENT, "bad argument");
    cn_status s = sync_bc(const_cast<cn_grid *>(ec), as_stream(stream));
    if (s != CN_OK) return s;
    const LabGeom Lf = make_geom(p, &kS1), Lct = make_geom(ec, &kS1t);
    const Tile T = tile_of(p->n);
    prolong_kernel<<<(unsigned)(p->nblocks * T.count), kTileThreads, 0, as_stream(stream)>>>(
        Lf, T, fptr(p), Lct, bc_view(ec, 0), reinterpret_cast<const float *>(ec->d_data));
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
