/*
 * cn_mg.c -- CPU oracle of the multigrid operators for div(k grad p) = f on a
 * periodic block grid (no BCs), TEST INFRASTRUCTURE ONLY.
 *
 * The reference announces multigrid solvers (README.rst:43-44) but has none;
 * this restates the standard cell-centred geometric multigrid method in the
 * operation order of the device kernels (compiled without contraction):
 *   kf(a,b) = (a*b + a*b)/(a+b)  harmonic face coefficient
 *   L p     = ih2*((fx + fy) + fz),  f_d = kf+ (p+ - p) - kf- (p - p-)
 *   D       = ih2*(((kx+ + kx-) + (ky+ + ky-)) + (kz+ + kz-))
 *   Jacobi  p' = p + omega*((L p - f)/D)
 *   restrict (((r0+r1)+(r2+r3)) + ((r4+r5)+(r6+r7))) * 0.125, children
 *           c = (x&1) | (y&1)<<1 | (z&1)<<2
 *   prolong trilinear, x then y then z, weights 0.75/0.25
 * Neighbours wrap periodically over the whole grid (the lab of a periodic
 * grid without BCs).
 */
#include "cn_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int nb[3], n[3];
    int64_t stride;
} mgeo;

static int64_t moff(const mgeo *g, int gx, int gy, int gz)
{
    const int GX = g->nb[0] * g->n[0], GY = g->nb[1] * g->n[1], GZ = g->nb[2] * g->n[2];
    gx = (gx % GX + GX) % GX;
    gy = (gy % GY + GY) % GY;
    gz = (gz % GZ + GZ) % GZ;
    const int b = gx / g->n[0] + g->nb[0] * (gy / g->n[1] + g->nb[1] * (gz / g->n[2]));
    return (int64_t)b * g->stride + gx % g->n[0] +
           (int64_t)g->n[0] * (gy % g->n[1] + (int64_t)g->n[1] * (gz % g->n[2]));
}

static float harmf(float a, float b)
{
    const float t = a * b;
    return (t + t) / (a + b);
}

static double harmd(double a, double b)
{
    const double t = a * b;
    return (t + t) / (a + b);
}

static void op7f(const mgeo *g, const float *p, const float *k, int x, int y, int z, float ih2,
                 float *Lp, float *D, float *pc)
{
    *pc = p[moff(g, x, y, z)];
    const float kc = k[moff(g, x, y, z)];
    float f[3], s[3];
    for (int d = 0; d < 3; ++d) {
        const int ox = d == 0, oy = d == 1, oz = d == 2;
        const float pp = p[moff(g, x + ox, y + oy, z + oz)];
        const float pm = p[moff(g, x - ox, y - oy, z - oz)];
        const float kp = harmf(kc, k[moff(g, x + ox, y + oy, z + oz)]);
        const float km = harmf(k[moff(g, x - ox, y - oy, z - oz)], kc);
        f[d] = kp * (pp - *pc) - km * (*pc - pm);
        s[d] = kp + km;
    }
    *Lp = ih2 * ((f[0] + f[1]) + f[2]);
    *D = ih2 * ((s[0] + s[1]) + s[2]);
}

#define FOR_CELLS(g)                                                           \
    for (int gz = 0; gz < (g)->nb[2] * (g)->n[2]; ++gz)                        \
        for (int gy = 0; gy < (g)->nb[1] * (g)->n[1]; ++gy)                    \
            for (int gx = 0; gx < (g)->nb[0] * (g)->n[0]; ++gx)

static mgeo mk(const int nb[3], const int n[3], int64_t stride)
{
    mgeo g;
    for (int d = 0; d < 3; ++d) {
        g.nb[d] = nb[d];
        g.n[d] = n[d];
    }
    g.stride = stride;
    return g;
}

void or_mg_jacobi(const int nb[3], const int n[3], int64_t stride, const float *pin,
                  const float *k, const float *f, float omega, float ih2, float *pout)
{
    const mgeo g = mk(nb, n, stride);
    /* cells are independent: every thread writes its own */
#pragma omp parallel for
    FOR_CELLS(&g)
    {
        const int64_t o = moff(&g, gx, gy, gz);
        float Lp, D, pc;
        if (pin) {
            op7f(&g, pin, k, gx, gy, gz, ih2, &Lp, &D, &pc);
            pout[o] = pc + omega * ((Lp - f[o]) / D);
        } else {
            const float kc = k[o];
            float s[3];
            for (int d = 0; d < 3; ++d) {
                const int ox = d == 0, oy = d == 1, oz = d == 2;
                const float kp = harmf(kc, k[moff(&g, gx + ox, gy + oy, gz + oz)]);
                const float km = harmf(k[moff(&g, gx - ox, gy - oy, gz - oz)], kc);
                s[d] = kp + km;
            }
            D = ih2 * ((s[0] + s[1]) + s[2]);
            pout[o] = 0.0f + omega * ((0.0f - f[o]) / D);
        }
    }
}

void or_mg_resid_restrict(const int nb[3], const int n[3], int64_t stride, const float *p,
                          const float *k, const float *f, float ih2, int64_t cstride, float *fc)
{
    const mgeo g = mk(nb, n, stride);
    const int nc[3] = {n[0] / 2, n[1] / 2, n[2] / 2};
    const mgeo gc = mk(nb, nc, cstride);
    /* cells are independent: every thread writes its own */
#pragma omp parallel for
    FOR_CELLS(&gc)
    {
        float r[8];
        for (int c = 0; c < 8; ++c) {
            const int x = 2 * gx + (c & 1), y = 2 * gy + ((c >> 1) & 1), z = 2 * gz + (c >> 2);
            float Lp, D, pc;
            op7f(&g, p, k, x, y, z, ih2, &Lp, &D, &pc);
            r[c] = f[moff(&g, x, y, z)] - Lp;
        }
        const float s = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        fc[moff(&gc, gx, gy, gz)] = s * 0.125f;
    }
}

void or_mg_restrict_mean(const int nb[3], const int n[3], int64_t stride, const float *kf,
                         int64_t cstride, float *kc)
{
    const mgeo g = mk(nb, n, stride);
    const int nc[3] = {n[0] / 2, n[1] / 2, n[2] / 2};
    const mgeo gc = mk(nb, nc, cstride);
    /* cells are independent: every thread writes its own */
#pragma omp parallel for
    FOR_CELLS(&gc)
    {
        float v[8];
        for (int c = 0; c < 8; ++c) {
            const int x = 2 * gx + (c & 1), y = 2 * gy + ((c >> 1) & 1), z = 2 * gz + (c >> 2);
            v[c] = kf[moff(&g, x, y, z)];
        }
        const float s = ((v[0] + v[1]) + (v[2] + v[3])) + ((v[4] + v[5]) + (v[6] + v[7]));
        kc[moff(&gc, gx, gy, gz)] = s * 0.125f;
    }
}

void or_mg_prolong(const int nb[3], const int n[3], int64_t stride, float *p, int64_t cstride,
                   const float *e)
{
    const mgeo g = mk(nb, n, stride);
    const int nc[3] = {n[0] / 2, n[1] / 2, n[2] / 2};
    const mgeo gc = mk(nb, nc, cstride);
    /* cells are independent: every thread writes its own */
#pragma omp parallel for
    FOR_CELLS(&g)
    {
        const int X = gx >> 1, Y = gy >> 1, Z = gz >> 1;
        const int sx = (gx & 1) ? 1 : -1, sy = (gy & 1) ? 1 : -1, sz = (gz & 1) ? 1 : -1;
        const float e000 = e[moff(&gc, X, Y, Z)], e100 = e[moff(&gc, X + sx, Y, Z)];
        const float e010 = e[moff(&gc, X, Y + sy, Z)], e110 = e[moff(&gc, X + sx, Y + sy, Z)];
        const float e001 = e[moff(&gc, X, Y, Z + sz)], e101 = e[moff(&gc, X + sx, Y, Z + sz)];
        const float e011 = e[moff(&gc, X, Y + sy, Z + sz)], e111 = e[moff(&gc, X + sx, Y + sy, Z + sz)];
        const float a0 = 0.75f * e000 + 0.25f * e100;
        const float a1 = 0.75f * e010 + 0.25f * e110;
        const float a2 = 0.75f * e001 + 0.25f * e101;
        const float a3 = 0.75f * e011 + 0.25f * e111;
        const float b0 = 0.75f * a0 + 0.25f * a1;
        const float b1 = 0.75f * a2 + 0.25f * a3;
        const float v = 0.75f * b0 + 0.25f * b1;
        const int64_t o = moff(&g, gx, gy, gz);
        p[o] = p[o] + v;
    }
}

/* r = f - L p64 in FP64; r32 = (float) r; returns sum r^2 and sum f^2 */
void or_mg_resid64(const int nb[3], const int n[3], int64_t stride64, const double *p,
                   int64_t stride32, const float *k, const float *f, double ih2, float *r32,
                   double *rr, double *ff)
{
    const mgeo gp = mk(nb, n, stride64), gk = mk(nb, n, stride32);
    /* per z-plane partial sums, added in plane order: the same result for
     * any number of threads */
    const int GZ = nb[2] * n[2];
    double *prr = (double *)calloc((size_t)GZ, sizeof(double));
    double *pff = (double *)calloc((size_t)GZ, sizeof(double));
#pragma omp parallel for
    for (int gz = 0; gz < GZ; ++gz)
        for (int gy = 0; gy < gp.nb[1] * gp.n[1]; ++gy)
            for (int gx = 0; gx < gp.nb[0] * gp.n[0]; ++gx) {
                const double pc = p[moff(&gp, gx, gy, gz)];
                const double kc = (double)k[moff(&gk, gx, gy, gz)];
                double fl[3];
                for (int d = 0; d < 3; ++d) {
                    const int ox = d == 0, oy = d == 1, oz = d == 2;
                    const double pp = p[moff(&gp, gx + ox, gy + oy, gz + oz)];
                    const double pm = p[moff(&gp, gx - ox, gy - oy, gz - oz)];
                    const double kp = harmd(kc, (double)k[moff(&gk, gx + ox, gy + oy, gz + oz)]);
                    const double km = harmd((double)k[moff(&gk, gx - ox, gy - oy, gz - oz)], kc);
                    fl[d] = kp * (pp - pc) - km * (pc - pm);
                }
                const double Lp = ih2 * ((fl[0] + fl[1]) + fl[2]);
                const int64_t o = moff(&gk, gx, gy, gz);
                const double fc = (double)f[o];
                const double r = fc - Lp;
                if (r32)
                    r32[o] = (float)r;
                prr[gz] += r * r;
                pff[gz] += fc * fc;
            }
    double srr = 0, sff = 0;
    for (int gz = 0; gz < GZ; ++gz) {
        srr += prr[gz];
        sff += pff[gz];
    }
    free(prr);
    free(pff);
    *rr = srr;
    *ff = sff;
}

/* coarsest level: CG in FP64 on -L x = -f (mean removed), mean-zero result */
int or_mg_coarse_cg(const int nb[3], const int n[3], int64_t stride, const float *f,
                    const float *k, double ih2, int max_iter, double rtol, float *p)
{
    const mgeo g = mk(nb, n, stride);
    const int GX = nb[0] * n[0], GY = nb[1] * n[1], GZ = nb[2] * n[2];
    const int N = GX * GY * GZ;
    double *x = calloc(N, sizeof(double)), *r = calloc(N, sizeof(double)),
           *d = calloc(N, sizeof(double)), *q = calloc(N, sizeof(double)),
           *kk = calloc(N, sizeof(double));
    if (!x || !r || !d || !q || !kk)
        return -1;
#define GI(X, Y, Z) ((((X) + GX) % GX) + GX * ((((Y) + GY) % GY) + GY * (((Z) + GZ) % GZ)))
    double mean = 0;
    for (int z = 0; z < GZ; ++z)
        for (int y = 0; y < GY; ++y)
            for (int xx = 0; xx < GX; ++xx) {
                const int i = GI(xx, y, z);
                kk[i] = k[moff(&g, xx, y, z)];
                r[i] = -(double)f[moff(&g, xx, y, z)];
                mean += r[i];
            }
    mean /= N;
    double rr = 0;
    for (int i = 0; i < N; ++i) {
        r[i] -= mean;
        d[i] = r[i];
        rr += r[i] * r[i];
    }
    const double stop = rtol * rtol * rr;
    int it = 0;
    for (; it < max_iter && rr > stop && rr > 0; ++it) {
        double dq = 0;
        for (int z = 0; z < GZ; ++z)
            for (int y = 0; y < GY; ++y)
                for (int xx = 0; xx < GX; ++xx) {
                    const int i = GI(xx, y, z);
                    const int nbr[6] = {GI(xx + 1, y, z), GI(xx - 1, y, z), GI(xx, y + 1, z),
                                        GI(xx, y - 1, z), GI(xx, y, z + 1), GI(xx, y, z - 1)};
                    double s = 0;
                    for (int m = 0; m < 6; ++m)
                        s += harmd(kk[i], kk[nbr[m]]) * (d[i] - d[nbr[m]]);
                    q[i] = ih2 * s;
                    dq += d[i] * q[i];
                }
        const double alpha = rr / dq;
        double rn = 0;
        for (int i = 0; i < N; ++i) {
            x[i] += alpha * d[i];
            r[i] -= alpha * q[i];
            rn += r[i] * r[i];
        }
        const double beta = rn / rr;
        rr = rn;
        for (int i = 0; i < N; ++i)
            d[i] = r[i] + beta * d[i];
    }
    double xm = 0;
    for (int i = 0; i < N; ++i)
        xm += x[i];
    xm /= N;
    for (int z = 0; z < GZ; ++z)
        for (int y = 0; y < GY; ++y)
            for (int xx = 0; xx < GX; ++xx)
                p[moff(&g, xx, y, z)] = (float)(x[GI(xx, y, z)] - xm);
#undef GI
    free(x);
    free(r);
    free(d);
    free(q);
    free(kk);
    return it;
}
