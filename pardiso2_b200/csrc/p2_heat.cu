// Heat equation step (titerate, pardiso/heat3mg.c:292-829) on the device.
//
// What runs where:
//   right-hand side and step limit   k_heat_rhs      heaterr mode 0 (6-291),
//                                                    the max |dT/dt| loop 331-374
//   coarse kt, cp, ro                k_heat_rocp     rocprestrict 1235-1332
//   implicit 7-point rows            k_heat_rows     heaterr mode 1 (196-248)
//   smoother                         k_heat_gs       gausmatt 1057-1120, here
//                                                    red-black over the heat rows,
//                                                    each colour pass also setting
//                                                    the boundary rows (tbonderr
//                                                    841-893) of the other colour's
//                                                    targets
//   residual                         k_heat_resid    gausmatt 1103-1119
//   residual restriction             k_heat_restrict trestrict 1122-1233
//   correction prolongation          k_heat_prolong  tprolong 954-1054
//   error and float temperatures     k_heat_error    heaterr mode 2 (250-289),
//                                                    the reload 505-512
//   marker temperatures              k_heat_markers  641-768 with tkcalc1
//                                    k_heat_anti     (mark3mg.c:1212-1282),
//                                                    antidiffusion 770-829
// The V-cycle has the reference's shape: pre-smoothing and restriction down
// to multinumt, then smoothing and prolongation back up, with no smoothing
// on level 0 after the last prolongation.  The smoother is the one
// difference: Gauss-Seidel in two colours instead of the lexicographic
// order, so the iterates differ while the discrete equations, and so the
// converged temperatures, are the reference's.
//
// This file is compiled without fused multiply-adds, so the expressions
// below round as the reference's x86 code does: float arrays are combined
// in float where the reference's C does so (ro*cp, kt+kt, tk-tk0, the stress
// products), everything else in double.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "p2_internal.cuh"
#include "p2_interp.cuh"
#include "p2_solver.h"

namespace p2 {

static inline unsigned hb(long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

struct HeatLv {
    int nx, ny, nz;
    long n;
    const double *g[3];
    const int *bci;      // 0 heat row, q + 1 boundary row q
    const float *kt, *cp, *ro;
    double *x, *r;       // node order
    // colour order: node (i, j, k) of colour c = (i + j + k) & 1 at
    // c * nh + (k * nx + i) * nyh + j / 2, nyh = (ny + 1) / 2, nh = nx * nz * nyh,
    // so that one colour pass reads its rows contiguously
    double *b;           // right-hand side
    double *a;           // 7 planes of 2 * nh: diagonal (0 on boundary rows), x-, x+, y-, y+, z-, z+
    long nh;
};

__device__ __forceinline__ long heat_ci(const HeatLv &L, int i, int j, int k)
{
    const int nyh = (L.ny + 1) / 2;
    return ((i + j + k) & 1) * L.nh + ((long)k * L.nx + i) * nyh + (j >> 1);
}

__device__ __forceinline__ double heat_kf(const double *g, int m) { return 2.0 / (g[m + 1] - g[m - 1]); }

__device__ __forceinline__ double rocp(float ro, float cp)
{
    double v = (double)(ro * cp);  // float product, as ro[]*cp[] in the reference
    return v < 2e+6 ? 2e+6 : v;
}

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_min(double v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

struct HeatRhsArgs {
    HeatLv L;
    const float *tk, *ht, *et;
    float *tk0, *tk1;
    const float *vel[3];
    const double *pr;
    const float *se[12];
    int adiabyn, frictyn;
    double GX, GY, GZ;
    GridSh G;
    unsigned long long *rate_max;  // bits of the largest |dT/dt| (non-negative double)
};

// heaterr mode 0 per level-0 node; tk0 = tk for every node.
__global__ void __launch_bounds__(256) k_heat_rhs(HeatRhsArgs A)
{
    const HeatLv &L = A.L;
    const long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double rate = 0;
    if (u < L.n) {
        A.tk0[u] = A.tk[u];
        if (!L.bci[u]) {
            const long nxy = (long)L.nx * L.ny, ny = L.ny;
            const int m3 = (int)(u / nxy), m1 = (int)((u / ny) % L.nx), m2 = (int)(u % ny);
            const double *gx = L.g[0], *gy = L.g[1], *gz = L.g[2];
            const double xkf = heat_kf(gx, m1), ykf = heat_kf(gy, m2), zkf = heat_kf(gz, m3);
            const double rocpkf = rocp(L.ro[u], L.cp[u]);
            const float t0 = A.tk[u], ro = L.ro[u];
            double ival = A.ht[u];
            double x = 0, y = 0, z = 0;
            long p[8];
            if (A.adiabyn == 2 || A.frictyn) {
                p[0] = u; p[1] = p[0] + 1; p[2] = p[0] + ny; p[3] = p[2] + 1;
                p[4] = p[0] + nxy; p[5] = p[4] + 1; p[6] = p[4] + ny; p[7] = p[6] + 1;
                x = (gx[m1] - gx[m1 - 1]) / 2.0 * xkf;
                y = (gy[m2] - gy[m2 - 1]) / 2.0 * ykf;
                z = (gz[m3] - gz[m3 - 1]) / 2.0 * zkf;
            }
            double v[3] = {0, 0, 0};
            if (A.adiabyn) vxyz_at(A.G, A.vel[0], A.vel[1], A.vel[2], gx[m1], gy[m2], gz[m3], v);
            if (A.adiabyn == 2 && ro > 2e+3) {
                const double *pr = A.pr;
                const double dpdx = xkf * ((1.0 - y) * (1.0 - z) * (pr[p[2]] - pr[p[0]]) + y * (1.0 - z) * (pr[p[3]] - pr[p[1]]) +
                                           (1.0 - y) * z * (pr[p[6]] - pr[p[4]]) + y * z * (pr[p[7]] - pr[p[5]]));
                const double dpdy = ykf * ((1.0 - x) * (1.0 - z) * (pr[p[1]] - pr[p[0]]) + x * (1.0 - z) * (pr[p[3]] - pr[p[2]]) +
                                           (1.0 - x) * z * (pr[p[5]] - pr[p[4]]) + x * z * (pr[p[7]] - pr[p[6]]));
                const double dpdz = zkf * ((1.0 - x) * (1.0 - y) * (pr[p[4]] - pr[p[0]]) + x * (1.0 - y) * (pr[p[6]] - pr[p[2]]) +
                                           (1.0 - x) * y * (pr[p[5]] - pr[p[1]]) + x * y * (pr[p[7]] - pr[p[3]]));
                ival += A.et[u] * t0 * (v[0] * dpdx + v[1] * dpdy + v[2] * dpdz);
            }
            if (A.adiabyn == 1 && ro > 2e+3) ival += A.et[u] * t0 * ro * (v[0] * A.GX + v[1] * A.GY + v[2] * A.GZ);
            if (A.frictyn && ro > 2e+3) {
                const float *const *s = A.se;
                auto D = [&](int q) { return s[0][p[q]] * s[6][p[q]] + s[1][p[q]] * s[7][p[q]] + s[2][p[q]] * s[8][p[q]]; };
                double ev = (1.0 - x) * (1.0 - y) * (1.0 - z) * D(0);
                ev += (1.0 - x) * (y) * (1.0 - z) * D(1);
                ev += (x) * (1.0 - y) * (1.0 - z) * D(2);
                ev += (x) * (y) * (1.0 - z) * D(3);
                ev += (1.0 - x) * (1.0 - y) * (z) * D(4);
                ev += (1.0 - x) * (y) * (z) * D(5);
                ev += (x) * (1.0 - y) * (z) * D(6);
                ev += (x) * (y) * (z) * D(7);
                ev += 2.0 * ((1.0 - z) * (s[3][u - nxy] * s[9][u - nxy]) + z * (s[3][u] * s[9][u]));
                ev += 2.0 * ((1.0 - y) * (s[4][u - 1] * s[10][u - 1]) + y * (s[4][u] * s[10][u]));
                ev += 2.0 * ((1.0 - x) * (s[5][u - ny] * s[11][u - ny]) + x * (s[5][u] * s[11][u]));
                ival += ev;
            }
            A.tk1[u] = (float)ival;
            rate = fabs(ival / rocpkf);
        }
    }
    rate = warp_max(rate);
    if ((threadIdx.x & 31) == 0 && rate > 0) atomicMax(A.rate_max, (unsigned long long)__double_as_longlong(rate));
}

// rocprestrict: coarse kt, cp, ro as weighted averages of the finer level,
// gathered per coarse node in the reference's scatter order (fine nodes z, x,
// y ascending) with float accumulators.
__global__ void k_heat_rocp(HeatLv F, HeatLv C, AxisMap mx, AxisMap my, AxisMap mz)
{
    const long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= C.n) return;
    const long cnxy = (long)C.nx * C.ny, fnxy = (long)F.nx * F.ny;
    const int c3 = (int)(u / cnxy), c1 = (int)((u / C.ny) % C.nx), c2 = (int)(u % C.ny);
    float acp = 0, akt = 0, aro = 0;
    double den = 0;
    for (int qz = mz.ptr[c3]; qz < mz.ptr[c3 + 1]; qz++) {
        const double wz = mz.w[qz];
        const long oz = (long)mz.idx[qz] * fnxy;
        for (int qx = mx.ptr[c1]; qx < mx.ptr[c1 + 1]; qx++) {
            const double wx = mx.w[qx];
            const long ox = oz + (long)mx.idx[qx] * F.ny;
            for (int qy = my.ptr[c2]; qy < my.ptr[c2 + 1]; qy++) {
                const long f = ox + my.idx[qy];
                const double swt = wx * my.w[qy] * wz;
                acp = (float)((double)acp + F.cp[f] * swt);
                akt = (float)((double)akt + F.kt[f] * swt);
                aro = (float)((double)aro + F.ro[f] * swt);
                den += swt;
            }
        }
    }
    ((float *)C.cp)[u] = (float)(acp / den);
    ((float *)C.kt)[u] = (float)(akt / den);
    ((float *)C.ro)[u] = (float)(aro / den);
}

// heaterr mode 1: the 7 coefficients of every heat row of a level and, on
// level 0, its right-hand side tk1 + tk0/dt*rocp.
__global__ void __launch_bounds__(256) k_heat_rows(HeatLv L, double dt, const float *tk0, const float *tk1)
{
    const long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= L.n) return;
    const long nxy = (long)L.nx * L.ny, ny = L.ny, A = 2 * L.nh;
    const int m3 = (int)(u / nxy), m1 = (int)((u / ny) % L.nx), m2 = (int)(u % ny);
    const long c = heat_ci(L, m1, m2, m3);
    double *a = L.a;
    if (L.bci[u]) { a[c] = 0; return; }
    const double *gx = L.g[0], *gy = L.g[1], *gz = L.g[2];
    const double xkf = heat_kf(gx, m1), ykf = heat_kf(gy, m2), zkf = heat_kf(gz, m3);
    const double rocpkf = rocp(L.ro[u], L.cp[u]);
    const float *kt = L.kt;
    const float k3 = kt[u];
    double d = rocpkf / dt, v;
    v = (kt[u - ny] + k3) / 2.0 * xkf / (gx[m1] - gx[m1 - 1]);
    a[A + c] = -v; d += v;
    v = (k3 + kt[u + ny]) / 2.0 * xkf / (gx[m1 + 1] - gx[m1]);
    d += v; a[2 * A + c] = -v;
    v = (kt[u - 1] + k3) / 2.0 * ykf / (gy[m2] - gy[m2 - 1]);
    a[3 * A + c] = -v; d += v;
    v = (k3 + kt[u + 1]) / 2.0 * ykf / (gy[m2 + 1] - gy[m2]);
    d += v; a[4 * A + c] = -v;
    v = (kt[u - nxy] + k3) / 2.0 * zkf / (gz[m3] - gz[m3 - 1]);
    a[5 * A + c] = -v; d += v;
    v = (k3 + kt[u + nxy]) / 2.0 * zkf / (gz[m3 + 1] - gz[m3]);
    d += v; a[6 * A + c] = -v;
    a[c] = d;
    if (tk0) L.b[c] = tk1[u] + tk0[u] / dt * rocpkf;
}

// A x of the heat row of node u (colour index c) in the reference's term
// order (centre, x-, x+, y-, y+, z-, z+)
__device__ __forceinline__ double heat_ax(const HeatLv &L, long u, long c, double ival)
{
    const long nxy = (long)L.nx * L.ny, ny = L.ny, A = 2 * L.nh;
    const double *a = L.a, *x = L.x;
    ival += a[c] * x[u];
    ival += a[A + c] * x[u - ny];
    ival += a[2 * A + c] * x[u + ny];
    ival += a[3 * A + c] * x[u - 1];
    ival += a[4 * A + c] * x[u + 1];
    ival += a[5 * A + c] * x[u - nxy];
    ival += a[6 * A + c] * x[u + nxy];
    return ival;
}

struct HeatBc {
    int nbc;
    const int *bu, *bt;            // unknown, resolved heat-row target (-1: none)
    const double *bk, *bconst;
    const unsigned char *bpass;    // colour pass that sets the row: the one after its target's
};

// One colour of Gauss-Seidel over the heat rows ((i + j + k) & 1 == colour),
// and in the same launch the boundary rows x_u = c + k x_t (c only on level
// 0) whose target has the other colour: those targets do not change in this
// pass, and each boundary row is set once per sweep, right after its target.
__global__ void __launch_bounds__(256) k_heat_gs(HeatLv L, HeatBc B, int colour, double t0koef, int level0)
{
    const int nyh = (L.ny + 1) / 2;
    const long half = (long)nyh * L.nx * L.nz;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= half) {
        const long q = t - half;
        if (q < B.nbc && B.bpass[q] == colour) {
            const double c = level0 ? B.bconst[q] : 0.0;
            const int tg = B.bt[q];
            L.x[B.bu[q]] = tg >= 0 ? c + B.bk[q] * L.x[tg] : c;
        }
        return;
    }
    const int jj = (int)(t % nyh);
    const long rest = t / nyh;
    const int i = (int)(rest % L.nx), k = (int)(rest / L.nx);
    const int j = 2 * jj + ((i + k + colour) & 1);
    if (j >= L.ny) return;
    const long c = colour * L.nh + t;
    const double d = L.a[c];
    if (d == 0) return;  // boundary row
    const long u = (long)k * L.nx * L.ny + (long)i * L.ny + j;
    const double ival = heat_ax(L, u, c, -L.b[c]);
    L.x[u] -= ival / d * t0koef;
}

__global__ void __launch_bounds__(256) k_heat_resid(HeatLv L, HeatBc B, int level0)
{
    const long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= L.n) return;
    const int q = L.bci[u];
    if (!q) {
        const long nxy = (long)L.nx * L.ny;
        const long c = heat_ci(L, (int)((u / L.ny) % L.nx), (int)(u % L.ny), (int)(u / nxy));
        L.r[u] = L.b[c] - (heat_ax(L, u, c, 0.0));
        return;
    }
    const double c = level0 ? B.bconst[q - 1] : 0.0;
    const int t = B.bt[q - 1];
    L.r[u] = t >= 0 ? (c - L.x[u]) + B.bk[q - 1] * L.x[t] : c - L.x[u];
}

// trestrict: coarse right-hand side = weighted mean of the fine residuals
// over the heat rows of the coarse level, 0 on its boundary rows; coarse
// solution reset to 0.
__global__ void k_heat_restrict(HeatLv F, HeatLv C, AxisMap mx, AxisMap my, AxisMap mz)
{
    const long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= C.n) return;
    C.x[u] = 0;
    const long cnxy = (long)C.nx * C.ny, fnxy = (long)F.nx * F.ny;
    const int c3 = (int)(u / cnxy), c1 = (int)((u / C.ny) % C.nx), c2 = (int)(u % C.ny);
    const long ci = heat_ci(C, c1, c2, c3);
    if (C.bci[u]) { C.b[ci] = 0; return; }
    double num = 0, den = 0;
    for (int qz = mz.ptr[c3]; qz < mz.ptr[c3 + 1]; qz++) {
        const double wz = mz.w[qz];
        const long oz = (long)mz.idx[qz] * fnxy;
        for (int qx = mx.ptr[c1]; qx < mx.ptr[c1 + 1]; qx++) {
            const double wx = mx.w[qx];
            const long ox = oz + (long)mx.idx[qx] * F.ny;
            for (int qy = my.ptr[c2]; qy < my.ptr[c2 + 1]; qy++) {
                const double swt = wx * my.w[qy] * wz;
                num += F.r[ox + my.idx[qy]] * swt;
                den += swt;
            }
        }
    }
    C.b[ci] = den != 0 ? num / den : num;
}

// tprolong: x_f += t1koef * trilinear(x_c) on the heat rows of the finer level
__global__ void __launch_bounds__(256) k_heat_prolong(HeatLv F, HeatLv C, AxisMap mx, AxisMap my, AxisMap mz, double t1koef)
{
    const long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= F.n || F.bci[u]) return;
    const long fnxy = (long)F.nx * F.ny, cnxy = (long)C.nx * C.ny;
    const int m3 = (int)(u / fnxy), m1 = (int)((u / F.ny) % F.nx), m2 = (int)(u % F.ny);
    const int lz = mz.lo[m3], lx = mx.lo[m1], ly = my.lo[m2];
    const double wz[2] = {mz.w0[m3], mz.w1[m3]}, wx[2] = {mx.w0[m1], mx.w1[m1]}, wy[2] = {my.w0[m2], my.w1[m2]};
    double s = F.x[u];
    for (int c = 0; c < 2; c++)
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) {
                const long v = (long)(lz + c) * cnxy + (long)(lx + a) * C.ny + (ly + b);
                s += C.x[v] * (wx[a] * wy[b] * wz[c]) * t1koef;
            }
    F.x[u] = s;
}

// tk = (float) x on level 0, the error of every heat row (heaterr mode 2,
// times dt) squared, and the temperature range: per-block partials
// [sum, count, min, max].
__global__ void __launch_bounds__(256) k_heat_error(HeatLv L, const double *dtp, float *tk, const float *tk0,
                                                    const float *tk1, double *partial)
{
    const double dt = *dtp;
    const long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double e2 = 0, cnt = 0, tmin = 1e30, tmax = -1e30;
    if (u < L.n) {
        const double *x = L.x;
        const float t3 = (float)x[u];
        tk[u] = t3;
        tmin = tmax = t3;
        if (!L.bci[u]) {
            const long nxy = (long)L.nx * L.ny, ny = L.ny;
            const int m3 = (int)(u / nxy), m1 = (int)((u / ny) % L.nx), m2 = (int)(u % ny);
            const double *gx = L.g[0], *gy = L.g[1], *gz = L.g[2];
            const double xkf = heat_kf(gx, m1), ykf = heat_kf(gy, m2), zkf = heat_kf(gz, m3);
            const double rocpkf = rocp(L.ro[u], L.cp[u]);
            const float *kt = L.kt;
            const float k3 = kt[u];
            const float t1 = (float)x[u - ny], t5 = (float)x[u + ny], t2 = (float)x[u - 1], t4 = (float)x[u + 1];
            const float t0 = (float)x[u - nxy], t6 = (float)x[u + nxy];
            double e = (t3 - tk0[u]) / dt, w;
            w = (kt[u - ny] + k3) / 2.0 * xkf / (gx[m1] - gx[m1 - 1]) / rocpkf;
            e += (t3 - t1) * w;
            w = (k3 + kt[u + ny]) / 2.0 * xkf / (gx[m1 + 1] - gx[m1]) / rocpkf;
            e -= (t5 - t3) * w;
            w = (kt[u - 1] + k3) / 2.0 * ykf / (gy[m2] - gy[m2 - 1]) / rocpkf;
            e += (t3 - t2) * w;
            w = (k3 + kt[u + 1]) / 2.0 * ykf / (gy[m2 + 1] - gy[m2]) / rocpkf;
            e -= (t4 - t3) * w;
            w = (kt[u - nxy] + k3) / 2.0 * zkf / (gz[m3] - gz[m3 - 1]) / rocpkf;
            e += (t3 - t0) * w;
            w = (k3 + kt[u + nxy]) / 2.0 * zkf / (gz[m3 + 1] - gz[m3]) / rocpkf;
            e -= (t6 - t3) * w;
            e -= tk1[u] / rocpkf;
            e *= dt;
            e2 = e * e;
            cnt = 1;
        }
    }
    __shared__ double sh[4][8];
    e2 = warp_sum(e2); cnt = warp_sum(cnt); tmin = warp_min(tmin); tmax = warp_max(tmax);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { sh[0][w] = e2; sh[1][w] = cnt; sh[2][w] = tmin; sh[3][w] = tmax; }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        for (int q = 1; q < nw; q++) {
            e2 += sh[0][q]; cnt += sh[1][q]; tmin = fmin(tmin, sh[2][q]); tmax = fmax(tmax, sh[3][q]);
        }
        partial[4 * (long)blockIdx.x + 0] = e2;
        partial[4 * (long)blockIdx.x + 1] = cnt;
        partial[4 * (long)blockIdx.x + 2] = tmin;
        partial[4 * (long)blockIdx.x + 3] = tmax;
    }
}

__global__ void k_heat_load(long n, const float *tk, double *x)
{
    const long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n) x[u] = tk[u];
}

// fixed-order sum of the per-block partials (one block)
__global__ void k_heat_error_final(const double *partial, int nblk, double *out)
{
    double e2 = 0, cnt = 0, tmin = 1e30, tmax = -1e30;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
        e2 += partial[4 * b]; cnt += partial[4 * b + 1];
        tmin = fmin(tmin, partial[4 * b + 2]); tmax = fmax(tmax, partial[4 * b + 3]);
    }
    __shared__ double sh[4][32];
    e2 = warp_sum(e2); cnt = warp_sum(cnt); tmin = warp_min(tmin); tmax = warp_max(tmax);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { sh[0][w] = e2; sh[1][w] = cnt; sh[2][w] = tmin; sh[3][w] = tmax; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 1; q < (int)(blockDim.x >> 5); q++) {
            e2 += sh[0][q]; cnt += sh[1][q]; tmin = fmin(tmin, sh[2][q]); tmax = fmax(tmax, sh[3][q]);
        }
        out[0] = e2; out[1] = cnt; out[2] = tmin; out[3] = tmax;
    }
}

struct HeatMarkArgs {
    long nmark;
    const float *mx, *my, *mz;
    const signed char *mt;
    float *mk;
    GridSh G;
    const float *tk, *tk2, *kt, *cp, *ro;
    // per node, fixed point (two's complement in 64 bits): sum of weights
    // (scale 2^40) and sum of weighted diffusion changes (scale 2^32); after
    // k_heat_node_mean S1 holds their quotient as a double
    unsigned long long *S0, *S1;
    unsigned long long *range;  // set when a change is beyond the fixed-point range
    double heatdif, dt, tdeep, zdeep;
};

// Marker sums into the nodes are integer additions of fixed-point values, so
// their result does not depend on the order in which the markers arrive (the
// reference adds per-thread arrays in thread order).  The scales leave a
// resolution of 2^-40 for the weights (at most 8 per marker, all in [0, 1])
// and 2^-32 K for the temperature changes; |change x weight| must stay below
// 2^29 K, far above any temperature, else `range` is set and the host fails.
constexpr double kHeatW = 1099511627776.0;  // 2^40
constexpr double kHeatT = 4294967296.0;     // 2^32
__device__ __forceinline__ unsigned long long heat_fixed(double v, double scale, unsigned long long *range)
{
    const double f = v * scale;
    if (!(fabs(f) < 2305843009213693952.0)) {  // 2^61
        atomicOr(range, 1ull);
        return 0ull;
    }
    return (unsigned long long)__double2ll_rn(f);
}

// tkcalc1: cell, spacings and the 8 node weights (z outer, x, y inner)
__device__ __forceinline__ void tk_weights(const GridSh &G, double x, double y, double z, int c[3], double h[3],
                                           long wn[8], double wi[8])
{
    c[0] = serch(G.g[0], G.n[0], x);
    c[1] = serch(G.g[1], G.n[1], y);
    c[2] = serch(G.g[2], G.n[2], z);
    h[0] = G.g[0][c[0] + 1] - G.g[0][c[0]];
    h[1] = G.g[1][c[1] + 1] - G.g[1][c[1]];
    h[2] = G.g[2][c[2] + 1] - G.g[2][c[2]];
    const long nxy = (long)G.n[0] * G.n[1], ny = G.n[1];
    int q = 0;
    for (int m3 = c[2]; m3 <= c[2] + 1; m3++) {
        const double ddz = 1.0 - fabs((G.g[2][m3] - z) / h[2]);
        for (int m1 = c[0]; m1 <= c[0] + 1; m1++) {
            const double ddx = 1.0 - fabs((G.g[0][m1] - x) / h[0]);
            for (int m2 = c[1]; m2 <= c[1] + 1; m2++) {
                const double ddy = 1.0 - fabs((G.g[1][m2] - y) / h[1]);
                wi[q] = ddx * ddy * ddz;
                wn[q] = (long)m3 * nxy + (long)m1 * ny + m2;
                q++;
            }
        }
    }
}

__device__ __forceinline__ bool tk_inside(const HeatMarkArgs &A, long q)
{
    const float x = A.mx[q], y = A.my[q], z = A.mz[q];
    return x > 0 && y > 0 && z > 0 && (double)x < A.G.size[0] && (double)y < A.G.size[1] && (double)z < A.G.size[2];
}

// marker temperatures after the step (heat3mg.c:641-768): types 50..99 take
// the new node temperature; types below 50 are initialised where markk <= 0,
// relaxed towards the old node temperature by the numerical diffusion and
// shifted by the node temperature change.
__global__ void __launch_bounds__(256) k_heat_markers(HeatMarkArgs A)
{
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= A.nmark || !tk_inside(A, q)) return;
    const int t = A.mt[q];
    if (t >= 100) return;
    int c[3];
    double h[3], wi[8];
    long wn[8];
    tk_weights(A.G, A.mx[q], A.my[q], A.mz[q], c, h, wn, wi);
    double e2 = 0, e3 = 0;
    for (int n1 = 0; n1 < 8; n1++) {
        e2 += wi[n1] * A.tk[wn[n1]];
        e3 += wi[n1] * A.tk2[wn[n1]];
    }
    if (t >= 50) { A.mk[q] = (float)e2; return; }
    float mk = A.mk[q];
    if (mk <= 0) {
        mk = (float)e3;
        if (A.my[q] > A.zdeep && mk < A.tdeep) mk = (float)A.tdeep;
    }
    if (A.heatdif != 0) {
        double mkt = 0, mcp = 0, mro = 0, mtk = A.tk[wn[0]];
        for (int n1 = 0; n1 < 8; n1++) {
            const long m4 = wn[n1];
            const double w = wi[n1];
            mkt += A.kt[m4] * w; mcp += A.cp[m4] * w; mro += A.ro[m4] * w;
            mtk = fmax(mtk, (double)A.tk[m4]);
        }
        const int nx = A.G.n[0], ny = A.G.n[1], nz = A.G.n[2];
        if ((c[0] <= 0 || c[0] >= nx - 2 || c[1] <= 0 || c[1] >= ny - 2 || c[2] <= 0 || c[2] >= nz - 2) &&
            (mk + e2 - e3) > mtk)
            mk = (float)(mtk - e2 + e3);
        const double dtk = e3 - (double)mk;
        double rocpkf = mro * mcp;
        if (rocpkf < 2e+6) rocpkf = 2e+6;
        double dtk1 = -A.heatdif * mkt / rocpkf * 2.0 * (1.0 / h[0] / h[0] + 1.0 / h[1] / h[1] + 1.0 / h[2] / h[2]) * A.dt;
        if (dtk1 < -150.0) dtk1 = -150.0;
        dtk1 = dtk * (1.0 - exp(dtk1));
        mk += (float)dtk1;
        for (int n1 = 0; n1 < 8; n1++) {
            atomicAdd(A.S1 + wn[n1], heat_fixed(dtk1 * wi[n1], kHeatT, A.range));
            atomicAdd(A.S0 + wn[n1], heat_fixed(wi[n1], kHeatW, A.range));
        }
    }
    mk += (float)(e2 - e3);
    A.mk[q] = mk;
}

// mean diffusion change per node, written over the fixed-point sum S1
__global__ void k_heat_node_mean(long n, const unsigned long long *S0, unsigned long long *S1)
{
    const long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    const long long w = (long long)S0[u], d = (long long)S1[u];
    const double mean = w != 0 ? ((double)d / kHeatT) / ((double)w / kHeatW) : 0.0;
    reinterpret_cast<double *>(S1)[u] = mean;
}

// antidiffusion (heat3mg.c:770-829): the mean node change taken back from
// the markers of types below 50
__global__ void __launch_bounds__(256) k_heat_anti(HeatMarkArgs A)
{
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= A.nmark || !tk_inside(A, q) || A.mt[q] >= 50) return;
    int c[3];
    double h[3], wi[8];
    long wn[8];
    tk_weights(A.G, A.mx[q], A.my[q], A.mz[q], c, h, wn, wi);
    float mk = A.mk[q];
    for (int n1 = 0; n1 < 8; n1++) {
        const double s = reinterpret_cast<const double *>(A.S1)[wn[n1]];
        if (s != 0) mk -= (float)(s * wi[n1]);
    }
    A.mk[q] = mk;
}

// ---------------------------------------------------------------------------
// host side

// per-axis transfer weights between a fine and the next coarser level
// (the coarse cell index of heat3mg.c:979-990 and its two weights)
static void heat_axis(const std::vector<double> &gf, const std::vector<double> &gc, HostAxis &A)
{
    const int nf = (int)gf.size(), nc = (int)gc.size();
    A.lo.assign(nf, 0); A.w0.assign(nf, 0); A.w1.assign(nf, 0);
    std::vector<std::vector<std::pair<int, double>>> lists(nc);
    for (int m = 0; m < nf; m++) {
        int c = (m - 2) / 2 + 2;
        if (m < 3) c = m;
        if (m > nf - 4) c = nc - (nf - m);
        if (c > nc - 2) c = nc - 2;
        const double d = gc[c + 1] - gc[c];
        double w0 = (gc[c] - gf[m]) / d;
        w0 = -w0;
        w0 = 1.0 - w0;
        const double w1 = 1.0 - (gc[c + 1] - gf[m]) / d;
        A.lo[m] = c; A.w0[m] = w0; A.w1[m] = w1;
        lists[c].push_back({m, w0});
        lists[c + 1].push_back({m, w1});
    }
    A.ptr.assign(nc + 1, 0); A.idx.clear(); A.w.clear();
    for (int c = 0; c < nc; c++) {
        std::sort(lists[c].begin(), lists[c].end(), [](auto &p, auto &q) { return p.first < q.first; });
        for (auto &e : lists[c]) { A.idx.push_back(e.first); A.w.push_back(e.second); }
        A.ptr[c + 1] = (int)A.idx.size();
    }
}

template <typename T>
static T *heat_put(DeviceArena &ar, cudaStream_t st, const std::vector<T> &v)
{
    T *d = (T *)ar.alloc(sizeof(T) * std::max<size_t>(v.size(), 1));
    if (!v.empty()) P2_CUDA_TRY(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st));
    return d;
}

void Solver::heat_set_bc(const int *bondm, long bondm_len, const float *bondv1, const int *bondn1, long bondnum)
{
    if (!grid_ready) throw Error(P2_ERR_STATE, "no grid");
    const long nodenum = (long)L[0].n;
    if (bondm_len < 8 * nodenum + total_nodes)
        throw Error(P2_ERR_ARG, "bondm shorter than 8 * nodenum + (sum of level nodes): no T rows");
    P2_CUDA_TRY(cudaStreamSynchronize(st));
    heat_arena.release();
    heat_arena.guard = arena.guard;
    heat = HeatState{};
    const int *bt_all = bondm + 8 * nodenum;
    for (long u = 0; u < total_nodes; u++)
        if (bt_all[u] < 0 || bt_all[u] > bondnum) throw Error(P2_ERR_ARG, "T boundary row number out of range");
    const int nl = (int)L.size();
    heat.lv.resize(nl);
    for (int l = 0; l < nl; l++) {
        const Level &Lv = L[l];
        HeatLevel &H = heat.lv[l];
        const long n = Lv.n;
        std::vector<int> bci(n, 0), bu, bt;
        std::vector<double> bk, bc;
        std::vector<unsigned char> bpass;
        for (long v = 0; v < n; v++) {
            const long u = Lv.off + v;
            const int b0 = bt_all[u];
            const int i = (int)((v / Lv.ny) % Lv.nx), j = (int)(v % Lv.ny), k = (int)(v / ((long)Lv.nx * Lv.ny));
            const bool wall = i == 0 || j == 0 || k == 0 || i == Lv.nx - 1 || j == Lv.ny - 1 || k == Lv.nz - 1;
            if (!b0) {
                if (wall) throw Error(P2_ERR_UNSUPPORTED, "a boundary node without a T boundary row");
                continue;
            }
            // x_u = c + k x_t, followed through boundary targets
            double c = bondv1[2 * b0], kk = 1.0;
            long t = bondn1[b0] ? bondn1[b0] - 1 : -1;
            if (t >= 0) kk = bondv1[2 * b0 + 1];
            int depth = 0;
            while (t >= 0 && bt_all[t]) {
                if (t < Lv.off || t >= Lv.off + n) throw Error(P2_ERR_UNSUPPORTED, "T boundary row coupled across levels");
                const int b1 = bt_all[t];
                c += kk * bondv1[2 * b1];
                if (bondn1[b1]) { kk *= bondv1[2 * b1 + 1]; t = bondn1[b1] - 1; }
                else { t = -1; }
                if (++depth > 64) throw Error(P2_ERR_UNSUPPORTED, "cyclic T boundary rows");
            }
            if (t >= 0 && (t < Lv.off || t >= Lv.off + n)) throw Error(P2_ERR_UNSUPPORTED, "T boundary row coupled across levels");
            bci[v] = (int)bu.size() + 1;
            bu.push_back((int)v);
            bt.push_back(t >= 0 ? (int)(t - Lv.off) : -1);
            bk.push_back(t >= 0 ? kk : 0.0);
            bc.push_back(c);
            if (t >= 0) {
                const long tl = t - Lv.off;
                const int ti = (int)((tl / Lv.ny) % Lv.nx), tj = (int)(tl % Lv.ny), tk = (int)(tl / ((long)Lv.nx * Lv.ny));
                bpass.push_back((unsigned char)(1 - ((ti + tj + tk) & 1)));
            } else {
                bpass.push_back(0);
            }
        }
        H.nbc = (int)bu.size();
        H.bci = heat_put(heat_arena, st, bci);
        H.bu = heat_put(heat_arena, st, bu);
        H.bt = heat_put(heat_arena, st, bt);
        H.bk = heat_put(heat_arena, st, bk);
        H.bconst = heat_put(heat_arena, st, bc);
        H.bpass = heat_put(heat_arena, st, bpass);
        for (int a = 0; a < 3; a++) H.g[a] = heat_put(heat_arena, st, Lv.g[a]);
        H.kt = l ? (float *)heat_arena.alloc(sizeof(float) * n) : nullptr;
        H.cp = l ? (float *)heat_arena.alloc(sizeof(float) * n) : nullptr;
        H.ro = l ? (float *)heat_arena.alloc(sizeof(float) * n) : nullptr;
        H.x = (double *)heat_arena.alloc(sizeof(double) * n);
        const long nh = (long)Lv.nx * Lv.nz * ((Lv.ny + 1) / 2);
        H.nh = nh;
        H.b = (double *)heat_arena.alloc(sizeof(double) * 2 * nh);
        H.r = (double *)heat_arena.alloc(sizeof(double) * n);
        H.a = (double *)heat_arena.alloc(sizeof(double) * 7 * 2 * nh);
        P2_CUDA_TRY(cudaMemsetAsync(H.x, 0, sizeof(double) * n, st));
        P2_CUDA_TRY(cudaMemsetAsync(H.b, 0, sizeof(double) * 2 * nh, st));
        if (l > 0) {
            for (int a = 0; a < 3; a++) {
                HostAxis ax;
                heat_axis(L[l - 1].g[a], Lv.g[a], ax);
                AxisMap &m = heat.lv[l - 1].map[a];
                m.lo = heat_put(heat_arena, st, ax.lo);
                m.w0 = heat_put(heat_arena, st, ax.w0);
                m.w1 = heat_put(heat_arena, st, ax.w1);
                m.ptr = heat_put(heat_arena, st, ax.ptr);
                m.idx = heat_put(heat_arena, st, ax.idx);
                m.w = heat_put(heat_arena, st, ax.w);
            }
        }
    }
    const long n0 = L[0].n;
    for (float **p : {&heat.tk, &heat.tk0, &heat.tk1, &heat.tk2, &heat.kt, &heat.cp, &heat.ro, &heat.ht, &heat.et})
        *p = (float *)heat_arena.alloc(sizeof(float) * n0);
    for (int a = 0; a < 3; a++) heat.vel[a] = (float *)heat_arena.alloc(sizeof(float) * n0);
    heat.pr = (double *)heat_arena.alloc(sizeof(double) * n0);
    for (int q = 0; q < 12; q++) heat.se[q] = (float *)heat_arena.alloc(sizeof(float) * n0);
    heat.nblk = (int)hb(n0);
    heat.partial = (double *)heat_arena.alloc(sizeof(double) * 4 * heat.nblk);
    heat.scal = (double *)heat_arena.alloc(sizeof(double) * 8);
    heat.S0 = (double *)heat_arena.alloc(sizeof(double) * n0);
    heat.S1 = (double *)heat_arena.alloc(sizeof(double) * n0);
    {
        cudaStream_t s2 = nullptr;
        P2_CUDA_TRY(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
        heat.mst_owner.reset(s2, [](CUstream_st *p) { cudaStreamDestroy(p); });
        heat.mst = s2;
        cudaEvent_t e2 = nullptr;
        P2_CUDA_TRY(cudaEventCreateWithFlags(&e2, cudaEventDisableTiming));
        heat.mev_owner.reset(e2, [](CUevent_st *p) { cudaEventDestroy(p); });
        heat.mev = e2;
    }
    P2_CUDA_TRY(cudaMallocHost((void **)&heat.host, sizeof(double) * 8));  // [0..3] error, range; [4] sub-step
    heat.host_owner.reset(heat.host, [](double *p) { cudaFreeHost(p); });
    P2_CUDA_TRY(cudaStreamSynchronize(st));
    heat.ready = true;
}

static HeatLv heat_view(const Level &Lv, const HeatLevel &H, const HeatState &S, int l)
{
    HeatLv v;
    v.nx = Lv.nx; v.ny = Lv.ny; v.nz = Lv.nz; v.n = Lv.n;
    for (int a = 0; a < 3; a++) v.g[a] = H.g[a];
    v.bci = H.bci;
    v.kt = l ? H.kt : S.kt;
    v.cp = l ? H.cp : S.cp;
    v.ro = l ? H.ro : S.ro;
    v.x = H.x; v.b = H.b; v.r = H.r; v.a = H.a; v.nh = H.nh;
    return v;
}

static HeatBc heat_bc_view(const HeatLevel &H) { return HeatBc{H.nbc, H.bu, H.bt, H.bk, H.bconst, H.bpass}; }

void Solver::heat_smooth(int l, int sweeps, double t0koef)
{
    const HeatLv V = heat_view(L[l], heat.lv[l], heat, l);
    const HeatBc B = heat_bc_view(heat.lv[l]);
    const long half = (long)((V.ny + 1) / 2) * V.nx * V.nz;
    for (int s = 0; s < sweeps; s++)
        for (int c = 0; c < 2; c++) {
            k_heat_gs<<<hb(half + B.nbc), 256, 0, st>>>(V, B, c, t0koef, l == 0);
            heat.kernels++;
        }
    k_heat_resid<<<hb(V.n), 256, 0, st>>>(V, B, l == 0);
    heat.kernels++;
}

// multicyct V-cycles on levels 0..multinumt (heat3mg.c:462-500), then the
// level-0 error and temperature range into heat.scal[0..3]
void Solver::heat_batch(const p2_heat_params &hp)
{
    const int nt = hp.multinumt;
    for (int c = 0; c < hp.multicyct; c++) {
        if (nt > 0) {
            for (int l = 0; l < nt; l++) {
                heat_smooth(l, hp.multittt[0][l], hp.t0koef);
                const HeatLv F = heat_view(L[l], heat.lv[l], heat, l), C = heat_view(L[l + 1], heat.lv[l + 1], heat, l + 1);
                const AxisMap *m = heat.lv[l].map;
                k_heat_restrict<<<hb(C.n), 256, 0, st>>>(F, C, m[0], m[1], m[2]);
                heat.kernels++;
            }
            for (int l = nt; l > 0; l--) {
                heat_smooth(l, hp.multittt[1][l], hp.t0koef);
                const HeatLv F = heat_view(L[l - 1], heat.lv[l - 1], heat, l - 1), C = heat_view(L[l], heat.lv[l], heat, l);
                const AxisMap *m = heat.lv[l - 1].map;
                k_heat_prolong<<<hb(F.n), 256, 0, st>>>(F, C, m[0], m[1], m[2], hp.t1koef);
                heat.kernels++;
            }
        } else {
            heat_smooth(0, hp.multittt[0][0], hp.t0koef);
        }
    }
    const HeatLv V0 = heat_view(L[0], heat.lv[0], heat, 0);
    k_heat_error<<<heat.nblk, 256, 0, st>>>(V0, heat.scal + 4, heat.tk, heat.tk0, heat.tk1, heat.partial);
    k_heat_error_final<<<1, 1024, 0, st>>>(heat.partial, heat.nblk, heat.scal);
    heat.kernels += 2;
}

p2_heat_info Solver::titerate(const p2_heat_params &hp, double timestep, float *tk, const float *kt, const float *cp,
                              const float *ro, const float *ht, const float *et, const float *vx, const float *vy,
                              const float *vz, const double *pr, const float *const *se, long nmark,
                              const float *mx, const float *my, const float *mz, const signed char *mt, float *markk)
{
    if (!heat.ready) throw Error(P2_ERR_STATE, "no T boundary rows (p2_heat_set_bc)");
    if (hp.multinumt < 0 || hp.multinumt >= (int)L.size()) throw Error(P2_ERR_ARG, "multinumt above the grid's levels");
    if (hp.multicyct < 1) throw Error(P2_ERR_ARG, "multicyct < 1");
    if (!tk || !kt || !cp || !ro || !ht || !et) throw Error(P2_ERR_ARG, "null node field");
    if (hp.adiabyn && (!vx || !vy || !vz)) throw Error(P2_ERR_ARG, "adiabyn needs vx, vy, vz");
    if (hp.adiabyn == 2 && !pr) throw Error(P2_ERR_ARG, "adiabyn 2 needs pr");
    if (hp.frictyn && !se) throw Error(P2_ERR_ARG, "frictyn needs the stress and strain-rate fields");
    if (nmark < 0 || (nmark > 0 && (!mx || !my || !mz || !mt || !markk))) throw Error(P2_ERR_ARG, "bad markers");
    if (timestep < 0) throw Error(P2_ERR_ARG, "negative timestep");
    const long n0 = L[0].n;
    const size_t fb = sizeof(float) * n0;
    p2_heat_info info{};
    info.tktimestep = 1e30;
    heat.kernels = 0;
    P2_CUDA_TRY(cudaEventRecord(ev[0], st));
    P2_CUDA_TRY(cudaMemcpyAsync(heat.tk, tk, fb, cudaMemcpyHostToDevice, st));
    P2_CUDA_TRY(cudaMemcpyAsync(heat.kt, kt, fb, cudaMemcpyHostToDevice, st));
    P2_CUDA_TRY(cudaMemcpyAsync(heat.cp, cp, fb, cudaMemcpyHostToDevice, st));
    P2_CUDA_TRY(cudaMemcpyAsync(heat.ro, ro, fb, cudaMemcpyHostToDevice, st));
    P2_CUDA_TRY(cudaMemcpyAsync(heat.ht, ht, fb, cudaMemcpyHostToDevice, st));
    P2_CUDA_TRY(cudaMemcpyAsync(heat.et, et, fb, cudaMemcpyHostToDevice, st));
    if (hp.adiabyn) {
        const float *v[3] = {vx, vy, vz};
        for (int a = 0; a < 3; a++) P2_CUDA_TRY(cudaMemcpyAsync(heat.vel[a], v[a], fb, cudaMemcpyHostToDevice, st));
    }
    if (hp.adiabyn == 2) P2_CUDA_TRY(cudaMemcpyAsync(heat.pr, pr, sizeof(double) * n0, cudaMemcpyHostToDevice, st));
    if (hp.frictyn)
        for (int q = 0; q < 12; q++) P2_CUDA_TRY(cudaMemcpyAsync(heat.se[q], se[q], fb, cudaMemcpyHostToDevice, st));

    GridSh G;
    for (int a = 0; a < 3; a++) {
        G.g[a] = heat.lv[0].g[a];
        G.n[a] = a == 0 ? L[0].nx : a == 1 ? L[0].ny : L[0].nz;
        G.size[a] = L[0].g[a].back() - L[0].g[a].front();
    }
    const HeatLv V0 = heat_view(L[0], heat.lv[0], heat, 0);
    {
        HeatRhsArgs A;
        A.L = V0;
        A.tk = heat.tk; A.ht = heat.ht; A.et = heat.et; A.tk0 = heat.tk0; A.tk1 = heat.tk1;
        for (int a = 0; a < 3; a++) A.vel[a] = heat.vel[a];
        A.pr = heat.pr;
        for (int q = 0; q < 12; q++) A.se[q] = heat.se[q];
        A.adiabyn = hp.adiabyn; A.frictyn = hp.frictyn;
        A.GX = prm.gxkoef; A.GY = prm.gykoef; A.GZ = prm.gzkoef;
        A.G = G;
        A.rate_max = (unsigned long long *)heat.scal;
        P2_CUDA_TRY(cudaMemsetAsync(heat.scal, 0, sizeof(double) * 8, st));
        k_heat_rhs<<<hb(n0), 256, 0, st>>>(A);
        heat.kernels++;
        P2_CUDA_TRY(cudaMemcpyAsync(heat.host, heat.scal, sizeof(double), cudaMemcpyDeviceToHost, st));
        P2_CUDA_TRY(cudaStreamSynchronize(st));
        P2_CUDA_TRY(cudaGetLastError());
    }
    const double maxtkrate = heat.host[0];
    double tktimestep = 1e30;
    if (maxtkrate) tktimestep = hp.maxtkstep / maxtkrate;
    info.tktimestep = tktimestep;
    info.maxtkrate = maxtkrate;
    info.converged = 1;
    if (timestep == 0 || tktimestep == 0) {
        P2_CUDA_TRY(cudaEventRecord(ev[1], st));
        P2_CUDA_TRY(cudaEventSynchronize(ev[1]));
        float ms = 0;
        P2_CUDA_TRY(cudaEventElapsedTime(&ms, ev[0], ev[1]));
        info.ms_total = ms;
        info.kernels = heat.kernels;
        return info;
    }
    // The markers are needed only after the last sub-step: a helper thread
    // copies them on a second stream while the sub-steps run (the copies
    // from pageable memory block the thread that issues them).
    struct Uploader {
        std::thread th;
        cudaError_t err = cudaSuccess;
        ~Uploader()
        {
            if (th.joinable()) th.join();
        }
    } up;
    if (nmark > 0) {
        if (nmark > heat.mcap) {
            P2_CUDA_TRY(cudaStreamSynchronize(st));
            heat_mk_arena.release();
            heat_mk_arena.guard = 0;
            heat.mx = (float *)heat_mk_arena.alloc(sizeof(float) * nmark);
            heat.my = (float *)heat_mk_arena.alloc(sizeof(float) * nmark);
            heat.mz = (float *)heat_mk_arena.alloc(sizeof(float) * nmark);
            heat.mk = (float *)heat_mk_arena.alloc(sizeof(float) * nmark);
            heat.mt = (signed char *)heat_mk_arena.alloc(nmark);
            heat.mcap = nmark;
        }
        const int device = dev;
        Uploader *u = &up;
        const HeatState *H = &heat;
        up.th = std::thread([u, H, device, nmark, mx, my, mz, mt, markk] {
            const size_t mb = sizeof(float) * nmark;
            cudaError_t e = cudaSetDevice(device);
            if (e == cudaSuccess) e = cudaMemcpyAsync(H->mx, mx, mb, cudaMemcpyHostToDevice, H->mst);
            if (e == cudaSuccess) e = cudaMemcpyAsync(H->my, my, mb, cudaMemcpyHostToDevice, H->mst);
            if (e == cudaSuccess) e = cudaMemcpyAsync(H->mz, mz, mb, cudaMemcpyHostToDevice, H->mst);
            if (e == cudaSuccess) e = cudaMemcpyAsync(H->mk, markk, mb, cudaMemcpyHostToDevice, H->mst);
            if (e == cudaSuccess) e = cudaMemcpyAsync(H->mt, mt, nmark, cudaMemcpyHostToDevice, H->mst);
            if (e == cudaSuccess) e = cudaEventRecord(H->mev, H->mst);
            u->err = e;
        });
    }
    P2_CUDA_TRY(cudaMemcpyAsync(heat.tk2, heat.tk, fb, cudaMemcpyDeviceToDevice, st));
    const int nt = hp.multinumt;
    for (int l = 1; l <= nt; l++) {
        const HeatLv F = heat_view(L[l - 1], heat.lv[l - 1], heat, l - 1), C = heat_view(L[l], heat.lv[l], heat, l);
        const AxisMap *m = heat.lv[l - 1].map;
        k_heat_rocp<<<hb(C.n), 256, 0, st>>>(F, C, m[0], m[1], m[2]);
        heat.kernels++;
    }
    const int maxcyc = hp.max_cycles > 0 ? hp.max_cycles : 10000;
    struct Batch {
        cudaGraphExec_t exec = nullptr;
        long long kernels = 0;
        ~Batch() { if (exec) cudaGraphExecDestroy(exec); }
    } batch;
    double tktimesum = 0, tktimesum0 = timestep, heatsum = 0;
    do {
        double dt = tktimesum0 < tktimestep ? tktimesum0 : tktimestep;
        if (dt > (tktimesum0 - tktimesum)) dt = tktimesum0 - tktimesum;
        info.substeps++;
        P2_CUDA_TRY(cudaMemcpyAsync(heat.tk0, heat.tk, fb, cudaMemcpyDeviceToDevice, st));
        k_heat_load<<<hb(n0), 256, 0, st>>>(n0, heat.tk, V0.x);
        heat.kernels++;
        for (int l = 0; l <= nt; l++) {
            const HeatLv V = heat_view(L[l], heat.lv[l], heat, l);
            k_heat_rows<<<hb(V.n), 256, 0, st>>>(V, dt, l ? nullptr : heat.tk0, heat.tk1);
            heat.kernels++;
        }
        // the sub-step size for the error kernel (device memory, so that one
        // captured batch serves every sub-step)
        heat.host[4] = dt;
        P2_CUDA_TRY(cudaMemcpyAsync(heat.scal + 4, heat.host + 4, sizeof(double), cudaMemcpyHostToDevice, st));
        if (!batch.exec) {
            // multicyct V-cycles and the error reduction as one graph
            const long long k0 = heat.kernels;
            cudaGraph_t g = nullptr;
            P2_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            heat_batch(hp);
            P2_CUDA_TRY(cudaStreamEndCapture(st, &g));
            const cudaError_t e = cudaGraphInstantiate(&batch.exec, g, 0);
            cudaGraphDestroy(g);
            P2_CUDA_TRY(e);
            batch.kernels = heat.kernels - k0;
            heat.kernels = k0;
        }
        int cyc = 0;
        do {
            P2_CUDA_TRY(cudaGraphLaunch(batch.exec, st));
            heat.kernels += batch.kernels;
            P2_CUDA_TRY(cudaMemcpyAsync(heat.host, heat.scal, sizeof(double) * 4, cudaMemcpyDeviceToHost, st));
            P2_CUDA_TRY(cudaStreamSynchronize(st));
            P2_CUDA_TRY(cudaGetLastError());
            heatsum = pow(heat.host[0] / heat.host[1], 0.5);
            info.mintk = heat.host[2];
            info.maxtk = heat.host[3];
            info.cycles++;
            cyc++;
            if (!(heatsum == heatsum)) throw Error(P2_ERR_NAN, "NaN in the heat equation error");
            if (heatsum > hp.heatmin && cyc >= maxcyc) { info.converged = 0; break; }
        } while (heatsum > hp.heatmin);
        tktimesum += dt;
        if (!info.converged) break;
    } while (tktimesum < tktimesum0);
    info.heatsum = heatsum;

    if (nmark > 0) {
        const size_t mb = sizeof(float) * nmark;
        up.th.join();
        P2_CUDA_TRY(up.err);
        P2_CUDA_TRY(cudaStreamWaitEvent(st, heat.mev, 0));
        P2_CUDA_TRY(cudaMemsetAsync(heat.S0, 0, sizeof(double) * n0, st));
        P2_CUDA_TRY(cudaMemsetAsync(heat.S1, 0, sizeof(double) * n0, st));
        HeatMarkArgs M;
        M.nmark = nmark; M.mx = heat.mx; M.my = heat.my; M.mz = heat.mz; M.mt = heat.mt; M.mk = heat.mk;
        M.G = G;
        M.tk = heat.tk; M.tk2 = heat.tk2; M.kt = heat.kt; M.cp = heat.cp; M.ro = heat.ro;
        M.S0 = (unsigned long long *)heat.S0; M.S1 = (unsigned long long *)heat.S1;
        M.range = (unsigned long long *)(heat.scal + 6);
        P2_CUDA_TRY(cudaMemsetAsync(heat.scal + 6, 0, sizeof(double), st));
        M.heatdif = hp.heatdif; M.dt = tktimesum0; M.tdeep = hp.tdeep; M.zdeep = hp.zdeep;
        k_heat_markers<<<hb(nmark), 256, 0, st>>>(M);
        heat.kernels++;
        if (hp.heatdif != 0) {
            k_heat_node_mean<<<hb(n0), 256, 0, st>>>(n0, M.S0, M.S1);
            k_heat_anti<<<hb(nmark), 256, 0, st>>>(M);
            heat.kernels += 2;
        }
        P2_CUDA_TRY(cudaMemcpyAsync(markk, heat.mk, mb, cudaMemcpyDeviceToHost, st));
        P2_CUDA_TRY(cudaMemcpyAsync(heat.host + 6, heat.scal + 6, sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    P2_CUDA_TRY(cudaMemcpyAsync(tk, heat.tk, fb, cudaMemcpyDeviceToHost, st));
    P2_CUDA_TRY(cudaEventRecord(ev[1], st));
    P2_CUDA_TRY(cudaEventSynchronize(ev[1]));
    P2_CUDA_TRY(cudaGetLastError());
    float ms = 0;
    P2_CUDA_TRY(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    if (nmark > 0) {
        unsigned long long range = 0;
        std::memcpy(&range, heat.host + 6, sizeof(range));
        if (range) throw Error(P2_ERR_ARG, "a marker temperature change is beyond 2^29 K (markk or tk corrupt)");
    }
    info.ms_total = ms;
    info.kernels = heat.kernels;
    return info;
}

}  // namespace p2
