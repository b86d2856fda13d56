// Point location and staggered velocity interpolation on the level-0 grid,
// shared by the marker kernels and the heat equation's adiabatic term.
#pragma once

#include <cuda_runtime.h>

namespace p2 {

// cell of x on gridlines g[0..n-1] by bisection (m1serch..m3serch,
// pardiso/mark3mg.c:1138-1204)
__device__ __forceinline__ int serch(const double *g, int n, double x)
{
    int a = 0, b = n - 1, m;
    do {
        m = (a + b) / 2;
        if (g[m] > x) b = m; else a = m;
    } while (b - a > 1);
    if (a > n - 2) a = n - 2;
    return a;
}

// ---------------------------------------------------------------------------
// Marker advection (movemark, pardiso/mark3mg.c:174-629, Runge-Kutta and
// single-velocity branches, non-periodic box): velocity at a point by
// staggered trilinear interpolation (vxyzcalc1, mark3mg.c:2963-3243) with the
// reference's clamping of points and cell indices at the walls, in the same
// double arithmetic without fused multiply-adds, so positions match the
// reference bit for bit.  Halvings are multiplications by 0.5 (the same
// correctly rounded value as a division by 2).  Per stage each axis's weights
// are computed once for the component aligned with it (node interval) and
// once for the two others (cell mid-points); the gridlines sit in shared
// memory for the binary searches.
__device__ __forceinline__ double dmid(const double *g, int m) { return __dmul_rn(__dadd_rn(g[m], g[m + 1]), 0.5); }

// component-aligned axis: the node interval of the cell (clamped), weights
// from the node positions
__device__ __forceinline__ void ax_node(const double *g, int n, int cell, double x, int &lo, double &w0, double &w1)
{
    lo = cell;
    if (lo < 0) lo = 0;
    if (lo > n - 2) lo = n - 2;
    const double d = __dsub_rn(g[lo + 1], g[lo]);
    w0 = __dsub_rn(1.0, -__ddiv_rn(__dsub_rn(g[lo], x), d));
    w1 = __dsub_rn(1.0, __ddiv_rn(__dsub_rn(g[lo + 1], x), d));
}

// cross axis: cell mid-points (staggered), point clamped onto the first or
// last mid-point outside the interior range
__device__ __forceinline__ void ax_mid(const double *g, int n, int cell, double x, int &lo, double &w0, double &w1)
{
    lo = cell;
    double X = x;
    const double m0 = dmid(g, lo);
    if (X < m0) lo -= 1;
    if (lo < 0) { lo = 0; X = dmid(g, 0); }
    if (lo > n - 3) { lo = n - 3; X = dmid(g, lo + 1); }
    const double d = __dmul_rn(__dsub_rn(g[lo + 2], g[lo]), 0.5);
    w0 = __dsub_rn(1.0, -__ddiv_rn(__dsub_rn(dmid(g, lo), X), d));
    w1 = __dsub_rn(1.0, __ddiv_rn(__dsub_rn(dmid(g, lo + 1), X), d));
}

// gridlines of the three axes, concatenated (x, y, z)
struct GridSh {
    const double *g[3];
    int n[3];
    double size[3];
};

__device__ inline void vxyz_at(const GridSh &G, const float *vx, const float *vy, const float *vz, double x, double y,
                        double z, double out[3])
{
    const double p[3] = {x < 0 ? 0.0 : (x > G.size[0] ? G.size[0] : x), y < 0 ? 0.0 : (y > G.size[1] ? G.size[1] : y),
                         z < 0 ? 0.0 : (z > G.size[2] ? G.size[2] : z)};
    int lon[3], lom[3];
    double wn[3][2], wm[3][2];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const int cell = serch(G.g[a], G.n[a], p[a]);
        ax_node(G.g[a], G.n[a], cell, p[a], lon[a], wn[a][0], wn[a][1]);
        ax_mid(G.g[a], G.n[a], cell, p[a], lom[a], wm[a][0], wm[a][1]);
    }
    const long nxy = (long)G.n[0] * G.n[1], ny = G.n[1];
    const float *v[3] = {vx, vy, vz};
#pragma unroll
    for (int comp = 0; comp < 3; comp++) {
        int lo[3];
        double w[3][2];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            lo[a] = a == comp ? lon[a] : lom[a];
            w[a][0] = a == comp ? wn[a][0] : wm[a][0];
            w[a][1] = a == comp ? wn[a][1] : wm[a][1];
        }
        // accumulation order of the reference: z outer, x, y inner
        double s = 0;
#pragma unroll
        for (int c = 0; c < 2; c++)
#pragma unroll
            for (int a = 0; a < 2; a++)
#pragma unroll
                for (int b = 0; b < 2; b++) {
                    const long idx = (long)(lo[2] + c) * nxy + (long)(lo[0] + a) * ny + (lo[1] + b);
                    const double swt = __dmul_rn(__dmul_rn(w[0][a], w[1][b]), w[2][c]);
                    s = __dadd_rn(s, __dmul_rn((double)__ldg(v[comp] + idx), swt));
                }
        out[comp] = s;
    }
}

}  // namespace p2
