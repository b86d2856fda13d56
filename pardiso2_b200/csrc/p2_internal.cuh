// Internal device/host definitions of the p2cuda Stokes multigrid.
//
// Discretisation (reference lines, paths relative to the reference project):
//   stresses sxx..syz .......... pardiso/move3mgNew.c:3-794
//   x/y/z-Stokes rows .......... pardiso/move3mgNew.c:796-1450
//   continuity row ............. pardiso/move3mgNew.c:1455-1576
//   boundary rows .............. pardiso/move3mgNew.c:1682-1729
// The rows are evaluated matrix-free from per-stencil viscosities instead of
// the reference's 57-coefficient row store (gausmat2, gaus3mg_SerieMG.c:312).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/p2cuda.h"

#define P2_CUDA_TRY(expr)                                                              \
    do {                                                                               \
        cudaError_t e_ = (expr);                                                       \
        if (e_ != cudaSuccess) throw p2::Error(P2_ERR_CUDA, std::string(#expr) + ": " + \
                                                             cudaGetErrorString(e_));  \
    } while (0)

namespace p2 {

// Kernels launched by this library on the calling host thread (a graph
// launch adds the number of kernel nodes it replays).
extern thread_local long long g_launches;

// Level-0 gridlines on the device for marker kernels.
struct Grid3 {
    const double *g[3];
    int n[3];        // xnumx, ynumy, znumz
    double size[3];  // xsize, ysize, zsize
};

// Replayable launch sequence of the coarsest LU and inverse (p2_lu.cu).
struct LuGraph {
    cudaGraphExec_t exec = nullptr;
    int n = 0, kl = -1, ku = -1;
    const double *A = nullptr, *Ainv = nullptr;
    const int *ipiv = nullptr, *info = nullptr;
    long long kernels = 0;
};
#define P2_COUNT_LAUNCH() (++p2::g_launches)

// Programmatic dependent launch (the V-cycle's kernels are launched with
// programmatic stream serialization, so the next grid is scheduled while the
// previous one drains): a kernel first waits until its predecessor grid has
// completed and its writes are visible (griddepcontrol.wait; a no-op when the
// launch has no programmatic dependency), then, if it fits in one wave, lets
// its own successor be scheduled.  Larger grids leave that to their exit, so
// waiting blocks of the next grid never take SM slots from their later waves.
constexpr unsigned kPdlOneWave = 296;  // two blocks per SM
__device__ __forceinline__ void pdl_enter()
{
#ifndef P2_NO_PDL
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (gridDim.x * gridDim.y * gridDim.z <= kPdlOneWave) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}

struct Error {
    p2_status code;
    std::string msg;
    Error(p2_status c, std::string m) : code(c), msg(std::move(m)) {}
};

// Bits of the per-node boundary mask: bit c set when unknown (node, c) is a
// boundary row (c = 0 P, 1 Vx, 2 Vy, 3 Vz).  The pinned pressure cell is not
// marked: it is smoothed as a continuity row and fixed by a pressure shift.
enum { BC_P = 1, BC_VX = 2, BC_VY = 4, BC_VZ = 8 };

// Inverse spacings of one axis (see the oracle's spacings()).
template <typename T>
struct Axis {
    const T *ih;   // 1/(g[i]-g[i-1])       i >= 1
    const T *ihc;  // 2/(g[i+1]-g[i-1])     1 <= i <= n-2
    const T *ihe;  // 1/(g[i+1]-g[i-1])     1 <= i <= n-2
    const T *ihv;  // 1/(g[i+1]-g[i])       i <= n-2
};

// Everything a stencil kernel needs about one level, passed by value.
template <typename T>
struct LevelView {
    int nx, ny, nz;
    int n;
    Axis<T> ax, ay, az;
    const float *ec, *exy, *exz, *eyz;  // per-stencil viscosity (float storage)
    double clamp_lo, clamp_hi;          // applied to ec.. when do_clamp (level-0 FP64 rows)
    int do_clamp;
    const uint8_t *bcm;                 // boundary mask per node
    int pin;                            // pinned pressure cell node, -1 if none
};

// Plain loads (not __ldg), as everywhere in the stencils below.
template <typename T>
__device__ __forceinline__ T eta_at(const LevelView<T> &L, const float *a, int i)
{
    T v = (T)a[i];
    if (L.do_clamp) {
        if (v > (T)L.clamp_hi) v = (T)L.clamp_hi;
        if (v < (T)L.clamp_lo) v = (T)L.clamp_lo;
    }
    return v;
}

// Read-only access to the 4 unknown fields in storage type S, computed in T.
template <typename T, typename S>
struct Fields {
    const S *p, *vx, *vy, *vz;
};

template <typename T, typename S>
__device__ __forceinline__ T ld(const S *a, int i)
{
    return (T)a[i];
}

#define P2IDX(L, i, j, k) ((k) * ((L).nx * (L).ny) + (i) * (L).ny + (j))

// The stencils below read the unknowns and viscosities through an accessor
// A with A.u(c, a, b, cc) (unknown c = 0 P, 1 Vx, 2 Vy, 3 Vz at node
// (a, b, cc)) and A.e(f, a, b, cc) (viscosity field f = 0 ec, 1 exy, 2 exz,
// 3 eyz, clamped as eta_at does), so the same expressions run on global
// arrays (NodeAcc) and on planes staged in shared memory (k_rows_zm).  The
// rows take their stresses from A.snn / A.sxy / A.sxz / A.syz: NodeAcc
// computes them in place, k_rows_zm reads them from planes of stresses that
// it computed once per cell and edge with the same expressions.
template <typename T, typename A>
__device__ __forceinline__ void cell_rates_a(const LevelView<T> &L, const A &X, int a, int b, int c, T &dxx, T &dyy,
                                             T &dzz)
{
    dxx = (X.u(1, a, b - 1, c - 1) - X.u(1, a - 1, b - 1, c - 1)) * L.ax.ih[a];
    dyy = (X.u(2, a - 1, b, c - 1) - X.u(2, a - 1, b - 1, c - 1)) * L.ay.ih[b];
    dzz = (X.u(3, a - 1, b - 1, c) - X.u(3, a - 1, b - 1, c - 1)) * L.az.ih[c];
}

// Normal stress component d (0 xx, 1 yy, 2 zz) in cell (a,b,c).
template <typename T, typename A>
__device__ __forceinline__ T snn_a(const LevelView<T> &L, const A &X, int d, int a, int b, int c)
{
    T dxx, dyy, dzz;
    cell_rates_a(L, X, a, b, c, dxx, dyy, dzz);
    T div3 = (dxx + dyy + dzz) / (T)3.0;
    T e = d == 0 ? dxx : (d == 1 ? dyy : dzz);
    return (T)2.0 * X.e(0, a, b, c) * (e - div3);
}

template <typename T, typename A>
__device__ __forceinline__ T sxy_a(const LevelView<T> &L, const A &X, int a, int b, int c)
{
    return (T)2.0 * X.e(1, a, b, c) *
           ((X.u(1, a, b, c) - X.u(1, a, b - 1, c)) * L.ay.ihe[b] + (X.u(2, a, b, c) - X.u(2, a - 1, b, c)) * L.ax.ihe[a]);
}
template <typename T, typename A>
__device__ __forceinline__ T sxz_a(const LevelView<T> &L, const A &X, int a, int b, int c)
{
    return (T)2.0 * X.e(2, a, b, c) *
           ((X.u(1, a, b, c) - X.u(1, a, b, c - 1)) * L.az.ihe[c] + (X.u(3, a, b, c) - X.u(3, a - 1, b, c)) * L.ax.ihe[a]);
}
template <typename T, typename A>
__device__ __forceinline__ T syz_a(const LevelView<T> &L, const A &X, int a, int b, int c)
{
    return (T)2.0 * X.e(3, a, b, c) *
           ((X.u(2, a, b, c) - X.u(2, a, b, c - 1)) * L.az.ihe[c] + (X.u(3, a, b, c) - X.u(3, a, b - 1, c)) * L.ay.ihe[b]);
}

// Accessor on global arrays; its stresses are computed where they are used.
template <typename T, typename S>
struct NodeAcc {
    const LevelView<T> &L;
    const Fields<T, S> &x;
    __device__ __forceinline__ T u(int c, int a, int b, int cc) const
    {
        const S *p = c == 0 ? x.p : (c == 1 ? x.vx : (c == 2 ? x.vy : x.vz));
        return ld<T>(p, P2IDX(L, a, b, cc));
    }
    __device__ __forceinline__ T e(int f, int a, int b, int cc) const
    {
        const float *p = f == 0 ? L.ec : (f == 1 ? L.exy : (f == 2 ? L.exz : L.eyz));
        return eta_at(L, p, P2IDX(L, a, b, cc));
    }
    __device__ __forceinline__ T snn(int d, int a, int b, int cc) const { return snn_a(L, *this, d, a, b, cc); }
    __device__ __forceinline__ T sxy(int a, int b, int cc) const { return sxy_a(L, *this, a, b, cc); }
    __device__ __forceinline__ T sxz(int a, int b, int cc) const { return sxz_a(L, *this, a, b, cc); }
    __device__ __forceinline__ T syz(int a, int b, int cc) const { return syz_a(L, *this, a, b, cc); }
};

// The rows take the stresses from the accessor (X.snn .. X.syz) and the
// pressures and velocities from X.u.
template <typename T, typename A>
__device__ __forceinline__ T row_vx_a(const LevelView<T> &L, const A &X, int i, int j, int k)
{
    return (X.snn(0, i + 1, j + 1, k + 1) - X.snn(0, i, j + 1, k + 1)) * L.ax.ihc[i] +
           (X.sxy(i, j + 1, k) - X.sxy(i, j, k)) * L.ay.ihv[j] +
           (X.sxz(i, j, k + 1) - X.sxz(i, j, k)) * L.az.ihv[k] -
           (X.u(0, i + 1, j + 1, k + 1) - X.u(0, i, j + 1, k + 1)) * L.ax.ihc[i];
}
template <typename T, typename A>
__device__ __forceinline__ T row_vy_a(const LevelView<T> &L, const A &X, int i, int j, int k)
{
    return (X.snn(1, i + 1, j + 1, k + 1) - X.snn(1, i + 1, j, k + 1)) * L.ay.ihc[j] +
           (X.sxy(i + 1, j, k) - X.sxy(i, j, k)) * L.ax.ihv[i] +
           (X.syz(i, j, k + 1) - X.syz(i, j, k)) * L.az.ihv[k] -
           (X.u(0, i + 1, j + 1, k + 1) - X.u(0, i + 1, j, k + 1)) * L.ay.ihc[j];
}
template <typename T, typename A>
__device__ __forceinline__ T row_vz_a(const LevelView<T> &L, const A &X, int i, int j, int k)
{
    return (X.snn(2, i + 1, j + 1, k + 1) - X.snn(2, i + 1, j + 1, k)) * L.az.ihc[k] +
           (X.sxz(i + 1, j, k) - X.sxz(i, j, k)) * L.ax.ihv[i] +
           (X.syz(i, j + 1, k) - X.syz(i, j, k)) * L.ay.ihv[j] -
           (X.u(0, i + 1, j + 1, k + 1) - X.u(0, i + 1, j + 1, k)) * L.az.ihc[k];
}
template <typename T, typename A>
__device__ __forceinline__ T row_p_a(const LevelView<T> &L, const A &X, int i, int j, int k)
{
    return (X.u(1, i, j - 1, k - 1) - X.u(1, i - 1, j - 1, k - 1)) * L.ax.ih[i] +
           (X.u(2, i - 1, j, k - 1) - X.u(2, i - 1, j - 1, k - 1)) * L.ay.ih[j] +
           (X.u(3, i - 1, j - 1, k) - X.u(3, i - 1, j - 1, k - 1)) * L.az.ih[k];
}

// The same on global arrays.
template <typename T, typename S>
__device__ __forceinline__ void cell_rates(const LevelView<T> &L, const Fields<T, S> &x, int a, int b, int c,
                                           T &dxx, T &dyy, T &dzz)
{
    cell_rates_a(L, NodeAcc<T, S>{L, x}, a, b, c, dxx, dyy, dzz);
}
template <typename T, typename S>
__device__ __forceinline__ T snn(const LevelView<T> &L, const Fields<T, S> &x, int d, int a, int b, int c)
{
    return snn_a(L, NodeAcc<T, S>{L, x}, d, a, b, c);
}
template <typename T, typename S>
__device__ __forceinline__ T sxy(const LevelView<T> &L, const Fields<T, S> &x, int a, int b, int c)
{
    return sxy_a(L, NodeAcc<T, S>{L, x}, a, b, c);
}
template <typename T, typename S>
__device__ __forceinline__ T sxz(const LevelView<T> &L, const Fields<T, S> &x, int a, int b, int c)
{
    return sxz_a(L, NodeAcc<T, S>{L, x}, a, b, c);
}
template <typename T, typename S>
__device__ __forceinline__ T syz(const LevelView<T> &L, const Fields<T, S> &x, int a, int b, int c)
{
    return syz_a(L, NodeAcc<T, S>{L, x}, a, b, c);
}

// Diagonals of the x-, y-, z-Stokes rows at node (i,j,k).
template <typename T>
__device__ __forceinline__ T diag_vx(const LevelView<T> &L, int i, int j, int k)
{
    return -(L.ax.ihc[i] * (T)(4.0 / 3.0) *
                 (eta_at(L, L.ec, P2IDX(L, i + 1, j + 1, k + 1)) * L.ax.ih[i + 1] +
                  eta_at(L, L.ec, P2IDX(L, i, j + 1, k + 1)) * L.ax.ih[i]) +
             L.ay.ihv[j] * (T)2.0 *
                 (eta_at(L, L.exy, P2IDX(L, i, j + 1, k)) * L.ay.ihe[j + 1] +
                  eta_at(L, L.exy, P2IDX(L, i, j, k)) * L.ay.ihe[j]) +
             L.az.ihv[k] * (T)2.0 *
                 (eta_at(L, L.exz, P2IDX(L, i, j, k + 1)) * L.az.ihe[k + 1] +
                  eta_at(L, L.exz, P2IDX(L, i, j, k)) * L.az.ihe[k]));
}
template <typename T>
__device__ __forceinline__ T diag_vy(const LevelView<T> &L, int i, int j, int k)
{
    return -(L.ay.ihc[j] * (T)(4.0 / 3.0) *
                 (eta_at(L, L.ec, P2IDX(L, i + 1, j + 1, k + 1)) * L.ay.ih[j + 1] +
                  eta_at(L, L.ec, P2IDX(L, i + 1, j, k + 1)) * L.ay.ih[j]) +
             L.ax.ihv[i] * (T)2.0 *
                 (eta_at(L, L.exy, P2IDX(L, i + 1, j, k)) * L.ax.ihe[i + 1] +
                  eta_at(L, L.exy, P2IDX(L, i, j, k)) * L.ax.ihe[i]) +
             L.az.ihv[k] * (T)2.0 *
                 (eta_at(L, L.eyz, P2IDX(L, i, j, k + 1)) * L.az.ihe[k + 1] +
                  eta_at(L, L.eyz, P2IDX(L, i, j, k)) * L.az.ihe[k]));
}
template <typename T>
__device__ __forceinline__ T diag_vz(const LevelView<T> &L, int i, int j, int k)
{
    return -(L.az.ihc[k] * (T)(4.0 / 3.0) *
                 (eta_at(L, L.ec, P2IDX(L, i + 1, j + 1, k + 1)) * L.az.ih[k + 1] +
                  eta_at(L, L.ec, P2IDX(L, i + 1, j + 1, k)) * L.az.ih[k]) +
             L.ax.ihv[i] * (T)2.0 *
                 (eta_at(L, L.exz, P2IDX(L, i + 1, j, k)) * L.ax.ihe[i + 1] +
                  eta_at(L, L.exz, P2IDX(L, i, j, k)) * L.ax.ihe[i]) +
             L.ay.ihv[j] * (T)2.0 *
                 (eta_at(L, L.eyz, P2IDX(L, i, j + 1, k)) * L.ay.ihe[j + 1] +
                  eta_at(L, L.eyz, P2IDX(L, i, j, k)) * L.ay.ihe[j]));
}

template <typename T, typename S>
__device__ __forceinline__ T row_vx(const LevelView<T> &L, const Fields<T, S> &x, int i, int j, int k, T *diag)
{
    T v = row_vx_a(L, NodeAcc<T, S>{L, x}, i, j, k);
    if (diag) *diag = diag_vx(L, i, j, k);
    return v;
}
template <typename T, typename S>
__device__ __forceinline__ T row_vy(const LevelView<T> &L, const Fields<T, S> &x, int i, int j, int k, T *diag)
{
    T v = row_vy_a(L, NodeAcc<T, S>{L, x}, i, j, k);
    if (diag) *diag = diag_vy(L, i, j, k);
    return v;
}
template <typename T, typename S>
__device__ __forceinline__ T row_vz(const LevelView<T> &L, const Fields<T, S> &x, int i, int j, int k, T *diag)
{
    T v = row_vz_a(L, NodeAcc<T, S>{L, x}, i, j, k);
    if (diag) *diag = diag_vz(L, i, j, k);
    return v;
}
template <typename T, typename S>
__device__ __forceinline__ T row_p(const LevelView<T> &L, const Fields<T, S> &x, int i, int j, int k)
{
    return row_p_a(L, NodeAcc<T, S>{L, x}, i, j, k);
}

__host__ __device__ __forceinline__ bool valid_pos(int c, int i, int j, int k, int nx, int ny, int nz)
{
    if (c == 0) return i > 0 && j > 0 && k > 0;
    if (c == 1) return j < ny - 1 && k < nz - 1;
    if (c == 2) return i < nx - 1 && k < nz - 1;
    return i < nx - 1 && j < ny - 1;
}

// Device vector of 4 node fields (P, Vx, Vy, Vz) in one allocation.
template <typename T>
struct Vec4 {
    T *c[4] = {nullptr, nullptr, nullptr, nullptr};
    int n = 0;
};


// Per-axis transfer tables (built on the host from the reference's index
// rules) and reduction job descriptors, shared by the kernels and the host.
constexpr int kRedBlocks = 592;  // 4 x 148 SMs
struct AxisMap {
    const int *lo;
    const double *w0, *w1;
    // inverse lists: coarse index I -> fine (idx, weight)
    const int *ptr, *idx;
    const double *w;
};
// type per axis: 0 node-located, 1 mid-located, 2 pressure cell centre
struct TransferView {
    AxisMap m[3][3];  // [axis][type]
};

struct DotJob {
    const double *a[4];
    const double *b[4];
};
constexpr int kMaxDots = 20;
struct DotJobs {
    DotJob j[kMaxDots];
    int nd;
};

struct VecList {
    const double *v[kMaxDots][4];
    int nv;
};
}  // namespace p2
