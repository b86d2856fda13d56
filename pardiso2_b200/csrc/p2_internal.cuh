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

// Plain loads (not __ldg): the row functions below also run on level views
// whose arrays are shared-memory copies of a brick (k_rows_tiled).
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

template <typename T, typename S>
__device__ __forceinline__ void cell_rates(const LevelView<T> &L, const Fields<T, S> &x, int a, int b, int c,
                                           T &dxx, T &dyy, T &dzz)
{
    dxx = (ld<T>(x.vx, P2IDX(L, a, b - 1, c - 1)) - ld<T>(x.vx, P2IDX(L, a - 1, b - 1, c - 1))) * L.ax.ih[a];
    dyy = (ld<T>(x.vy, P2IDX(L, a - 1, b, c - 1)) - ld<T>(x.vy, P2IDX(L, a - 1, b - 1, c - 1))) * L.ay.ih[b];
    dzz = (ld<T>(x.vz, P2IDX(L, a - 1, b - 1, c)) - ld<T>(x.vz, P2IDX(L, a - 1, b - 1, c - 1))) * L.az.ih[c];
}

// Normal stress component d (0 xx, 1 yy, 2 zz) in cell (a,b,c).
template <typename T, typename S>
__device__ __forceinline__ T snn(const LevelView<T> &L, const Fields<T, S> &x, int d, int a, int b, int c)
{
    T dxx, dyy, dzz;
    cell_rates(L, x, a, b, c, dxx, dyy, dzz);
    T div3 = (dxx + dyy + dzz) / (T)3.0;
    T e = d == 0 ? dxx : (d == 1 ? dyy : dzz);
    return (T)2.0 * eta_at(L, L.ec, P2IDX(L, a, b, c)) * (e - div3);
}

template <typename T, typename S>
__device__ __forceinline__ T sxy(const LevelView<T> &L, const Fields<T, S> &x, int a, int b, int c)
{
    return (T)2.0 * eta_at(L, L.exy, P2IDX(L, a, b, c)) *
           ((ld<T>(x.vx, P2IDX(L, a, b, c)) - ld<T>(x.vx, P2IDX(L, a, b - 1, c))) * L.ay.ihe[b] +
            (ld<T>(x.vy, P2IDX(L, a, b, c)) - ld<T>(x.vy, P2IDX(L, a - 1, b, c))) * L.ax.ihe[a]);
}
template <typename T, typename S>
__device__ __forceinline__ T sxz(const LevelView<T> &L, const Fields<T, S> &x, int a, int b, int c)
{
    return (T)2.0 * eta_at(L, L.exz, P2IDX(L, a, b, c)) *
           ((ld<T>(x.vx, P2IDX(L, a, b, c)) - ld<T>(x.vx, P2IDX(L, a, b, c - 1))) * L.az.ihe[c] +
            (ld<T>(x.vz, P2IDX(L, a, b, c)) - ld<T>(x.vz, P2IDX(L, a - 1, b, c))) * L.ax.ihe[a]);
}
template <typename T, typename S>
__device__ __forceinline__ T syz(const LevelView<T> &L, const Fields<T, S> &x, int a, int b, int c)
{
    return (T)2.0 * eta_at(L, L.eyz, P2IDX(L, a, b, c)) *
           ((ld<T>(x.vy, P2IDX(L, a, b, c)) - ld<T>(x.vy, P2IDX(L, a, b, c - 1))) * L.az.ihe[c] +
            (ld<T>(x.vz, P2IDX(L, a, b, c)) - ld<T>(x.vz, P2IDX(L, a, b - 1, c))) * L.ay.ihe[b]);
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
    T v = (snn(L, x, 0, i + 1, j + 1, k + 1) - snn(L, x, 0, i, j + 1, k + 1)) * L.ax.ihc[i] +
          (sxy(L, x, i, j + 1, k) - sxy(L, x, i, j, k)) * L.ay.ihv[j] +
          (sxz(L, x, i, j, k + 1) - sxz(L, x, i, j, k)) * L.az.ihv[k] -
          (ld<T>(x.p, P2IDX(L, i + 1, j + 1, k + 1)) - ld<T>(x.p, P2IDX(L, i, j + 1, k + 1))) * L.ax.ihc[i];
    if (diag) *diag = diag_vx(L, i, j, k);
    return v;
}
template <typename T, typename S>
__device__ __forceinline__ T row_vy(const LevelView<T> &L, const Fields<T, S> &x, int i, int j, int k, T *diag)
{
    T v = (snn(L, x, 1, i + 1, j + 1, k + 1) - snn(L, x, 1, i + 1, j, k + 1)) * L.ay.ihc[j] +
          (sxy(L, x, i + 1, j, k) - sxy(L, x, i, j, k)) * L.ax.ihv[i] +
          (syz(L, x, i, j, k + 1) - syz(L, x, i, j, k)) * L.az.ihv[k] -
          (ld<T>(x.p, P2IDX(L, i + 1, j + 1, k + 1)) - ld<T>(x.p, P2IDX(L, i + 1, j, k + 1))) * L.ay.ihc[j];
    if (diag) *diag = diag_vy(L, i, j, k);
    return v;
}
template <typename T, typename S>
__device__ __forceinline__ T row_vz(const LevelView<T> &L, const Fields<T, S> &x, int i, int j, int k, T *diag)
{
    T v = (snn(L, x, 2, i + 1, j + 1, k + 1) - snn(L, x, 2, i + 1, j + 1, k)) * L.az.ihc[k] +
          (sxz(L, x, i + 1, j, k) - sxz(L, x, i, j, k)) * L.ax.ihv[i] +
          (syz(L, x, i, j + 1, k) - syz(L, x, i, j, k)) * L.ay.ihv[j] -
          (ld<T>(x.p, P2IDX(L, i + 1, j + 1, k + 1)) - ld<T>(x.p, P2IDX(L, i + 1, j + 1, k))) * L.az.ihc[k];
    if (diag) *diag = diag_vz(L, i, j, k);
    return v;
}
template <typename T, typename S>
__device__ __forceinline__ T row_p(const LevelView<T> &L, const Fields<T, S> &x, int i, int j, int k)
{
    return (ld<T>(x.vx, P2IDX(L, i, j - 1, k - 1)) - ld<T>(x.vx, P2IDX(L, i - 1, j - 1, k - 1))) * L.ax.ih[i] +
           (ld<T>(x.vy, P2IDX(L, i - 1, j, k - 1)) - ld<T>(x.vy, P2IDX(L, i - 1, j - 1, k - 1))) * L.ay.ih[j] +
           (ld<T>(x.vz, P2IDX(L, i - 1, j - 1, k)) - ld<T>(x.vz, P2IDX(L, i - 1, j - 1, k - 1))) * L.az.ih[k];
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
