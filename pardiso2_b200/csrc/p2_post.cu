// Post-solve fields of vpiterate (pardiso/move3mgNew.c:2908-3038 and
// 3293-3316): deviatoric stresses sxx..syz and strain rates exx..eyz on level
// 0 from the float velocities the solve hands back, and the velocity ranges
// that bound the marker time step.
//
// Each value is the reference's value-mode stencil (sxxcalc .. syzcalc with
// ynval = 0, move3mgNew.c:3-130, 132-257, 259-386, 388-518, 520-657,
// 659-794): a float difference of two velocities, scaled in double by the
// reciprocal gridline distance, combined and multiplied by 2 nueff (the
// level-0 stencil viscosity clamped to [nubeg, nuend]), stored as float.
// The arithmetic is spelled out with round-to-nearest intrinsics (no fused
// multiply-add), so every stored value equals the reference's bit for bit.
// Positions the reference does not write (non-periodic box) are left as
// they are.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>

#include "p2_internal.cuh"
#include "p2_solver.h"

namespace p2 {

namespace {

inline unsigned nblocks(long n, int t) { return (unsigned)((n + t - 1) / t); }

struct PostOut {
    float *s[6];  // sxx syy szz sxy sxz syz
    float *e[6];  // exx eyy ezz exy exz eyz
};

__device__ __forceinline__ double nu_clamped(float v, double nubeg, double nuend)
{
    double n = (double)v;
    if (n > nuend) n = nuend;
    if (n < nubeg) n = nubeg;
    return n;
}

// d(float difference) * kf, with the difference rounded to float first
__device__ __forceinline__ double fdiff(float a, float b, double kf) { return __dmul_rn((double)__fsub_rn(a, b), kf); }

__device__ __forceinline__ void put(float *s, float *e, long u, double left, double nueff)
{
    if (e) e[u] = __double2float_rn(left);
    if (s) s[u] = __double2float_rn(__dmul_rn(__dmul_rn(2.0, nueff), left));
}

__global__ void k_stress_strain(Grid3 G, const float *vx, const float *vy, const float *vz, const float *nxx,
                                const float *nxy, const float *nxz, const float *nyz, double nubeg, double nuend,
                                PostOut o)
{
    const int nx = G.n[0], ny = G.n[1], nz = G.n[2];
    const long nxy_ = (long)nx * ny;
    const long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nxy_ * nz) return;
    const int m2 = (int)(u % ny), m1 = (int)((u / ny) % nx), m3 = (int)(u / nxy_);
    const double *gx = G.g[0], *gy = G.g[1], *gz = G.g[2];
    // normal components: cell with upper corner at this node (sxxcalc..szzcalc)
    if (m1 > 0 && m2 > 0 && m3 > 0) {
        const double xkf = __ddiv_rn(1.0, __dsub_rn(gx[m1], gx[m1 - 1]));
        const double ykf = __ddiv_rn(1.0, __dsub_rn(gy[m2], gy[m2 - 1]));
        const double zkf = __ddiv_rn(1.0, __dsub_rn(gz[m3], gz[m3 - 1]));
        const long v0 = u - nxy_ - ny - 1;
        const double dvxdx = fdiff(vx[v0 + ny], vx[v0], xkf);
        const double dvydy = fdiff(vy[v0 + 1], vy[v0], ykf);
        const double dvzdz = fdiff(vz[v0 + nxy_], vz[v0], zkf);
        const double div3 = __ddiv_rn(__dadd_rn(__dadd_rn(dvxdx, dvydy), dvzdz), 3.0);
        const double nueff = nu_clamped(nxx[u], nubeg, nuend);
        put(o.s[0], o.e[0], u, __dsub_rn(dvxdx, div3), nueff);
        put(o.s[1], o.e[1], u, __dsub_rn(dvydy, div3), nueff);
        put(o.s[2], o.e[2], u, __dsub_rn(dvzdz, div3), nueff);
    }
    // xy: z-edge (sxycalc); v3 is this node, v2 one y back, v1 one x back
    if (m1 > 0 && m1 < nx - 1 && m2 > 0 && m2 < ny - 1 && m3 < nz - 1) {
        const double xkf = __ddiv_rn(1.0, __dsub_rn(gx[m1 + 1], gx[m1 - 1]));
        const double ykf = __ddiv_rn(1.0, __dsub_rn(gy[m2 + 1], gy[m2 - 1]));
        const double left = __dadd_rn(fdiff(vx[u], vx[u - 1], ykf), fdiff(vy[u], vy[u - ny], xkf));
        put(o.s[3], o.e[3], u, left, nu_clamped(nxy[u], nubeg, nuend));
    }
    // xz: y-edge (sxzcalc); v6 this node, v2 one z back, v4 one x back
    if (m1 > 0 && m1 < nx - 1 && m3 > 0 && m3 < nz - 1 && m2 < ny - 1) {
        const double xkf = __ddiv_rn(1.0, __dsub_rn(gx[m1 + 1], gx[m1 - 1]));
        const double zkf = __ddiv_rn(1.0, __dsub_rn(gz[m3 + 1], gz[m3 - 1]));
        const double left = __dadd_rn(fdiff(vx[u], vx[u - nxy_], zkf), fdiff(vz[u], vz[u - ny], xkf));
        put(o.s[4], o.e[4], u, left, nu_clamped(nxz[u], nubeg, nuend));
    }
    // yz: x-edge (syzcalc); v5 this node, v1 one z back, v4 one y back
    if (m2 > 0 && m2 < ny - 1 && m3 > 0 && m3 < nz - 1 && m1 < nx - 1) {
        const double ykf = __ddiv_rn(1.0, __dsub_rn(gy[m2 + 1], gy[m2 - 1]));
        const double zkf = __ddiv_rn(1.0, __dsub_rn(gz[m3 + 1], gz[m3 - 1]));
        const double left = __dadd_rn(fdiff(vy[u], vy[u - nxy_], zkf), fdiff(vz[u], vz[u - 1], ykf));
        put(o.s[5], o.e[5], u, left, nu_clamped(nyz[u], nubeg, nuend));
    }
}

// min / max of vx, vy, vz over their valid positions (move3mgNew.c:2862-2890);
// per-block partials, then one block folds them (order-free: min and max are
// exact)
constexpr int kRangeThreads = 256;
constexpr int kRangeBlocks = 296;  // two per SM

__global__ void __launch_bounds__(kRangeThreads) k_vrange_partial(int nx, int ny, int nz, const float *vx,
                                                                  const float *vy, const float *vz, float *partial)
{
    __shared__ float sh[6][kRangeThreads / 32];
    float r[6] = {FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX};
    const long n = (long)nx * ny * nz;
    for (long u = (long)blockIdx.x * blockDim.x + threadIdx.x; u < n; u += (long)gridDim.x * blockDim.x) {
        const int j = (int)(u % ny), i = (int)((u / ny) % nx), k = (int)(u / ((long)nx * ny));
        const float *v[3] = {vx, vy, vz};
#pragma unroll
        for (int c = 0; c < 3; c++)
            if (valid_pos(c + 1, i, j, k, nx, ny, nz)) {
                const float a = v[c][u];
                r[2 * c] = fminf(r[2 * c], a);
                r[2 * c + 1] = fmaxf(r[2 * c + 1], a);
            }
    }
#pragma unroll
    for (int q = 0; q < 6; q++)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const float o = __shfl_xor_sync(0xffffffffu, r[q], off);
            r[q] = (q & 1) ? fmaxf(r[q], o) : fminf(r[q], o);
        }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
        for (int q = 0; q < 6; q++) sh[q][w] = r[q];
    __syncthreads();
    if (threadIdx.x < 6) {
        const int q = threadIdx.x;
        float a = sh[q][0];
        for (int x = 1; x < kRangeThreads / 32; x++) a = (q & 1) ? fmaxf(a, sh[q][x]) : fminf(a, sh[q][x]);
        partial[(long)blockIdx.x * 6 + q] = a;
    }
}

__global__ void k_vrange_final(int nparts, const float *partial, double *out)
{
    const int q = threadIdx.x;
    if (q >= 6) return;
    float a = (q & 1) ? -FLT_MAX : FLT_MAX;
    for (int b = 0; b < nparts; b++) a = (q & 1) ? fmaxf(a, partial[b * 6 + q]) : fminf(a, partial[b * 6 + q]);
    out[q] = (double)a;
}

}  // namespace

// Stress and strain-rate fields from the last solution: in/out host arrays
// (nullptr skips a field), vrange = {min vx, max vx, min vy, max vy, min vz,
// max vz} over the valid velocity positions.
void Solver::stress_strain(float *const s[6], float *const e[6], double vrange[6])
{
    if (!solution_ready) throw Error(P2_ERR_STATE, "stress and strain rates before a solve");
    if (!nodes_ready) throw Error(P2_ERR_STATE, "no node viscosities");
    ensure_move_buffers(0);
    const Level &L0 = L[0];
    const long n = L0.n;
    if (!post_out[0]) {
        for (int q = 0; q < 12; q++) post_out[q] = (float *)post_arena.alloc(sizeof(float) * n);
        post_partial = (float *)post_arena.alloc(sizeof(float) * 6 * kRangeBlocks);
        post_range = (double *)post_arena.alloc(sizeof(double) * 6);
    }
    velocity_f32();
    PostOut o;
    for (int q = 0; q < 6; q++) {
        float *const hs = s ? s[q] : nullptr, *const he = e ? e[q] : nullptr;
        o.s[q] = hs ? post_out[q] : nullptr;
        o.e[q] = he ? post_out[6 + q] : nullptr;
        // positions the reference leaves alone keep the caller's values
        if (hs) P2_CUDA_TRY(cudaMemcpyAsync(o.s[q], hs, sizeof(float) * n, cudaMemcpyHostToDevice, st));
        if (he) P2_CUDA_TRY(cudaMemcpyAsync(o.e[q], he, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    }
    k_stress_strain<<<nblocks(n, 256), 256, 0, st>>>(grid3(), mv_vel[0], mv_vel[1], mv_vel[2], f0.nxx, f0.nxy,
                                                     f0.nxz, f0.nyz, prm.nubeg, prm.nuend, o); P2_COUNT_LAUNCH();
    k_vrange_partial<<<kRangeBlocks, kRangeThreads, 0, st>>>(L0.nx, L0.ny, L0.nz, mv_vel[0], mv_vel[1], mv_vel[2],
                                                             post_partial); P2_COUNT_LAUNCH();
    k_vrange_final<<<1, 32, 0, st>>>(kRangeBlocks, post_partial, post_range); P2_COUNT_LAUNCH();
    P2_CUDA_TRY(cudaGetLastError());
    for (int q = 0; q < 6; q++) {
        if (o.s[q]) P2_CUDA_TRY(cudaMemcpyAsync(s[q], o.s[q], sizeof(float) * n, cudaMemcpyDeviceToHost, st));
        if (o.e[q]) P2_CUDA_TRY(cudaMemcpyAsync(e[q], o.e[q], sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    }
    double r[6];
    P2_CUDA_TRY(cudaMemcpyAsync(r, post_range, sizeof(r), cudaMemcpyDeviceToHost, st));
    P2_CUDA_TRY(cudaStreamSynchronize(st));
    if (vrange)
        for (int q = 0; q < 6; q++) vrange[q] = r[q];
}

}  // namespace p2
