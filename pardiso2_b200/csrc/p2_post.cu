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

// ---------------------------------------------------------------------------
// Effective bulk viscosity diagnostics (effbulkvisccalc mode 1,
// pardiso/mark3mg.c:2-150): over the level-0 nodes with ro > 1500 (and index
// > 0 on every axis), the strain-rate and stress invariants of the cell
// behind the node (shear terms averaged over the cell's four edges of each
// orientation), their visco-plastic variant, the dissipation, the averages
// of the tensor components split into inclusions (ro > 3850) and matrix, and
// the harmonic mean of nxx.  Per-node values follow the reference's float /
// double mix operation by operation; the sums are taken per block and then
// in block order (deterministic, a different order from the reference's
// sequential loop).
constexpr int kBulkSums = 30;  // see k_effbulk for the slots
constexpr int kBulkBlocks = 296;

struct BulkIn {
    const float *ro, *nxx, *nxy, *nxz, *nyz;
    const float *e[6], *s[6];  // exx eyy ezz exy exz eyz, sxx .. syz
};

__device__ __forceinline__ float sq(float a) { return __fmul_rn(a, a); }
// (a[0]^2 + a[1]^2 + a[2]^2 + a[3]^2) / 4 in float
__device__ __forceinline__ float avg_sq4(float a, float b, float c, float d)
{
    return __fdiv_rn(__fadd_rn(__fadd_rn(__fadd_rn(sq(a), sq(b)), sq(c)), sq(d)), 4.0f);
}
// (a + b + c + d) / 4 in float
__device__ __forceinline__ float avg4(float a, float b, float c, float d)
{
    return __fdiv_rn(__fadd_rn(__fadd_rn(__fadd_rn(a, b), c), d), 4.0f);
}
// pow(s / 2 / n, 2): the quotient in float, squared in double
__device__ __forceinline__ double vp2(float s, float n)
{
    const double q = (double)__fdiv_rn(__fdiv_rn(s, 2.0f), n);
    return __dmul_rn(q, q);
}
// s * s / 2 / n in float
__device__ __forceinline__ float heat1(float s, float n) { return __fdiv_rn(__fdiv_rn(sq(s), 2.0f), n); }

__global__ void __launch_bounds__(256) k_effbulk(int nx, int ny, int nz, BulkIn in, double *partial)
{
    // slots: 0 eiin, 1 tau2, 2 siin, 3 hsn, 4 eiivp, 5 nubulkn, 6 numtot, 7 numinc, 8 nummat,
    //        9..14 inclusion exx..eyz, 15..20 inclusion sxx..syz, 21..26 matrix exx..eyz,
    //        27..29 matrix sxx, syy, szz (the matrix shear stresses go to 30..32 below)
    __shared__ double sh[32];
    double acc[kBulkSums + 3];
#pragma unroll
    for (int q = 0; q < kBulkSums + 3; q++) acc[q] = 0;
    const long n = (long)nx * ny * nz, sxy_ = ny, sz = (long)nx * ny;
    for (long m4 = (long)blockIdx.x * blockDim.x + threadIdx.x; m4 < n; m4 += (long)gridDim.x * blockDim.x) {
        const int m2 = (int)(m4 % ny), m1 = (int)((m4 / ny) % nx), m3 = (int)(m4 / sz);
        if (!((double)in.ro[m4] > 1500 && m1 > 0 && m2 > 0 && m3 > 0)) continue;
        const long v0 = m4 - sz - sxy_ - 1, v1 = v0 + 1, v2 = v0 + sxy_, v3 = v2 + 1, v4 = v0 + sz, v5 = v4 + 1,
                   v6 = v4 + sxy_;
        const float *const *e = in.e, *const *s = in.s;
        const float nxx = in.nxx[m4];
        acc[6] += 1;
        acc[5] = __dadd_rn(acc[5], (double)__fdiv_rn(1.0f, nxx));
        // strain-rate and stress second invariants
        const double Exy = avg_sq4(e[3][v0], e[3][v1], e[3][v2], e[3][v3]);
        const double Exz = avg_sq4(e[4][v0], e[4][v2], e[4][v4], e[4][v6]);
        const double Eyz = avg_sq4(e[5][v0], e[5][v1], e[5][v4], e[5][v5]);
        const double Sxy = avg_sq4(s[3][v0], s[3][v1], s[3][v2], s[3][v3]);
        const double Sxz = avg_sq4(s[4][v0], s[4][v2], s[4][v4], s[4][v6]);
        const double Syz = avg_sq4(s[5][v0], s[5][v1], s[5][v4], s[5][v5]);
        const double ne = (double)__fadd_rn(__fadd_rn(sq(e[0][m4]), sq(e[1][m4])), sq(e[2][m4]));
        const double ns = (double)__fadd_rn(__fadd_rn(sq(s[0][m4]), sq(s[1][m4])), sq(s[2][m4]));
        const double eii = __dsqrt_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(0.5, ne), Exy), Exz), Eyz));
        const double sii = __dsqrt_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(0.5, ns), Sxy), Sxz), Syz));
        // visco-plastic strain rate from the stresses
        const float *nxy = in.nxy, *nxz = in.nxz, *nyz = in.nyz;
        const double Vxy = __ddiv_rn(__dadd_rn(__dadd_rn(__dadd_rn(vp2(s[3][v0], nxy[v0]), vp2(s[3][v1], nxy[v1])),
                                                         vp2(s[3][v2], nxy[v2])), vp2(s[3][v3], nxy[v3])), 4.0);
        const double Vxz = __ddiv_rn(__dadd_rn(__dadd_rn(__dadd_rn(vp2(s[4][v0], nxz[v0]), vp2(s[4][v2], nxz[v2])),
                                                         vp2(s[4][v4], nxz[v4])), vp2(s[4][v6], nxz[v6])), 4.0);
        const double Vyz = __ddiv_rn(__dadd_rn(__dadd_rn(__dadd_rn(vp2(s[5][v0], nyz[v0]), vp2(s[5][v1], nyz[v1])),
                                                         vp2(s[5][v4], nyz[v4])), vp2(s[5][v5], nyz[v5])), 4.0);
        const double vn = __dadd_rn(__dadd_rn(vp2(s[0][m4], nxx), vp2(s[1][m4], nxx)), vp2(s[2][m4], nxx));
        const double eiivp = __dsqrt_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(0.5, vn), Vxy), Vxz), Vyz));
        // dissipation
        const double Hxy = avg4(heat1(s[3][v0], nxy[v0]), heat1(s[3][v1], nxy[v1]), heat1(s[3][v2], nxy[v2]),
                                heat1(s[3][v3], nxy[v3]));
        const double Hxz = avg4(heat1(s[4][v0], nxz[v0]), heat1(s[4][v2], nxz[v2]), heat1(s[4][v4], nxz[v4]),
                                heat1(s[4][v6], nxz[v6]));
        const double Hyz = avg4(heat1(s[5][v0], nyz[v0]), heat1(s[5][v1], nyz[v1]), heat1(s[5][v4], nyz[v4]),
                                heat1(s[5][v5], nyz[v5]));
        const double hs = __dadd_rn((double)__fdiv_rn(__fdiv_rn(__fadd_rn(__fadd_rn(sq(s[0][m4]), sq(s[1][m4])),
                                                                          sq(s[2][m4])), 2.0f), nxx),
                                    __dmul_rn(2.0, __dadd_rn(__dadd_rn(Hxy, Hxz), Hyz)));
        acc[0] = __dadd_rn(acc[0], eii);
        acc[1] = __dadd_rn(acc[1], __dmul_rn((double)nxx, eii));
        acc[2] = __dadd_rn(acc[2], sii);
        acc[3] = __dadd_rn(acc[3], hs);
        acc[4] = __dadd_rn(acc[4], eiivp);
        // tensor components: inclusions (ro > 3850) or matrix
        const int base = (double)in.ro[m4] > 3850 ? 9 : 21;
        acc[(double)in.ro[m4] > 3850 ? 7 : 8] += 1;
        const float comp[12] = {e[0][m4], e[1][m4], e[2][m4], avg4(e[3][v0], e[3][v1], e[3][v2], e[3][v3]),
                                avg4(e[4][v0], e[4][v2], e[4][v4], e[4][v6]), avg4(e[5][v0], e[5][v1], e[5][v4], e[5][v5]),
                                s[0][m4], s[1][m4], s[2][m4], avg4(s[3][v0], s[3][v1], s[3][v2], s[3][v3]),
                                avg4(s[4][v0], s[4][v2], s[4][v4], s[4][v6]), avg4(s[5][v0], s[5][v1], s[5][v4], s[5][v5])};
#pragma unroll
        for (int q = 0; q < 12; q++) {
            const int slot = base + q;  // 21..32 for the matrix
            acc[slot] = __dadd_rn(acc[slot], (double)comp[q]);
        }
    }
#pragma unroll
    for (int q = 0; q < kBulkSums + 3; q++) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
            partial[(long)q * gridDim.x + blockIdx.x] = t;
        }
        __syncthreads();
    }
}

__global__ void k_effbulk_final(int nparts, const double *partial, double *out)
{
    const int q = threadIdx.x;
    if (q >= kBulkSums + 3) return;
    double t = 0;
    for (int b = 0; b < nparts; b++) t += partial[(long)q * nparts + b];
    out[q] = t;
}

}  // namespace

// effbulkvisccalc(1) on host arrays of the level-0 node fields; out[] as
// p2_effbulk (include/p2cuda.h).
void Solver::effbulk(const float *ro, const float *nxx, const float *nxy, const float *nxz, const float *nyz,
                     const float *const e[6], const float *const s[6], p2_effbulk *res)
{
    if (!grid_ready) throw Error(P2_ERR_STATE, "diagnostics before p2_set_grid");
    const Level &L0 = L[0];
    const long n = L0.n;
    if (!bulk_in[0]) {
        for (int q = 0; q < 17; q++) bulk_in[q] = (float *)post_arena.alloc(sizeof(float) * n);
        bulk_partial = (double *)post_arena.alloc(sizeof(double) * (kBulkSums + 3) * kBulkBlocks);
        bulk_out = (double *)post_arena.alloc(sizeof(double) * (kBulkSums + 3));
    }
    const float *src[17] = {ro, nxx, nxy, nxz, nyz, e[0], e[1], e[2], e[3], e[4], e[5],
                            s[0], s[1], s[2], s[3], s[4], s[5]};
    for (int q = 0; q < 17; q++) {
        if (!src[q]) throw Error(P2_ERR_ARG, "null node field");
        P2_CUDA_TRY(cudaMemcpyAsync(bulk_in[q], src[q], sizeof(float) * n, cudaMemcpyHostToDevice, st));
    }
    BulkIn in;
    in.ro = bulk_in[0]; in.nxx = bulk_in[1]; in.nxy = bulk_in[2]; in.nxz = bulk_in[3]; in.nyz = bulk_in[4];
    for (int q = 0; q < 6; q++) { in.e[q] = bulk_in[5 + q]; in.s[q] = bulk_in[11 + q]; }
    k_effbulk<<<kBulkBlocks, 256, 0, st>>>(L0.nx, L0.ny, L0.nz, in, bulk_partial); P2_COUNT_LAUNCH();
    k_effbulk_final<<<1, 64, 0, st>>>(kBulkBlocks, bulk_partial, bulk_out); P2_COUNT_LAUNCH();
    P2_CUDA_TRY(cudaGetLastError());
    double a[kBulkSums + 3];
    P2_CUDA_TRY(cudaMemcpyAsync(a, bulk_out, sizeof(a), cudaMemcpyDeviceToHost, st));
    P2_CUDA_TRY(cudaStreamSynchronize(st));
    // the reference's final divisions (mark3mg.c:101-114)
    p2_effbulk r{};
    r.numtot = (long)a[6];
    r.numinc = (long)a[7];
    r.nummat = (long)a[8];
    const double nt = (double)r.numtot;
    r.eiin = a[0] / nt;
    r.tau2 = a[1] / nt;
    r.siin = a[2] / nt;
    r.hsn = a[3] / nt;
    r.eiivp = a[4] / nt;
    r.nubulkn = nt / a[5];
    for (int q = 0; q < 12; q++) {
        r.incl[q] = r.numinc > 0 ? a[9 + q] / (double)r.numinc : 0.0;
        r.matrix[q] = r.nummat > 0 ? a[21 + q] / (double)r.nummat : 0.0;
    }
    r.nubulk1 = r.tau2 / r.eiin;
    r.nubulk2 = r.hsn / 4 / r.eiin / r.eiin;
    r.nubulk3 = r.hsn / 4 / r.eiivp / r.eiivp;
    r.nubulk4 = r.siin / 2 / r.eiin;
    if (res) *res = r;
}

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
