// Operator rows (residual b - A x, or A x) of a level, marching up in z with
// rings of node planes and of stress planes in shared memory.
//
// k_rows evaluates the four rows of a node from global memory, and every row
// recomputes the stresses it differences: the normal stresses of a cell are
// formed six times per node (each with its division of the divergence by 3)
// and each edge stress twice, about 700 instructions and a hundred loads per
// node, which leaves a large level far below the memory bandwidth.  Here a
// block owns a column of TX x TY nodes (y fastest, as the node layout) and a
// chunk of KZ node planes.  Per plane c it computes, once per cell and edge
// of the column (a one-node border on the + sides included), the cell's
// three normal stresses and the three edge stresses (move3mgNew.c:3-794
// through snn_a .. syz_a, the same expressions as k_rows') into a two-slot
// ring of stress planes, and the rows of plane k (move3mgNew.c:796-1576,
// row_vx_a .. row_p_a) are differences of the stresses of planes k and k+1
// and of the pressures and velocities of planes k-1..k+1.  Unknown planes,
// with a one-node halo in x and y, sit in a four-slot ring (slot = plane &
// 3) and viscosity planes in a two-slot ring, both filled by asynchronous
// copies (cp.async): while plane k is evaluated, plane k+2 is in flight.
// Global reads per node: its 4 unknowns and 4 viscosities once (plus the
// halo, (TX+2)(TY+2)/(TX TY) = 1.33x, mostly from L2), its mask byte and,
// for the residual, its 4 right-hand sides.  Results agree with k_rows' to
// rounding (a stress read back from shared memory cannot be contracted into
// a fused multiply-add with the difference that uses it).
#pragma once

#include "p2_internal.cuh"

namespace p2 {

constexpr int kZmTX = 8, kZmTY = 32, kZmKZ = 32;
constexpr int kZmThreads = kZmTX * kZmTY;
constexpr int kZmRX = kZmTX + 2, kZmRY = kZmTY + 2, kZmPlane = kZmRX * kZmRY;  // unknowns, viscosities
constexpr int kZmSX = kZmTX + 1, kZmSY = kZmTY + 1, kZmSPlane = kZmSX * kZmSY;  // stresses

// shared memory of k_rows_zm<T, S>: four slots of 4 unknown planes (S), two
// slots of 4 viscosity planes (float), two slots of 6 stress planes (T)
template <typename T, typename S>
constexpr size_t zm_smem_bytes()
{
    return (size_t)4 * 4 * kZmPlane * sizeof(S) + (size_t)2 * 4 * kZmPlane * sizeof(float) +
           (size_t)2 * 6 * kZmSPlane * sizeof(T);
}

__device__ __forceinline__ void zm_cp_async4(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void zm_cp_async8(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}

// Accessors relative to one node (a0, b0) of plane c0: every access is a
// compile-time offset from one of a few plane pointers held in registers
// (the offsets a - a0, b - b0, cc - c0 are constants once the stencil is
// inlined), so a load costs one shared-memory instruction.
//
// Unknowns of planes c0 - 1, c0 and the viscosities of plane c0 (stress
// computation).
template <typename T, typename S>
struct ZmNodes {
    const LevelView<T> &L;
    const S *um, *u0;  // unknown ring at planes c0 - 1, c0, offset to (a0, b0)
    const float *ep;   // viscosity ring at plane c0, offset to (a0, b0)
    int a0, b0, c0;
    __device__ __forceinline__ T u(int c, int a, int b, int cc) const
    {
        return (T)(cc < c0 ? um : u0)[c * kZmPlane + (a - a0) * kZmRY + (b - b0)];
    }
    __device__ __forceinline__ T e(int f, int a, int b, int cc) const
    {
        (void)cc;  // always c0
        T v = (T)ep[f * kZmPlane + (a - a0) * kZmRY + (b - b0)];
        if (L.do_clamp) {
            if (v > (T)L.clamp_hi) v = (T)L.clamp_hi;
            if (v < (T)L.clamp_lo) v = (T)L.clamp_lo;
        }
        return v;
    }
};

// Unknowns of planes k - 1 .. k + 1 and stresses of planes k, k + 1 around
// node (a0, b0) of plane c0 = k (rows).
template <typename T, typename S>
struct ZmRows {
    const S *um, *u0, *up;  // unknown ring at planes k - 1, k, k + 1, offset to (a0, b0)
    const T *s0, *s1;       // stress ring at planes k, k + 1, offset to (a0, b0)
    int a0, b0, c0;
    __device__ __forceinline__ T u(int c, int a, int b, int cc) const
    {
        return (T)(cc < c0 ? um : (cc == c0 ? u0 : up))[c * kZmPlane + (a - a0) * kZmRY + (b - b0)];
    }
    __device__ __forceinline__ T st(int q, int a, int b, int cc) const
    {
        return (cc == c0 ? s0 : s1)[q * kZmSPlane + (a - a0) * kZmSY + (b - b0)];
    }
    __device__ __forceinline__ T snn(int d, int a, int b, int cc) const { return st(d, a, b, cc); }
    __device__ __forceinline__ T sxy(int a, int b, int cc) const { return st(3, a, b, cc); }
    __device__ __forceinline__ T sxz(int a, int b, int cc) const { return st(4, a, b, cc); }
    __device__ __forceinline__ T syz(int a, int b, int cc) const { return st(5, a, b, cc); }
};

// Per-thread staging slots of a column plane: a thread copies the plane
// elements tid, tid + kZmThreads (kZmStage of them) of every staged plane;
// their x / y offsets and level membership do not change with the plane.
constexpr int kZmStage = (kZmPlane + kZmThreads - 1) / kZmThreads;

// grid (ceil(nx/kZmTX), ceil(ny/kZmTY), ceil(nz/kZmKZ)), kZmThreads threads,
// zm_smem_bytes<T, S>() of dynamic shared memory.  out = b - A x (mode 0) or
// A x (mode 1) on every node of the level; boundary rows and positions that
// are not unknowns get 0 (k_bc_rows sets the boundary rows afterwards), as
// k_rows does.
template <typename T, typename S>
__global__ void __launch_bounds__(kZmThreads) k_rows_zm(LevelView<T> L, Fields<T, S> x, Vec4<T> b, Vec4<T> out,
                                                        Vec4<float> out32, int mode)
{
    pdl_enter();
    extern __shared__ __align__(16) unsigned char zm_smem[];
    S *U = reinterpret_cast<S *>(zm_smem);
    float *E = reinterpret_cast<float *>(U + 4 * 4 * kZmPlane);
    T *SS = reinterpret_cast<T *>(E + 2 * 4 * kZmPlane);
    const int nx = L.nx, ny = L.ny, nz = L.nz, sy = ny, sz = nx * ny;
    const int I0 = blockIdx.x * kZmTX, J0 = blockIdx.y * kZmTY;
    const int K0 = blockIdx.z * kZmKZ, K1 = min(nz, K0 + kZmKZ);
    const int X0 = I0 - 1, Y0 = J0 - 1;
    const S *src[4] = {x.p, x.vx, x.vy, x.vz};
    const float *esrc[4] = {L.ec, L.exy, L.exz, L.eyz};
    // this thread's staging elements: in-plane node offset, or -1 outside
    // the level (or beyond the plane)
    int soff[kZmStage];
#pragma unroll
    for (int q = 0; q < kZmStage; q++) {
        const int e = threadIdx.x + q * kZmThreads;
        const int xr = e / kZmRY, yr = e - xr * kZmRY;
        const int gx = X0 + xr, gy = Y0 + yr;
        soff[q] = (e < kZmPlane && gx >= 0 && gx < nx && gy >= 0 && gy < ny) ? gx * sy + gy : -1;
    }
    // node plane p (-1 <= p <= nz) of the unknowns into ring slot p & 3
    // and, with vis, of the viscosities into slot p & 1; nodes outside the
    // level are zero (only stresses and rows that no computed row uses read
    // them)
    auto stage = [&](int p, bool vis) {
        const bool zin = p >= 0 && p < nz;
        S *ud = U + (p & 3) * 4 * kZmPlane;
        float *ed = E + (p & 1) * 4 * kZmPlane;
        const long pbase = (long)p * sz;
#pragma unroll
        for (int q = 0; q < kZmStage; q++) {
            const int e = threadIdx.x + q * kZmThreads;
            if (e >= kZmPlane) break;
            const bool in = zin && soff[q] >= 0;
            const long u = in ? pbase + soff[q] : 0;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                S *d = ud + c * kZmPlane + e;
                if (in) {
                    if (sizeof(S) == 8) zm_cp_async8(d, src[c] + u);
                    else zm_cp_async4(d, src[c] + u);
                } else {
                    *d = (S)0;
                }
            }
            if (vis) {
#pragma unroll
                for (int f = 0; f < 4; f++) {
                    float *d = ed + f * kZmPlane + e;
                    if (in) zm_cp_async4(d, esrc[f] + u);
                    else *d = 0.0f;
                }
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    // the stresses of node plane c at the positions (a, b) in [I0, I0 + TX] x
    // [J0, J0 + TY] inside the level (0 outside) into stress slot c & 1; they
    // read unknown planes c - 1, c and viscosity plane c
    auto stresses = [&](int c) {
        const S *um = U + ((c - 1) & 3) * 4 * kZmPlane, *u0 = U + (c & 3) * 4 * kZmPlane;
        const float *e0 = E + (c & 1) * 4 * kZmPlane;
        T *sd = SS + (c & 1) * 6 * kZmSPlane;
        for (int e = threadIdx.x; e < kZmSPlane; e += kZmThreads) {
            const int xa = e / kZmSY, yb = e - xa * kZmSY;
            const int a = I0 + xa, bb = J0 + yb;
            T sn[3] = {0, 0, 0}, sxy = 0, sxz = 0, syz = 0;
            if (a < nx && bb < ny && c < nz) {
                const int o = (xa + 1) * kZmRY + (yb + 1);  // ring index of (a, bb)
                const ZmNodes<T, S> N{L, um + o, u0 + o, e0 + o, a, bb, c};
                T dxx, dyy, dzz;
                cell_rates_a(L, N, a, bb, c, dxx, dyy, dzz);
                const T div3 = (dxx + dyy + dzz) / (T)3.0;
                const T e2 = (T)2.0 * N.e(0, a, bb, c);
                sn[0] = e2 * (dxx - div3);
                sn[1] = e2 * (dyy - div3);
                sn[2] = e2 * (dzz - div3);
                sxy = sxy_a(L, N, a, bb, c);
                sxz = sxz_a(L, N, a, bb, c);
                syz = syz_a(L, N, a, bb, c);
            }
            T *d = sd + e;
            d[0] = sn[0];
            d[kZmSPlane] = sn[1];
            d[2 * kZmSPlane] = sn[2];
            d[3 * kZmSPlane] = sxy;
            d[4 * kZmSPlane] = sxz;
            d[5 * kZmSPlane] = syz;
        }
    };
    stage(K0 - 1, false);
    stage(K0, true);
    stage(K0 + 1, true);
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    stresses(K0);
    // the first step's copies of plane K0+2 go to the viscosity slot that
    // stresses(K0) reads
    __syncthreads();
    const int tx = threadIdx.x / kZmTY, ty = threadIdx.x - tx * kZmTY;
    const int i = I0 + tx, j = J0 + ty;
    const bool mine = i < nx && j < ny;
    const int ro = (tx + 1) * kZmRY + (ty + 1), so = tx * kZmSY + ty;  // ring / stress index of (i, j)
    for (int k = K0; k < K1; k++) {
        // node plane k+2 for the next step: its unknown slot held plane k-2
        // and its viscosity slot plane k, both last read before the previous
        // step's final barrier
        if (k + 1 < K1) stage(k + 2, true);
        // stresses of plane k+1 (unknown planes k, k+1, viscosity plane k+1),
        // into the slot of plane k-1's, last read by the previous step's rows
        stresses(k + 1);
        __syncthreads();
        if (mine) {
            const long u = (long)k * sz + (long)i * sy + j;
            const uint8_t m = __ldg(L.bcm + u);
            const ZmRows<T, S> R{U + ((k - 1) & 3) * 4 * kZmPlane + ro, U + (k & 3) * 4 * kZmPlane + ro,
                                 U + ((k + 1) & 3) * 4 * kZmPlane + ro, SS + (k & 1) * 6 * kZmSPlane + so,
                                 SS + ((k + 1) & 1) * 6 * kZmSPlane + so, i, j, k};
#pragma unroll
            for (int c = 0; c < 4; c++) {
                T v = 0;
                if (valid_pos(c, i, j, k, nx, ny, nz) && !(m & (1 << c))) {
                    T ax;
                    if (c == 0) ax = row_p_a(L, R, i, j, k);
                    else if (c == 1) ax = row_vx_a(L, R, i, j, k);
                    else if (c == 2) ax = row_vy_a(L, R, i, j, k);
                    else ax = row_vz_a(L, R, i, j, k);
                    v = mode == 0 ? b.c[c][u] - ax : ax;
                }
                out.c[c][u] = v;
                if (out32.c[0]) out32.c[c][u] = (float)v;
            }
        }
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();
    }
}

}  // namespace p2
