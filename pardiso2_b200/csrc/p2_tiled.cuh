// One colour pass of the stored-factor cell-block smoother with a block's
// unknowns and per-stencil viscosities staged in shared memory.
//
// k_vanka_stored reads each cell's ~45 unknowns and ~20 viscosities with
// separate loads from L1/L2/HBM as the cell's arithmetic needs them; at 72
// registers (7 blocks of 128 threads per SM) its warps wait on those loads
// (long-scoreboard stalls).  Here a block owns a brick of TX x TY x TZ cells
// (y fastest, as the node layout), first copies the nodes the brick's cells
// read — [I0-2, I0+TX] x [J0-2, J0+TY] x [K0-2, K0+TZ], 4 unknowns and 4
// viscosity fields — into shared memory with asynchronous 4- or 8-byte copies
// (cp.async: no register holds the data in flight, so every thread can have
// dozens of loads outstanding; rows along y are contiguous in global memory),
// then relaxes the colour's cells of the brick from shared memory.  The cell
// update (residuals from shared stresses, stored factors, right-hand sides) is
// vanka_update, the same expression sequence as k_vanka_stored; the stored
// factors, right-hand sides and boundary masks are still read from global
// memory (each once per cell).  Reads and writes follow k_vanka_stored:
// velocities from vin, the colour's faces to vout, pressures in place (a
// cell's pressure is read only by its own rows within one colour, so the
// pressures of same-colour cells that a brick also copies are never used).
#pragma once

#include "p2_sweep.cuh"

namespace p2 {

constexpr int kTileThreads = 256;

// brick dimensions per precision (shared memory: 4 unknowns of T and 4
// viscosities of float per node of the brick)
template <typename T>
struct TileShape;
template <>
struct TileShape<float> { static constexpr int TX = 8, TY = 32, TZ = 4; };
template <>
struct TileShape<double> { static constexpr int TX = 8, TY = 32, TZ = 2; };

template <typename T>
constexpr int tile_nodes()
{
    return (TileShape<T>::TX + 3) * (TileShape<T>::TY + 3) * (TileShape<T>::TZ + 3);
}
template <typename T>
constexpr size_t tile_smem_bytes()
{
    return (sizeof(T) * 4 + sizeof(float) * 4) * (size_t)tile_nodes<T>();
}

template <typename T>
struct BrickAcc {
    static constexpr int RX = TileShape<T>::TX + 3, RY = TileShape<T>::TY + 3, RZ = TileShape<T>::TZ + 3;
    const T *S;      // [4][RZ][RX][RY]
    const float *E;  // [4][RZ][RX][RY]
    int fx, fy, fz;  // the cell's low corner F in brick coordinates
    __device__ __forceinline__ T v(int comp, int dx, int dy, int dz) const
    {
        return S[((comp * RZ + fz + dz) * RX + fx + dx) * RY + fy + dy];
    }
    __device__ __forceinline__ T eta(const LevelView<T> &, int f, int dx, int dy, int dz) const
    {
        return (T)E[((f * RZ + fz + dz) * RX + fx + dx) * RY + fy + dy];
    }
};

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// grid (ceil((nx-1)/TX), ceil((ny-1)/TY), ceil((nz-1)/TZ)), kTileThreads
// threads, tile_smem_bytes<T>() of dynamic shared memory.  The level's view
// must not clamp its viscosities (the V-cycle's views do not).
template <typename T>
__global__ void __launch_bounds__(kTileThreads, 2) k_vanka_tiled(LevelView<T> L, T *P, Vec4<T> vin, Vec4<T> vout,
                                                                Vec4<T> b, T omega, int col,
                                                                const factor_t<T> *__restrict__ blk, long stride)
{
    pdl_enter();
    constexpr int TX = TileShape<T>::TX, TY = TileShape<T>::TY, TZ = TileShape<T>::TZ;
    constexpr int RX = TX + 3, RY = TY + 3, RZ = TZ + 3, NN = RX * RY * RZ;
    extern __shared__ __align__(16) unsigned char tile_smem[];
    T *S = reinterpret_cast<T *>(tile_smem);
    float *E = reinterpret_cast<float *>(S + 4 * NN);
    const int nx = L.nx, ny = L.ny, nz = L.nz, sy = ny, sz = nx * ny;
    const int I0 = 1 + blockIdx.x * TX, J0 = 1 + blockIdx.y * TY, K0 = 1 + blockIdx.z * TZ;
    const int X0 = I0 - 2, Y0 = J0 - 2, Z0 = K0 - 2;
    const T *src[4] = {P, vin.c[1], vin.c[2], vin.c[3]};
    const float *esrc[4] = {L.ec, L.exy, L.exz, L.eyz};
    // stage the brick: 8 fields x NN nodes, consecutive threads on consecutive y
    for (int e = threadIdx.x; e < 8 * NN; e += kTileThreads) {
        const int f = e / NN, r = e - f * NN;
        const int zr = r / (RX * RY), r2 = r - zr * (RX * RY), xr = r2 / RY, yr = r2 - xr * RY;
        const int x = X0 + xr, y = Y0 + yr, z = Z0 + zr;
        const bool in = x >= 0 && x < nx && y >= 0 && y < ny && z >= 0 && z < nz;
        const long u = (long)z * sz + (long)x * sy + y;
        if (f < 4) {
            T *d = S + f * NN + r;
            if (in) {
                if (sizeof(T) == 8) cp_async8(d, src[f] + u);
                else cp_async4(d, src[f] + u);
            } else {
                *d = (T)0;
            }
        } else {
            float *d = E + (f - 4) * NN + r;
            if (in) cp_async4(d, esrc[f - 4] + u);
            else *d = 0.0f;
        }
    }
    cp_async_wait_all();
    __syncthreads();
    // the colour's cells of the brick: per z layer and x row, every other y
    constexpr int half = TY / 2, ncell = TX * half * TZ;
    for (int c = threadIdx.x; c < ncell; c += kTileThreads) {
        const int hz = c / (TX * half), rem = c - hz * (TX * half), hx = rem / half, hy = rem - hx * half;
        const int i = I0 + hx, k = K0 + hz;
        const int j = J0 + 2 * hy + ((i + J0 + k + col) & 1);  // (i + j + k) & 1 == col
        if (i > nx - 1 || j > ny - 1 || k > nz - 1) continue;
        const int F = (k - 1) * sz + (i - 1) * sy + (j - 1);
        BrickAcc<T> A{S, E, i - 1 - X0, j - 1 - Y0, k - 1 - Z0};
        const uint8_t fm[6] = {__ldg(L.bcm + F), __ldg(L.bcm + F + sy), __ldg(L.bcm + F), __ldg(L.bcm + F + 1),
                               __ldg(L.bcm + F), __ldg(L.bcm + F + sz)};
        T vn[6], pn;
        bool act[6];
        vanka_update(L, A, i, j, k, F, fm, blk, stride, colour_slot(nx, ny, i, j, k), b, omega, vn, act, pn);
        const int fo[6] = {F, F + sy, F, F + 1, F, F + sz};
        const int fcmp[6] = {1, 1, 2, 2, 3, 3};
#pragma unroll
        for (int q = 0; q < 6; q++)
            if (act[q]) vout.c[fcmp[q]][fo[q]] = vn[q];
        P[F + sz + sy + 1] = pn;
    }
}

}  // namespace p2

namespace p2 {

// k_rows (out = b - A x, or A x) with the brick of nodes a tile's rows read —
// [I0-1, I0+TX] x [J0-1, J0+TY] x [K0-1, K0+TZ], the 4 unknowns and the 4
// viscosity fields — staged in shared memory by cp.async: the row functions
// (row_vx .. row_p) then run unchanged on a level view whose arrays are the
// brick (nx, ny, nz the brick's, spacing tables offset to its origin).  One
// row function reads 20-30 values; from shared memory they no longer wait on
// L2.  Boundary rows and non-unknown positions get 0, as in k_rows.
template <typename S>
struct RowTile {
    static constexpr int TX = 8, TY = 32, TZ = 4;
    static constexpr int RX = TX + 2, RY = TY + 2, RZ = TZ + 2, NN = RX * RY * RZ;
    static constexpr size_t smem = (sizeof(S) * 4 + sizeof(float) * 4) * (size_t)NN;
};

template <typename T>
__device__ __forceinline__ Axis<T> axis_offset(const Axis<T> &a, int o)
{
    return Axis<T>{a.ih + o, a.ihc + o, a.ihe + o, a.ihv + o};
}

template <typename T, typename S>
__global__ void __launch_bounds__(kTileThreads, 2) k_rows_tiled(LevelView<T> L, Fields<T, S> x, Vec4<T> b,
                                                               Vec4<T> out, Vec4<float> out32, int mode)
{
    pdl_enter();
    using RT = RowTile<S>;
    constexpr int TX = RT::TX, TY = RT::TY, TZ = RT::TZ, RX = RT::RX, RY = RT::RY, NN = RT::NN;
    extern __shared__ __align__(16) unsigned char rows_smem[];
    S *X = reinterpret_cast<S *>(rows_smem);
    float *E = reinterpret_cast<float *>(X + 4 * NN);
    const int nx = L.nx, ny = L.ny, nz = L.nz, sy = ny, sz = nx * ny;
    const int I0 = blockIdx.x * TX, J0 = blockIdx.y * TY, K0 = blockIdx.z * TZ;
    const int X0 = I0 - 1, Y0 = J0 - 1, Z0 = K0 - 1;
    const S *src[4] = {x.p, x.vx, x.vy, x.vz};
    const float *esrc[4] = {L.ec, L.exy, L.exz, L.eyz};
    for (int e = threadIdx.x; e < 8 * NN; e += kTileThreads) {
        const int f = e / NN, r = e - f * NN;
        const int zr = r / (RX * RY), r2 = r - zr * (RX * RY), xr = r2 / RY, yr = r2 - xr * RY;
        const int gx = X0 + xr, gy = Y0 + yr, gz = Z0 + zr;
        const bool in = gx >= 0 && gx < nx && gy >= 0 && gy < ny && gz >= 0 && gz < nz;
        const long u = (long)gz * sz + (long)gx * sy + gy;
        if (f < 4) {
            S *d = X + f * NN + r;
            if (in) {
                if (sizeof(S) == 8) cp_async8(d, src[f] + u);
                else cp_async4(d, src[f] + u);
            } else {
                *d = (S)0;
            }
        } else {
            float *d = E + (f - 4) * NN + r;
            if (in) cp_async4(d, esrc[f - 4] + u);
            else *d = 0.0f;
        }
    }
    cp_async_wait_all();
    __syncthreads();
    LevelView<T> LL = L;
    LL.nx = RX;
    LL.ny = RY;
    LL.nz = RT::RZ;
    LL.n = NN;
    LL.ax = axis_offset(L.ax, X0);
    LL.ay = axis_offset(L.ay, Y0);
    LL.az = axis_offset(L.az, Z0);
    LL.ec = E;
    LL.exy = E + NN;
    LL.exz = E + 2 * NN;
    LL.eyz = E + 3 * NN;
    const Fields<T, S> xl{X, X + NN, X + 2 * NN, X + 3 * NN};
    for (int c0 = threadIdx.x; c0 < TX * TY * TZ; c0 += kTileThreads) {
        const int hz = c0 / (TX * TY), rem = c0 - hz * (TX * TY), hx = rem / TY, hy = rem - hx * TY;
        const int i = I0 + hx, j = J0 + hy, k = K0 + hz;
        if (i >= nx || j >= ny || k >= nz) continue;
        const int u = k * sz + i * sy + j;
        const int li = i - X0, lj = j - Y0, lk = k - Z0;
        const uint8_t m = __ldg(L.bcm + u);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            T v = 0;
            if (valid_pos(c, i, j, k, nx, ny, nz) && !(m & (1 << c))) {
                T ax;
                if (c == 0) ax = row_p(LL, xl, li, lj, lk);
                else if (c == 1) ax = row_vx(LL, xl, li, lj, lk, (T *)nullptr);
                else if (c == 2) ax = row_vy(LL, xl, li, lj, lk, (T *)nullptr);
                else ax = row_vz(LL, xl, li, lj, lk, (T *)nullptr);
                v = mode == 0 ? b.c[c][u] - ax : ax;
            }
            out.c[c][u] = v;
            if (out32.c[0]) out32.c[c][u] = (float)v;
        }
    }
}

}  // namespace p2
