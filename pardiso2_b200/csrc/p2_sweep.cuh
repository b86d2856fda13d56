// Fused sweep of the stored-factor cell-block smoother: both colours of one
// sweep in one launch, so that a sweep reads the level's fields once.
//
// The two colour passes of k_vanka_stored, each followed by the boundary
// rows (k_bc_set_chain), compute
//   S1 = red pass of S0, then the boundary rows of S1 (from S1's targets);
//   S2 = black pass of S1.
// Here a block owns a tile of kSwTX x kSwTY cells in (x, y) and a chunk of
// cell planes in z, and marches upwards in z.  At step s it
//   1. loads node plane s of S0 (the four unknowns and the boundary mask)
//      over its tile plus a halo into a ring of kSwRing planes in shared
//      memory (the ring holds S1 as it is being formed);
//   2. relaxes the red cells of cell plane s over the tile plus a ring of
//      one cell (those cells' updates are also computed by the neighbouring
//      tiles; the arithmetic is the same, so the results are identical),
//      reading S0 from global memory and writing the updated faces and
//      pressures into the ring;
//   3. sets the boundary rows of node plane s - 2 in the ring (their targets,
//      within one node, are final red values by then);
//   4. relaxes the black cells of cell plane s - 3 of the tile from the ring
//      (S1) and writes their faces and pressures, and the red cells'
//      pressures, to the output fields (S2).
// The lags follow from the stencil: a cell (i, j, k) reads nodes
// [i-2, i+1] x [j-2, j+1] x [k-2, k+1] and writes its faces at node planes
// k-1 and k; node plane p of S1 is final after the red cells of planes p and
// p + 1.  The boundary rows of S2 are set afterwards by k_bc_set_chain on the
// output, as after the black pass.  The input S0 is never written during the
// sweep (the output is a second buffer), so the overlapping tiles and chunks
// read consistent data.  Chunks start 3 planes early (red cells and boundary
// rows only) to rebuild the S1 planes below them.
//
// Requirements (checked on the host per level): every boundary row's resolved
// target lies within one node of its unknown in each axis.
#pragma once

#include "p2_kernels.cuh"

namespace p2 {

constexpr int kSwTX = 16, kSwTY = 16;               // cells per tile, x and y
constexpr int kSwRX = kSwTX + 5, kSwRY = kSwTY + 5;  // nodes of the shared region: [I0-3, I0+TX+1]
constexpr int kSwRing = 6;                           // node planes held
constexpr int kSwThreads = 256;
constexpr int kSwPlaneNodes = kSwRX * kSwRY;

template <typename T>
constexpr size_t sweep_smem_bytes()
{
    return sizeof(T) * kSwRing * 4 * kSwPlaneNodes + kSwRing * kSwPlaneNodes;
}

// boundary rows of a level by node: the rows of node u are order[first[u] ..]
// in component order (one per set bit of the node's mask); row indices refer
// to the depth-sorted arrays bu / bt / bk / bnext of k_bc_set_chain
struct SweepBC {
    const int *first, *order;
    const int *bu, *bt, *bnext;
    const float *bk;
};

__device__ __forceinline__ int sw_ring(int p) { return (p + 4 * kSwRing) % kSwRing; }

// per-stencil viscosity field f (0 ec, 1 exy, 2 exz, 3 eyz) of a level
template <typename T>
__device__ __forceinline__ const float *eta_field(const LevelView<T> &L, int f)
{
    return f == 0 ? L.ec : (f == 1 ? L.exy : (f == 2 ? L.exz : L.eyz));
}

// unknowns read from global memory, addressed from the cell's low corner F;
// viscosities from global memory
template <typename T>
struct GlobalAcc {
    const T *c[4];
    int F, sy, sz;
    __device__ __forceinline__ T v(int comp, int dx, int dy, int dz) const
    {
        return __ldg(c[comp] + F + dx * sy + dy + dz * sz);
    }
    __device__ __forceinline__ T eta(const LevelView<T> &L, int f, int dx, int dy, int dz) const
    {
        return eta_at(L, eta_field(L, f), F + dx * sy + dy + dz * sz);
    }
};

// unknowns read from the shared ring: F at region coordinates (fx, fy), plane
// fz (F itself is the node index of the cell's low corner); viscosities from
// global memory
template <typename T>
struct RingAcc {
    const T *B;
    int fx, fy, fz;
    int F, sy, sz;
    __device__ __forceinline__ T v(int comp, int dx, int dy, int dz) const
    {
        return B[((sw_ring(fz + dz) * 4 + comp) * kSwRX + fx + dx) * kSwRY + fy + dy];
    }
    __device__ __forceinline__ T eta(const LevelView<T> &L, int f, int dx, int dy, int dz) const
    {
        return eta_at(L, eta_field(L, f), F + dx * sy + dy + dz * sz);
    }
};

// cell_rows with the unknowns and the viscosities taken from an accessor
// (same terms and order)
template <typename T, typename Acc>
__device__ __forceinline__ void cell_rows_acc(const LevelView<T> &L, const Acc &A, int i, int j, int k, T ax[6],
                                              T &div)
{
    const T vx0 = A.v(1, 0, 0, 0), vxX = A.v(1, 1, 0, 0), vxXX = A.v(1, 2, 0, 0), vxm = A.v(1, -1, 0, 0);
    const T vxY = A.v(1, 0, 1, 0), vxy_ = A.v(1, 0, -1, 0), vxXY = A.v(1, 1, 1, 0), vxXy = A.v(1, 1, -1, 0);
    const T vxZ = A.v(1, 0, 0, 1), vxz_ = A.v(1, 0, 0, -1), vxXZ = A.v(1, 1, 0, 1), vxXz = A.v(1, 1, 0, -1);
    const T vy0 = A.v(2, 0, 0, 0), vyY = A.v(2, 0, 1, 0), vyYY = A.v(2, 0, 2, 0), vym = A.v(2, 0, -1, 0);
    const T vyX = A.v(2, 1, 0, 0), vyx_ = A.v(2, -1, 0, 0), vyXY = A.v(2, 1, 1, 0), vyxY = A.v(2, -1, 1, 0);
    const T vyZ = A.v(2, 0, 0, 1), vyz_ = A.v(2, 0, 0, -1), vyYZ = A.v(2, 0, 1, 1), vyYz = A.v(2, 0, 1, -1);
    const T vz0 = A.v(3, 0, 0, 0), vzZ = A.v(3, 0, 0, 1), vzZZ = A.v(3, 0, 0, 2), vzm = A.v(3, 0, 0, -1);
    const T vzX = A.v(3, 1, 0, 0), vzx_ = A.v(3, -1, 0, 0), vzXZ = A.v(3, 1, 0, 1), vzxZ = A.v(3, -1, 0, 1);
    const T vzY = A.v(3, 0, 1, 0), vzy_ = A.v(3, 0, -1, 0), vzYZ = A.v(3, 0, 1, 1), vzyZ = A.v(3, 0, -1, 1);
    const T third = (T)(1.0 / 3.0), two = (T)2.0;
    const T hx0 = L.ax.ih[i - 1], hx1 = L.ax.ih[i], hx2 = L.ax.ih[i + 1];
    const T hy0 = L.ay.ih[j - 1], hy1 = L.ay.ih[j], hy2 = L.ay.ih[j + 1];
    const T hz0 = L.az.ih[k - 1], hz1 = L.az.ih[k], hz2 = L.az.ih[k + 1];
    const T exx = (vxX - vx0) * hx1, eyy = (vyY - vy0) * hy1, ezz = (vzZ - vz0) * hz1;
    div = exx + eyy + ezz;
    const T E2 = two * A.eta(L, 0, 1, 1, 1);
    const T s0 = E2 * (exx - div * third), s1 = E2 * (eyy - div * third), s2 = E2 * (ezz - div * third);
    T sL, sR, sF, sB, sD, sU;
    {
        const T a = (vx0 - vxm) * hx0, b = (vyxY - vyx_) * hy1, c = (vzxZ - vzx_) * hz1;
        sL = two * A.eta(L, 0, 0, 1, 1) * (a - (a + b + c) * third);
    }
    {
        const T a = (vxXX - vxX) * hx2, b = (vyXY - vyX) * hy1, c = (vzXZ - vzX) * hz1;
        sR = two * A.eta(L, 0, 2, 1, 1) * (a - (a + b + c) * third);
    }
    {
        const T a = (vxXy - vxy_) * hx1, b = (vy0 - vym) * hy0, c = (vzyZ - vzy_) * hz1;
        sF = two * A.eta(L, 0, 1, 0, 1) * (b - (a + b + c) * third);
    }
    {
        const T a = (vxXY - vxY) * hx1, b = (vyYY - vyY) * hy2, c = (vzYZ - vzY) * hz1;
        sB = two * A.eta(L, 0, 1, 2, 1) * (b - (a + b + c) * third);
    }
    {
        const T a = (vxXz - vxz_) * hx1, b = (vyYz - vyz_) * hy1, c = (vz0 - vzm) * hz0;
        sD = two * A.eta(L, 0, 1, 1, 0) * (c - (a + b + c) * third);
    }
    {
        const T a = (vxXZ - vxZ) * hx1, b = (vyYZ - vyZ) * hy1, c = (vzZZ - vzZ) * hz2;
        sU = two * A.eta(L, 0, 1, 1, 2) * (c - (a + b + c) * third);
    }
    const T ex0 = L.ax.ihe[i - 1], ex1 = L.ax.ihe[i], ey0 = L.ay.ihe[j - 1], ey1 = L.ay.ihe[j];
    const T ez0 = L.az.ihe[k - 1], ez1 = L.az.ihe[k];
    const T xy00 = two * A.eta(L, 1, 0, 0, 0) * ((vx0 - vxy_) * ey0 + (vy0 - vyx_) * ex0);
    const T xy01 = two * A.eta(L, 1, 0, 1, 0) * ((vxY - vx0) * ey1 + (vyY - vyxY) * ex0);
    const T xy10 = two * A.eta(L, 1, 1, 0, 0) * ((vxX - vxXy) * ey0 + (vyX - vy0) * ex1);
    const T xy11 = two * A.eta(L, 1, 1, 1, 0) * ((vxXY - vxX) * ey1 + (vyXY - vyY) * ex1);
    const T xz00 = two * A.eta(L, 2, 0, 0, 0) * ((vx0 - vxz_) * ez0 + (vz0 - vzx_) * ex0);
    const T xz01 = two * A.eta(L, 2, 0, 0, 1) * ((vxZ - vx0) * ez1 + (vzZ - vzxZ) * ex0);
    const T xz10 = two * A.eta(L, 2, 1, 0, 0) * ((vxX - vxXz) * ez0 + (vzX - vz0) * ex1);
    const T xz11 = two * A.eta(L, 2, 1, 0, 1) * ((vxXZ - vxX) * ez1 + (vzXZ - vzZ) * ex1);
    const T yz00 = two * A.eta(L, 3, 0, 0, 0) * ((vy0 - vyz_) * ez0 + (vz0 - vzy_) * ey0);
    const T yz01 = two * A.eta(L, 3, 0, 0, 1) * ((vyZ - vy0) * ez1 + (vzZ - vzyZ) * ey0);
    const T yz10 = two * A.eta(L, 3, 0, 1, 0) * ((vyY - vyYz) * ez0 + (vzY - vz0) * ey1);
    const T yz11 = two * A.eta(L, 3, 0, 1, 1) * ((vyYZ - vyY) * ez1 + (vzYZ - vzZ) * ey1);
    const T p0 = A.v(0, 1, 1, 1), pL = A.v(0, 0, 1, 1), pR = A.v(0, 2, 1, 1), pF = A.v(0, 1, 0, 1);
    const T pB = A.v(0, 1, 2, 1), pD = A.v(0, 1, 1, 0), pU = A.v(0, 1, 1, 2);
    const T cx0 = L.ax.ihc[i - 1], cx1 = L.ax.ihc[i], cy0 = L.ay.ihc[j - 1], cy1 = L.ay.ihc[j];
    const T cz0 = L.az.ihc[k - 1], cz1 = L.az.ihc[k];
    const T wx = L.ax.ihv[i - 1], wy = L.ay.ihv[j - 1], wz = L.az.ihv[k - 1];
    ax[0] = (s0 - sL) * cx0 + (xy01 - xy00) * wy + (xz01 - xz00) * wz - (p0 - pL) * cx0;
    ax[1] = (sR - s0) * cx1 + (xy11 - xy10) * wy + (xz11 - xz10) * wz - (pR - p0) * cx1;
    ax[2] = (s1 - sF) * cy0 + (xy10 - xy00) * wx + (yz01 - yz00) * wz - (p0 - pF) * cy0;
    ax[3] = (sB - s1) * cy1 + (xy11 - xy01) * wx + (yz11 - yz10) * wz - (pB - p0) * cy1;
    ax[4] = (s2 - sD) * cz0 + (xz10 - xz00) * wx + (yz10 - yz00) * wy - (p0 - pD) * cz0;
    ax[5] = (sU - s2) * cz1 + (xz11 - xz01) * wx + (yz11 - yz01) * wy - (pU - p0) * cz1;
}

// The k_vanka_stored update of cell (i, j, k) with the unknowns from A and the
// face masks from m (bits of the six faces' nodes): the new face values
// vnew[q] (valid where act[q]) and the new pressure pnew.
template <typename T, typename Acc>
__device__ __forceinline__ void vanka_update(const LevelView<T> &L, const Acc &A, int i, int j, int k, int F,
                                             const uint8_t fm[6], const factor_t<T> *__restrict__ blk, long stride,
                                             long t,
                                             const Vec4<T> &b, T omega, T vnew[6], bool act[6], T &pnew)
{
    const int sy = L.ny, sz = L.nx * L.ny;
    const int fc[6] = {1, 1, 2, 2, 3, 3};
    const int fi[6] = {F, F + sy, F, F + 1, F, F + sz};
    T ax[6], div;
    cell_rows_acc(L, A, i, j, k, ax, div);
    const T hx = L.ax.ih[i], hy = L.ay.ih[j], hz = L.az.ih[k];
    const T cc[6] = {-hx, hx, -hy, hy, -hz, hz};
    T v[6];
    face_volumes(L, i, j, k, v);
    T vr[6];
#pragma unroll
    for (int q = 0; q < 6; q++) {
        act[q] = !(fm[q] & (1 << fc[q]));
        vr[q] = act[q] ? (__ldg(b.c[fc[q]] + fi[q]) - ax[q]) * v[q] : (T)0;
    }
    T y1[6] = {0, 0, 0, 0, 0, 0}, y2[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int a = 0; a < 6; a++) {
#pragma unroll
        for (int c = a; c < 6; c++) {
            const T m = ld_factor(blk + (long)tri_index(a, c) * stride + t);
            y1[a] += m * vr[c];
            y2[a] += m * cc[c];
            if (c != a) {
                y1[c] += m * vr[a];
                y2[c] += m * cc[a];
            }
        }
    }
    const T inv = ld_factor(blk + 21L * stride + t);
    const T pold = A.v(0, 1, 1, 1);
    T dp = 0;
    pnew = pold;
    if (inv != (T)0) {
        T num = -(__ldg(b.c[0] + F + sz + sy + 1) - div);
#pragma unroll
        for (int q = 0; q < 6; q++) num += cc[q] * y1[q];
        dp = num * inv;
        pnew = pold + omega * dp;
    }
    const T vold[6] = {A.v(1, 0, 0, 0), A.v(1, 1, 0, 0), A.v(2, 0, 0, 0), A.v(2, 0, 1, 0), A.v(3, 0, 0, 0),
                       A.v(3, 0, 0, 1)};
#pragma unroll
    for (int q = 0; q < 6; q++) vnew[q] = vold[q] + omega * (y1[q] - dp * y2[q]);
}

// slot of cell (i, j, k) in its colour's factor arrays (colour_cell inverse:
// on each line a colour's cells start at j = 1 or 2 and step by 2, so the
// slot within the line is (j - 1) / 2 for either colour)
__device__ __forceinline__ long colour_slot(int nx, int ny, int i, int j, int k)
{
    const int half = ny / 2;
    return ((long)(k - 1) * (nx - 1) + (i - 1)) * half + (j - 1) / 2;
}

// One sweep x_in (S0) -> x_out (S2) as described at the top of this file.
// grid (ceil((nx-1)/kSwTX), ceil((ny-1)/kSwTY), ceil((nz-1)/chunk)); red is
// colour 0 ((i + j + k) even), black colour 1.
template <typename T>
__global__ void __launch_bounds__(kSwThreads) k_vanka_sweep(LevelView<T> L, Vec4<T> xin, Vec4<T> xout, Vec4<T> b,
                                                           T omega, const factor_t<T> *__restrict__ blk0,
                                                           const factor_t<T> *__restrict__ blk1, long stride, SweepBC bc,
                                                           int chunk)
{
    pdl_enter();
    extern __shared__ __align__(16) unsigned char sw_smem[];
    T *B = reinterpret_cast<T *>(sw_smem);
    uint8_t *M = sw_smem + sizeof(T) * kSwRing * 4 * kSwPlaneNodes;
    const int nx = L.nx, ny = L.ny, nz = L.nz, sy = ny, sz = nx * ny;
    const int I0 = 1 + blockIdx.x * kSwTX, J0 = 1 + blockIdx.y * kSwTY;
    const int X0 = I0 - 3, Y0 = J0 - 3;
    const int k0 = 1 + blockIdx.z * chunk;
    const int k1 = min(nz, k0 + chunk);  // black cell planes [k0, k1)
    for (int e = threadIdx.x; e < kSwRing * kSwPlaneNodes; e += blockDim.x) M[e] = 0;
    __syncthreads();
    // node plane p of S0 into its ring slot (zeros outside the level)
    auto load_plane = [&](int p) {
        const int slot = sw_ring(p);
        for (int e = threadIdx.x; e < kSwPlaneNodes; e += blockDim.x) {
            const int xr = e / kSwRY, yr = e - xr * kSwRY;
            const int x = X0 + xr, y = Y0 + yr;
            const bool in = p >= 0 && p < nz && x >= 0 && x < nx && y >= 0 && y < ny;
            const long u = in ? (long)p * sz + (long)x * sy + y : 0;
#pragma unroll
            for (int c = 0; c < 4; c++) B[(slot * 4 + c) * kSwPlaneNodes + e] = in ? xin.c[c][u] : (T)0;
            M[slot * kSwPlaneNodes + e] = in ? L.bcm[u] : (uint8_t)0;
        }
    };
    auto mask_at = [&](int x, int y, int z) -> uint8_t { return M[sw_ring(z) * kSwPlaneNodes + (x - X0) * kSwRY + (y - Y0)]; };
    load_plane(k0 - 4);
    for (int s = k0 - 3; s <= k1 + 2; s++) {
        load_plane(s);
        __syncthreads();
        // 2. red cells of plane s over the tile and a ring of one cell, S0 -> ring
        if (s >= 1 && s <= nz - 1) {
            constexpr int rw = (kSwTY + 2) / 2;
            const int t = threadIdx.x;
            if (t < (kSwTX + 2) * rw) {
                const int i = I0 - 1 + t / rw;
                const int j = J0 - 1 + 2 * (t % rw) + ((i + J0 - 1 + s) & 1);
                if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 1) {
                    const int F = (s - 1) * sz + (i - 1) * sy + (j - 1);
                    GlobalAcc<T> A{{xin.c[0], xin.c[1], xin.c[2], xin.c[3]}, F, sy, sz};
                    const uint8_t fm[6] = {mask_at(i - 1, j - 1, s - 1), mask_at(i, j - 1, s - 1),
                                           mask_at(i - 1, j - 1, s - 1), mask_at(i - 1, j, s - 1),
                                           mask_at(i - 1, j - 1, s - 1), mask_at(i - 1, j - 1, s)};
                    T vn[6], pn;
                    bool act[6];
                    vanka_update(L, A, i, j, s, F, fm, blk0, stride, colour_slot(nx, ny, i, j, s), b, omega, vn,
                                 act, pn);
                    const int xr = i - 1 - X0, yr = j - 1 - Y0;  // F in region coordinates
                    const int fx[6] = {xr, xr + 1, xr, xr, xr, xr}, fy[6] = {yr, yr, yr, yr + 1, yr, yr};
                    const int fz[6] = {s - 1, s - 1, s - 1, s - 1, s - 1, s};
                    const int fcmp[6] = {1, 1, 2, 2, 3, 3};
#pragma unroll
                    for (int q = 0; q < 6; q++)
                        if (act[q]) B[((sw_ring(fz[q]) * 4 + fcmp[q]) * kSwRX + fx[q]) * kSwRY + fy[q]] = vn[q];
                    B[(sw_ring(s) * 4 * kSwRX + xr + 1) * kSwRY + yr + 1] = pn;
                }
            }
        }
        __syncthreads();
        // 3. boundary rows of node plane s - 2 over the black cells' reach
        const int p = s - 2;
        if (p >= k0 - 2 && p <= k1 && p >= 0 && p <= nz - 1) {
            const int slot = sw_ring(p);
            constexpr int bw = kSwTY + 3;
            for (int e = threadIdx.x; e < (kSwTX + 3) * bw; e += blockDim.x) {
                const int xr = 1 + e / bw, yr = 1 + e % bw;
                const uint8_t mm = M[slot * kSwPlaneNodes + xr * kSwRY + yr] & 0xF;
                if (!mm) continue;
                const long u = (long)p * sz + (long)(X0 + xr) * sy + (Y0 + yr);
                int q = __ldg(bc.first + u);
#pragma unroll 1
                for (int c = 0; c < 4; c++) {
                    if (!(mm & (1 << c))) continue;
                    int chain[kMaxBcChain];
                    int m = 0, r = __ldg(bc.order + q);
                    q++;
                    chain[m++] = r;
                    while (__ldg(bc.bnext + r) >= 0 && m < kMaxBcChain) {
                        r = __ldg(bc.bnext + r);
                        chain[m++] = r;
                    }
                    const int tt = __ldg(bc.bt + r);
                    T v = 0;
                    if (tt >= 0) {
                        const int tn = tt >> 2, tz = tn / sz, tx = (tn - tz * sz) / sy, ty = tn - tz * sz - tx * sy;
                        v = (T)__ldg(bc.bk + r) * B[((sw_ring(tz) * 4 + (tt & 3)) * kSwRX + tx - X0) * kSwRY + ty - Y0];
                    }
                    int uc = __ldg(bc.bu + r);
                    v = __ldg(b.c[uc & 3] + (uc >> 2)) + v;
                    for (int s2 = m - 2; s2 >= 0; s2--) {
                        const int rr = chain[s2];
                        uc = __ldg(bc.bu + rr);
                        v = __ldg(b.c[uc & 3] + (uc >> 2)) + (T)__ldg(bc.bk + rr) * v;
                    }
                    B[((slot * 4 + c) * kSwRX + xr) * kSwRY + yr] = v;
                }
            }
        }
        __syncthreads();
        // 4. black cells of plane s - 3 of the tile, ring (S1) -> output; the
        //    red cells' pressures of that plane, ring -> output
        const int kb = s - 3;
        if (kb >= k0 && kb < k1) {
            constexpr int bw = kSwTY / 2, nb = kSwTX * bw;
            const int t = threadIdx.x;
            const bool black = t < nb;
            const int tt = black ? t : t - nb;
            if (tt < nb) {
                const int i = I0 + tt / bw;
                const int j = J0 + 2 * (tt % bw) + ((i + J0 + kb + (black ? 1 : 0)) & 1);
                if (i <= nx - 1 && j <= ny - 1) {
                    const int xr = i - 1 - X0, yr = j - 1 - Y0;
                    const int F = (kb - 1) * sz + (i - 1) * sy + (j - 1);
                    if (black) {
                        RingAcc<T> A{B, xr, yr, kb - 1, F, sy, sz};
                        const uint8_t fm[6] = {mask_at(i - 1, j - 1, kb - 1), mask_at(i, j - 1, kb - 1),
                                               mask_at(i - 1, j - 1, kb - 1), mask_at(i - 1, j, kb - 1),
                                               mask_at(i - 1, j - 1, kb - 1), mask_at(i - 1, j - 1, kb)};
                        T vn[6], pn;
                        bool act[6];
                        vanka_update(L, A, i, j, kb, F, fm, blk1, stride, colour_slot(nx, ny, i, j, kb), b, omega, vn,
                                     act, pn);
                        const int fo[6] = {F, F + sy, F, F + 1, F, F + sz};
                        const int fcmp[6] = {1, 1, 2, 2, 3, 3};
#pragma unroll
                        for (int q = 0; q < 6; q++)
                            if (act[q]) xout.c[fcmp[q]][fo[q]] = vn[q];
                        xout.c[0][F + sz + sy + 1] = pn;
                    } else {
                        xout.c[0][F + sz + sy + 1] = B[(sw_ring(kb) * 4 * kSwRX + xr + 1) * kSwRY + yr + 1];
                    }
                }
            }
        }
        __syncthreads();
    }
}

}  // namespace p2
