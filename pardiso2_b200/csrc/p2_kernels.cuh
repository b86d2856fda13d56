// Stencil, transfer and reduction kernels of the p2cuda Stokes multigrid.
#pragma once

#include "p2_internal.cuh"

namespace p2 {

// Storage type of the stored cell factors of a V-cycle computing in T (the
// cycle's own type: bfloat16 factors for the FP32 cycle were measured to cost
// 26 -> 31 outer iterations at 257^3 for a 1 % faster pass, which is latency-
// rather than bandwidth-bound).
template <typename T>
using factor_t = T;

__device__ __forceinline__ float ld_factor(const float *p) { return __ldg(p); }
__device__ __forceinline__ double ld_factor(const double *p) { return __ldg(p); }
template <typename S>
__device__ __forceinline__ S to_factor(double v) { return (S)v; }

constexpr int kThreads = 256;

// ---------------------------------------------------------------------------
// Rows: out = b - A x (mode 0) or out = A x (mode 1) on every non-boundary
// row; boundary rows and non-unknown positions get 0 here (boundary rows are
// written by k_bc_rows).  Optionally also writes a float copy (the FP32
// right-hand side of the mixed-precision V-cycle).
template <typename T, typename S>
__device__ __forceinline__ void rows_item(const LevelView<T> &L, const Fields<T, S> &x, const Vec4<T> &b,
                                          const Vec4<T> &out, const Vec4<float> &out32, int mode, int u)
{
    if (u >= L.n) return;
    int j = u % L.ny, i = (u / L.ny) % L.nx, k = u / (L.nx * L.ny);
    uint8_t m = L.bcm[u];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        T v = 0;
        if (valid_pos(c, i, j, k, L.nx, L.ny, L.nz) && !(m & (1 << c))) {
            T ax;
            if (c == 0) ax = row_p(L, x, i, j, k);
            else if (c == 1) ax = row_vx(L, x, i, j, k, (T *)nullptr);
            else if (c == 2) ax = row_vy(L, x, i, j, k, (T *)nullptr);
            else ax = row_vz(L, x, i, j, k, (T *)nullptr);
            v = mode == 0 ? b.c[c][u] - ax : ax;
        }
        out.c[c][u] = v;
        if (out32.c[0]) out32.c[c][u] = (float)v;
    }
}
template <typename T, typename S>
__global__ void k_rows(LevelView<T> L, Fields<T, S> x, Vec4<T> b, Vec4<T> out, Vec4<float> out32, int mode)
{
    pdl_enter();
    rows_item(L, x, b, out, out32, mode, blockIdx.x * blockDim.x + threadIdx.x);
}

// Boundary rows x_u = b_u + koef * x_t: residual (mode 0) b_u + koef x_t - x_u,
// or operator (mode 1) x_u - koef x_t.
template <typename T, typename S>
__device__ __forceinline__ void bc_rows_item(int nbc, const int *bu, const int *bt, const float *bk,
                                             const Fields<T, S> &x, const Vec4<T> &b, const Vec4<T> &out,
                                             const Vec4<float> &out32, int mode, int q)
{
    if (q >= nbc) return;
    int uc = bu[q], c = uc & 3, u = uc >> 2, t = bt[q];
    const S *xs[4] = {x.p, x.vx, x.vy, x.vz};
    T xt = t >= 0 ? (T)bk[q] * (T)xs[t & 3][t >> 2] : (T)0;
    T v = mode == 0 ? b.c[c][u] + xt - (T)xs[c][u] : (T)xs[c][u] - xt;
    out.c[c][u] = v;
    if (out32.c[0]) out32.c[c][u] = (float)v;
}
template <typename T, typename S>
__global__ void k_bc_rows(int nbc, const int *bu, const int *bt, const float *bk, Fields<T, S> x, Vec4<T> b,
                          Vec4<T> out, Vec4<float> out32, int mode)
{
    pdl_enter();
    bc_rows_item(nbc, bu, bt, bk, x, b, out, out32, mode, blockIdx.x * blockDim.x + threadIdx.x);
}

// All boundary rows in one launch: each row walks its copy chain (the rows
// owning its successive targets, bnext) and evaluates it from the innermost
// row outwards, x = b + koef * x_target, the same arithmetic as applying the
// chain-depth groups one after another.  Only the final target (a regular
// unknown) is read from x, and each row writes only its own unknown.
constexpr int kMaxBcChain = 8;

template <typename T>
__device__ __forceinline__ void bc_set_chain_item(int nbc, const int *bu, const int *bt, const float *bk,
                                                  const int *bnext, const Vec4<T> &x, const Vec4<T> &b, int q)
{
    if (q >= nbc) return;
    int chain[kMaxBcChain];
    int m = 0, r = q;
    chain[m++] = r;
    while (bnext[r] >= 0 && m < kMaxBcChain) {
        r = bnext[r];
        chain[m++] = r;
    }
    const int t = bt[r];                      // innermost row's target (regular unknown or none)
    T v = t >= 0 ? (T)bk[r] * x.c[t & 3][t >> 2] : (T)0;
    int uc = bu[r];
    v = b.c[uc & 3][uc >> 2] + v;
    for (int s = m - 2; s >= 0; s--) {
        const int rr = chain[s];
        uc = bu[rr];
        v = b.c[uc & 3][uc >> 2] + (T)bk[rr] * v;
    }
    uc = bu[q];
    x.c[uc & 3][uc >> 2] = v;
}
template <typename T>
__global__ void k_bc_set_chain(int nbc, const int *bu, const int *bt, const float *bk, const int *bnext, Vec4<T> x,
                               Vec4<T> b)
{
    pdl_enter();
    bc_set_chain_item(nbc, bu, bt, bk, bnext, x, b, blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------------------
// One colour pass of the cell-block smoother (diagonal Vanka / SCGS) over the
// cells with (i+j+k)&1 == col.  Each cell corrects its six face velocities and
// its pressure together with the velocity block replaced by its diagonal:
//   d_v dv_v + g_v dp = r_v,  sum_v c_v dv_v = r_p.
// Every cell of the colour reads the state from before the pass: velocities
// are read from vin and written to vout (each face belongs to exactly one
// cell of each colour), the pressure is updated in place (a cell's pressure is
// read only by its own face rows among the cells of one colour).
template <typename T>
__device__ __forceinline__ void vanka_item(const LevelView<T> &L, T *P, const Vec4<T> &vin, const Vec4<T> &vout,
                                           const Vec4<T> &b, T omega, int col, long t)
{
    int half = (L.ny) / 2;  // >= number of cells of one colour on a y-line
    long lines = (long)(L.nx - 1) * (L.nz - 1);
    if (t >= lines * half) return;
    int jj = (int)(t % half);
    long line = t / half;
    int i = 1 + (int)(line % (L.nx - 1)), k = 1 + (int)(line / (L.nx - 1));
    int j0 = (((1 + i + k) & 1) == col) ? 1 : 2;
    int j = j0 + 2 * jj;
    if (j > L.ny - 1) return;
    Fields<T, T> x{P, vin.c[1], vin.c[2], vin.c[3]};
    int u = P2IDX(L, i, j, k);
    bool pbc = (L.bcm[u] & BC_P) != 0;
    int fi[6], fc[6];
    T g[6], cc[6], r[6], d[6];
    fc[0] = 1; fi[0] = P2IDX(L, i - 1, j - 1, k - 1); g[0] = -L.ax.ihc[i - 1]; cc[0] = -L.ax.ih[i];
    fc[1] = 1; fi[1] = P2IDX(L, i, j - 1, k - 1);     g[1] = L.ax.ihc[i];      cc[1] = L.ax.ih[i];
    fc[2] = 2; fi[2] = P2IDX(L, i - 1, j - 1, k - 1); g[2] = -L.ay.ihc[j - 1]; cc[2] = -L.ay.ih[j];
    fc[3] = 2; fi[3] = P2IDX(L, i - 1, j, k - 1);     g[3] = L.ay.ihc[j];      cc[3] = L.ay.ih[j];
    fc[4] = 3; fi[4] = P2IDX(L, i - 1, j - 1, k - 1); g[4] = -L.az.ihc[k - 1]; cc[4] = -L.az.ih[k];
    fc[5] = 3; fi[5] = P2IDX(L, i - 1, j - 1, k);     g[5] = L.az.ihc[k];      cc[5] = L.az.ih[k];
    const int ofs[6][3] = {{-1, -1, -1}, {0, -1, -1}, {-1, -1, -1}, {-1, 0, -1}, {-1, -1, -1}, {-1, -1, 0}};
    T num = 0, den = 0;
#pragma unroll
    for (int q = 0; q < 6; q++) {
        int a = i + ofs[q][0], bb = j + ofs[q][1], c = k + ofs[q][2];
        d[q] = 0;
        r[q] = 0;
        if (L.bcm[fi[q]] & (1 << fc[q])) continue;
        T ax;
        if (fc[q] == 1) ax = row_vx(L, x, a, bb, c, &d[q]);
        else if (fc[q] == 2) ax = row_vy(L, x, a, bb, c, &d[q]);
        else ax = row_vz(L, x, a, bb, c, &d[q]);
        r[q] = b.c[fc[q]][fi[q]] - ax;
        num += cc[q] * r[q] / d[q];
        den += cc[q] * g[q] / d[q];
    }
    T dp = 0;
    if (!pbc && den != (T)0) {
        T rp = b.c[0][u] - row_p(L, x, i, j, k);
        dp = (num - rp) / den;
        P[u] += omega * dp;
    }
#pragma unroll
    for (int q = 0; q < 6; q++) {
        if (d[q] != (T)0) vout.c[fc[q]][fi[q]] = vin.c[fc[q]][fi[q]] + omega * (r[q] - g[q] * dp) / d[q];
    }
}
template <typename T>
__global__ void k_vanka(LevelView<T> L, T *P, Vec4<T> vin, Vec4<T> vout, Vec4<T> b, T omega, int col)
{
    pdl_enter();
    vanka_item(L, P, vin, vout, b, omega, col, (long)blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------------------
// Full cell-block variant: the cell's 6 face velocities and its pressure are
// solved together with the exact 7x7 cell system
//   [M g; cc^T 0] [dv; dp] = [r; rp],
// M the face-face block of the momentum rows.  Its off-diagonal entries come
// from the cell's normal stresses (every face enters e_xx, e_yy, e_zz and the
// divergence) and from the shear stresses on the edges two faces share; they
// are the coefficients of the row functions above (checked entry by entry
// against the assembled operator).  Faces under a boundary row are held; the
// pressure is held where the cell pressure is a boundary unknown.  M is
// eliminated without pivoting (-M is diagonally dominant).  Read/write
// pattern and buffering as k_vanka.
template <typename T>
__device__ __forceinline__ void face_block(const LevelView<T> &L, int i, int j, int k, T M[6][6])
{
    const T Ec = eta_at(L, L.ec, P2IDX(L, i, j, k));
    const T hx = L.ax.ih[i], hy = L.ay.ih[j], hz = L.az.ih[k];
    const T t43 = (T)(4.0 / 3.0), t23 = (T)(2.0 / 3.0);
    // d snn_d(cell) / d face, times Ec
    const T dn[3][6] = {{-t43 * hx, t43 * hx, t23 * hy, -t23 * hy, t23 * hz, -t23 * hz},
                        {t23 * hx, -t23 * hx, -t43 * hy, t43 * hy, t23 * hz, -t23 * hz},
                        {t23 * hx, -t23 * hx, t23 * hy, -t23 * hy, -t43 * hz, t43 * hz}};
    const T s0 = Ec * L.ax.ihc[i - 1], s1 = -Ec * L.ax.ihc[i], s2 = Ec * L.ay.ihc[j - 1], s3 = -Ec * L.ay.ihc[j],
            s4 = Ec * L.az.ihc[k - 1], s5 = -Ec * L.az.ihc[k];
#pragma unroll
    for (int b = 0; b < 6; b++) {
        M[0][b] = s0 * dn[0][b];
        M[1][b] = s1 * dn[0][b];
        M[2][b] = s2 * dn[1][b];
        M[3][b] = s3 * dn[1][b];
        M[4][b] = s4 * dn[2][b];
        M[5][b] = s5 * dn[2][b];
    }
    const T two = (T)2.0;
    const T exy00 = eta_at(L, L.exy, P2IDX(L, i - 1, j - 1, k - 1)), exy01 = eta_at(L, L.exy, P2IDX(L, i - 1, j, k - 1));
    const T exy10 = eta_at(L, L.exy, P2IDX(L, i, j - 1, k - 1)), exy11 = eta_at(L, L.exy, P2IDX(L, i, j, k - 1));
    const T exz00 = eta_at(L, L.exz, P2IDX(L, i - 1, j - 1, k - 1)), exz01 = eta_at(L, L.exz, P2IDX(L, i - 1, j - 1, k));
    const T exz10 = eta_at(L, L.exz, P2IDX(L, i, j - 1, k - 1)), exz11 = eta_at(L, L.exz, P2IDX(L, i, j - 1, k));
    const T eyz00 = eta_at(L, L.eyz, P2IDX(L, i - 1, j - 1, k - 1)), eyz01 = eta_at(L, L.eyz, P2IDX(L, i - 1, j - 1, k));
    const T eyz10 = eta_at(L, L.eyz, P2IDX(L, i - 1, j, k - 1)), eyz11 = eta_at(L, L.eyz, P2IDX(L, i - 1, j, k));
    const T hex0 = L.ax.ihe[i - 1], hex1 = L.ax.ihe[i], hey0 = L.ay.ihe[j - 1], hey1 = L.ay.ihe[j];
    const T hez0 = L.az.ihe[k - 1], hez1 = L.az.ihe[k];
    const T hvx = L.ax.ihv[i - 1], hvy = L.ay.ihv[j - 1], hvz = L.az.ihv[k - 1];
    // vx faces: shear with the vy (front/back) and vz (bottom/top) faces
    M[0][3] += two * exy01 * hex0 * hvy;  M[0][2] -= two * exy00 * hex0 * hvy;
    M[0][5] += two * exz01 * hex0 * hvz;  M[0][4] -= two * exz00 * hex0 * hvz;
    M[1][3] -= two * exy11 * hex1 * hvy;  M[1][2] += two * exy10 * hex1 * hvy;
    M[1][5] -= two * exz11 * hex1 * hvz;  M[1][4] += two * exz10 * hex1 * hvz;
    // vy faces
    M[2][1] += two * exy10 * hey0 * hvx;  M[2][0] -= two * exy00 * hey0 * hvx;
    M[2][5] += two * eyz01 * hey0 * hvz;  M[2][4] -= two * eyz00 * hey0 * hvz;
    M[3][1] -= two * exy11 * hey1 * hvx;  M[3][0] += two * exy01 * hey1 * hvx;
    M[3][5] -= two * eyz11 * hey1 * hvz;  M[3][4] += two * eyz10 * hey1 * hvz;
    // vz faces
    M[4][1] += two * exz10 * hez0 * hvx;  M[4][0] -= two * exz00 * hez0 * hvx;
    M[4][3] += two * eyz10 * hez0 * hvy;  M[4][2] -= two * eyz00 * hez0 * hvy;
    M[5][1] -= two * exz11 * hez1 * hvx;  M[5][0] += two * exz01 * hez1 * hvx;
    M[5][3] -= two * eyz11 * hez1 * hvy;  M[5][2] += two * eyz01 * hez1 * hvy;
}

template <typename T>
__global__ void __launch_bounds__(128) k_vanka_full(LevelView<T> L, T *P, Vec4<T> vin, Vec4<T> vout, Vec4<T> b,
                                                    T omega, int col)
{
    pdl_enter();
    int half = (L.ny) / 2;
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long lines = (long)(L.nx - 1) * (L.nz - 1);
    if (t >= lines * half) return;
    int jj = (int)(t % half);
    long line = t / half;
    int i = 1 + (int)(line % (L.nx - 1)), k = 1 + (int)(line / (L.nx - 1));
    int j0 = (((1 + i + k) & 1) == col) ? 1 : 2;
    int j = j0 + 2 * jj;
    if (j > L.ny - 1) return;
    Fields<T, T> x{P, vin.c[1], vin.c[2], vin.c[3]};
    int u = P2IDX(L, i, j, k);
    const bool pact = (L.bcm[u] & BC_P) == 0;
    int fi[6];
    const int fc[6] = {1, 1, 2, 2, 3, 3};
    T g[6], cc[6], r[6];
    bool act[6];
    fi[0] = P2IDX(L, i - 1, j - 1, k - 1); g[0] = -L.ax.ihc[i - 1]; cc[0] = -L.ax.ih[i];
    fi[1] = P2IDX(L, i, j - 1, k - 1);     g[1] = L.ax.ihc[i];      cc[1] = L.ax.ih[i];
    fi[2] = P2IDX(L, i - 1, j - 1, k - 1); g[2] = -L.ay.ihc[j - 1]; cc[2] = -L.ay.ih[j];
    fi[3] = P2IDX(L, i - 1, j, k - 1);     g[3] = L.ay.ihc[j];      cc[3] = L.ay.ih[j];
    fi[4] = P2IDX(L, i - 1, j - 1, k - 1); g[4] = -L.az.ihc[k - 1]; cc[4] = -L.az.ih[k];
    fi[5] = P2IDX(L, i - 1, j - 1, k);     g[5] = L.az.ihc[k];      cc[5] = L.az.ih[k];
    const int ofs[6][3] = {{-1, -1, -1}, {0, -1, -1}, {-1, -1, -1}, {-1, 0, -1}, {-1, -1, -1}, {-1, -1, 0}};
    T M[6][6];
    face_block(L, i, j, k, M);
#pragma unroll
    for (int q = 0; q < 6; q++) {
        int a = i + ofs[q][0], bb = j + ofs[q][1], c = k + ofs[q][2];
        T d = 0;
        act[q] = !(L.bcm[fi[q]] & (1 << fc[q]));
        r[q] = 0;
        if (act[q]) {
            T ax;
            if (fc[q] == 1) ax = row_vx(L, x, a, bb, c, &d);
            else if (fc[q] == 2) ax = row_vy(L, x, a, bb, c, &d);
            else ax = row_vz(L, x, a, bb, c, &d);
            r[q] = b.c[fc[q]][fi[q]] - ax;
        }
        M[q][q] = d;
    }
    // masked system: held faces become identity rows / zero columns
    T y1[6], y2[6];
#pragma unroll
    for (int a = 0; a < 6; a++) {
#pragma unroll
        for (int c = 0; c < 6; c++)
            if (!(act[a] && act[c])) M[a][c] = a == c ? (T)1 : (T)0;
        y1[a] = act[a] ? r[a] : (T)0;
        y2[a] = act[a] ? g[a] : (T)0;
    }
    // constant trip counts so that M, y1, y2 stay in registers
#pragma unroll
    for (int c = 0; c < 6; c++) {
        const T ip = (T)1 / M[c][c];
#pragma unroll
        for (int a = 0; a < 6; a++) {
            if (a > c) {
                const T f = M[a][c] * ip;
#pragma unroll
                for (int e = 0; e < 6; e++)
                    if (e > c) M[a][e] -= f * M[c][e];
                y1[a] -= f * y1[c];
                y2[a] -= f * y2[c];
            }
        }
    }
#pragma unroll
    for (int cc5 = 0; cc5 < 6; cc5++) {
        const int c = 5 - cc5;
#pragma unroll
        for (int e = 0; e < 6; e++) {
            if (e > c) {
                y1[c] -= M[c][e] * y1[e];
                y2[c] -= M[c][e] * y2[e];
            }
        }
        const T ip = (T)1 / M[c][c];
        y1[c] *= ip;
        y2[c] *= ip;
    }
    T dp = 0;
    if (pact) {
        T num = -(b.c[0][u] - row_p(L, x, i, j, k)), den = 0;
#pragma unroll
        for (int q = 0; q < 6; q++) {
            num += cc[q] * y1[q];
            den += cc[q] * y2[q];
        }
        if (den != (T)0) {
            dp = num / den;
            P[u] += omega * dp;
        }
    }
#pragma unroll
    for (int q = 0; q < 6; q++)
        if (act[q]) vout.c[fc[q]][fi[q]] = vin.c[fc[q]][fi[q]] + omega * (y1[q] - dp * y2[q]);
}

// Momentum parts (A v + grad p) of the six face rows of cell (i, j, k) from
// shared stresses, and the cell's divergence: the cell's three normal
// stresses from one set of strain rates, the six neighbour cells' normal
// stresses along their face normals, the twelve edge shear stresses once
// each.  Every velocity, viscosity and pressure is loaded once, addressed
// from the cell's low corner F = (i-1, j-1, k-1) (y stride 1, x stride ny, z
// stride nx*ny); the deviatoric third is a multiplication by 1/3.  The same
// terms as row_vx/row_vy/row_vz up to rounding.
template <typename T>
__device__ __forceinline__ void cell_rows(const LevelView<T> &L, const Fields<T, T> &x, int i, int j, int k,
                                          const int fi[6], T ax[6], T &div)
{
    const int sy = L.ny, sz = L.nx * L.ny;
    const int F = fi[0];
    const T *vx = x.vx + F, *vy = x.vy + F, *vz = x.vz + F;
    // velocities around the cell (offsets from F)
    const T vx0 = __ldg(vx), vxX = __ldg(vx + sy), vxXX = __ldg(vx + 2 * sy), vxm = __ldg(vx - sy);
    const T vxY = __ldg(vx + 1), vxy_ = __ldg(vx - 1), vxXY = __ldg(vx + sy + 1), vxXy = __ldg(vx + sy - 1);
    const T vxZ = __ldg(vx + sz), vxz_ = __ldg(vx - sz), vxXZ = __ldg(vx + sy + sz), vxXz = __ldg(vx + sy - sz);
    const T vy0 = __ldg(vy), vyY = __ldg(vy + 1), vyYY = __ldg(vy + 2), vym = __ldg(vy - 1);
    const T vyX = __ldg(vy + sy), vyx_ = __ldg(vy - sy), vyXY = __ldg(vy + sy + 1), vyxY = __ldg(vy - sy + 1);
    const T vyZ = __ldg(vy + sz), vyz_ = __ldg(vy - sz), vyYZ = __ldg(vy + 1 + sz), vyYz = __ldg(vy + 1 - sz);
    const T vz0 = __ldg(vz), vzZ = __ldg(vz + sz), vzZZ = __ldg(vz + 2 * sz), vzm = __ldg(vz - sz);
    const T vzX = __ldg(vz + sy), vzx_ = __ldg(vz - sy), vzXZ = __ldg(vz + sy + sz), vzxZ = __ldg(vz - sy + sz);
    const T vzY = __ldg(vz + 1), vzy_ = __ldg(vz - 1), vzYZ = __ldg(vz + 1 + sz), vzyZ = __ldg(vz - 1 + sz);
    const T third = (T)(1.0 / 3.0), two = (T)2.0;
    const T hx0 = L.ax.ih[i - 1], hx1 = L.ax.ih[i], hx2 = L.ax.ih[i + 1];
    const T hy0 = L.ay.ih[j - 1], hy1 = L.ay.ih[j], hy2 = L.ay.ih[j + 1];
    const T hz0 = L.az.ih[k - 1], hz1 = L.az.ih[k], hz2 = L.az.ih[k + 1];
    const int u = F + sz + sy + 1;
    // own cell
    const T exx = (vxX - vx0) * hx1, eyy = (vyY - vy0) * hy1, ezz = (vzZ - vz0) * hz1;
    div = exx + eyy + ezz;
    const T E2 = two * eta_at(L, L.ec, u);
    const T s0 = E2 * (exx - div * third), s1 = E2 * (eyy - div * third), s2 = E2 * (ezz - div * third);
    // neighbour cells: normal stress along the shared face's normal
    T sL, sR, sF, sB, sD, sU;
    {   // cell (i-1, j, k): faces vx[F-sy], vx[F]; vy[F-sy], vy[F-sy+1]; vz[F-sy], vz[F-sy+sz]
        const T a = (vx0 - vxm) * hx0, b = (vyxY - vyx_) * hy1, c = (vzxZ - vzx_) * hz1;
        sL = two * eta_at(L, L.ec, u - sy) * (a - (a + b + c) * third);
    }
    {   // cell (i+1, j, k)
        const T a = (vxXX - vxX) * hx2, b = (vyXY - vyX) * hy1, c = (vzXZ - vzX) * hz1;
        sR = two * eta_at(L, L.ec, u + sy) * (a - (a + b + c) * third);
    }
    {   // cell (i, j-1, k)
        const T a = (vxXy - vxy_) * hx1, b = (vy0 - vym) * hy0, c = (vzyZ - vzy_) * hz1;
        sF = two * eta_at(L, L.ec, u - 1) * (b - (a + b + c) * third);
    }
    {   // cell (i, j+1, k)
        const T a = (vxXY - vxY) * hx1, b = (vyYY - vyY) * hy2, c = (vzYZ - vzY) * hz1;
        sB = two * eta_at(L, L.ec, u + 1) * (b - (a + b + c) * third);
    }
    {   // cell (i, j, k-1)
        const T a = (vxXz - vxz_) * hx1, b = (vyYz - vyz_) * hy1, c = (vz0 - vzm) * hz0;
        sD = two * eta_at(L, L.ec, u - sz) * (c - (a + b + c) * third);
    }
    {   // cell (i, j, k+1)
        const T a = (vxXZ - vxZ) * hx1, b = (vyYZ - vyZ) * hy1, c = (vzZZ - vzZ) * hz2;
        sU = two * eta_at(L, L.ec, u + sz) * (c - (a + b + c) * third);
    }
    // edge shear stresses (sxy, sxz, syz at the cell's twelve edges)
    const T ex0 = L.ax.ihe[i - 1], ex1 = L.ax.ihe[i], ey0 = L.ay.ihe[j - 1], ey1 = L.ay.ihe[j];
    const T ez0 = L.az.ihe[k - 1], ez1 = L.az.ihe[k];
    const T xy00 = two * eta_at(L, L.exy, F) * ((vx0 - vxy_) * ey0 + (vy0 - vyx_) * ex0);
    const T xy01 = two * eta_at(L, L.exy, F + 1) * ((vxY - vx0) * ey1 + (vyY - vyxY) * ex0);
    const T xy10 = two * eta_at(L, L.exy, F + sy) * ((vxX - vxXy) * ey0 + (vyX - vy0) * ex1);
    const T xy11 = two * eta_at(L, L.exy, F + sy + 1) * ((vxXY - vxX) * ey1 + (vyXY - vyY) * ex1);
    const T xz00 = two * eta_at(L, L.exz, F) * ((vx0 - vxz_) * ez0 + (vz0 - vzx_) * ex0);
    const T xz01 = two * eta_at(L, L.exz, F + sz) * ((vxZ - vx0) * ez1 + (vzZ - vzxZ) * ex0);
    const T xz10 = two * eta_at(L, L.exz, F + sy) * ((vxX - vxXz) * ez0 + (vzX - vz0) * ex1);
    const T xz11 = two * eta_at(L, L.exz, F + sy + sz) * ((vxXZ - vxX) * ez1 + (vzXZ - vzZ) * ex1);
    const T yz00 = two * eta_at(L, L.eyz, F) * ((vy0 - vyz_) * ez0 + (vz0 - vzy_) * ey0);
    const T yz01 = two * eta_at(L, L.eyz, F + sz) * ((vyZ - vy0) * ez1 + (vzZ - vzyZ) * ey0);
    const T yz10 = two * eta_at(L, L.eyz, F + 1) * ((vyY - vyYz) * ez0 + (vzY - vz0) * ey1);
    const T yz11 = two * eta_at(L, L.eyz, F + 1 + sz) * ((vyYZ - vyY) * ez1 + (vzYZ - vzZ) * ey1);
    const T *pp = x.p + u;
    const T p0 = __ldg(pp), pL = __ldg(pp - sy), pR = __ldg(pp + sy), pF = __ldg(pp - 1),
            pB = __ldg(pp + 1);
    const T pD = __ldg(pp - sz), pU = __ldg(pp + sz);
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

// Cell of thread t in colour col (cells with (i + j + k) of one parity), or
// false when the slot is past the last cell of its line.
template <typename T>
__device__ __forceinline__ bool colour_cell(const LevelView<T> &L, int col, long t, int &i, int &j, int &k)
{
    const int half = L.ny / 2;
    const long lines = (long)(L.nx - 1) * (L.nz - 1);
    if (t >= lines * half) return false;
    const int jj = (int)(t % half);
    const long line = t / half;
    i = 1 + (int)(line % (L.nx - 1));
    k = 1 + (int)(line / (L.nx - 1));
    j = ((((1 + i + k) & 1) == col) ? 1 : 2) + 2 * jj;
    return j <= L.ny - 1;
}

// the six faces of cell (i, j, k): low and high x, y, z faces
template <typename T>
__device__ __forceinline__ void cell_faces(const LevelView<T> &L, int i, int j, int k, int fi[6])
{
    fi[0] = P2IDX(L, i - 1, j - 1, k - 1);
    fi[1] = P2IDX(L, i, j - 1, k - 1);
    fi[2] = fi[0];
    fi[3] = P2IDX(L, i - 1, j, k - 1);
    fi[4] = fi[0];
    fi[5] = P2IDX(L, i - 1, j - 1, k);
}

// ---------------------------------------------------------------------------
// k_vanka_full with the six momentum residuals from cell_rows (shared
// stresses): same terms as row_vx/row_vy/row_vz, about half the loads and
// arithmetic.  The cell system is built and eliminated on every sweep.
template <typename T>
__global__ void __launch_bounds__(128) k_vanka_fast(LevelView<T> L, T *P, Vec4<T> vin, Vec4<T> vout, Vec4<T> b,
                                                    T omega, int col)
{
    pdl_enter();
    int i, j, k;
    if (!colour_cell(L, col, (long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
    Fields<T, T> x{P, vin.c[1], vin.c[2], vin.c[3]};
    const int u = P2IDX(L, i, j, k);
    const bool pact = (L.bcm[u] & BC_P) == 0;
    int fi[6];
    const int fc[6] = {1, 1, 2, 2, 3, 3};
    cell_faces(L, i, j, k, fi);
    const T g[6] = {-L.ax.ihc[i - 1], L.ax.ihc[i], -L.ay.ihc[j - 1], L.ay.ihc[j], -L.az.ihc[k - 1], L.az.ihc[k]};
    const T hx = L.ax.ih[i], hy = L.ay.ih[j], hz = L.az.ih[k];
    const T cc[6] = {-hx, hx, -hy, hy, -hz, hz};
    T ax[6], div;
    cell_rows(L, x, i, j, k, fi, ax, div);
    T M[6][6];
    face_block(L, i, j, k, M);
    M[0][0] = diag_vx(L, i - 1, j - 1, k - 1);
    M[1][1] = diag_vx(L, i, j - 1, k - 1);
    M[2][2] = diag_vy(L, i - 1, j - 1, k - 1);
    M[3][3] = diag_vy(L, i - 1, j, k - 1);
    M[4][4] = diag_vz(L, i - 1, j - 1, k - 1);
    M[5][5] = diag_vz(L, i - 1, j - 1, k);
    bool act[6];
    T y1[6], y2[6];
#pragma unroll
    for (int q = 0; q < 6; q++) act[q] = !(L.bcm[fi[q]] & (1 << fc[q]));
#pragma unroll
    for (int a = 0; a < 6; a++) {
#pragma unroll
        for (int c = 0; c < 6; c++)
            if (!(act[a] && act[c])) M[a][c] = a == c ? (T)1 : (T)0;
        y1[a] = act[a] ? b.c[fc[a]][fi[a]] - ax[a] : (T)0;
        y2[a] = act[a] ? g[a] : (T)0;
    }
#pragma unroll
    for (int c = 0; c < 6; c++) {
        const T ip = (T)1 / M[c][c];
#pragma unroll
        for (int a = 0; a < 6; a++) {
            if (a > c) {
                const T f = M[a][c] * ip;
#pragma unroll
                for (int e = 0; e < 6; e++)
                    if (e > c) M[a][e] -= f * M[c][e];
                y1[a] -= f * y1[c];
                y2[a] -= f * y2[c];
            }
        }
    }
#pragma unroll
    for (int cc5 = 0; cc5 < 6; cc5++) {
        const int c = 5 - cc5;
#pragma unroll
        for (int e = 0; e < 6; e++) {
            if (e > c) {
                y1[c] -= M[c][e] * y1[e];
                y2[c] -= M[c][e] * y2[e];
            }
        }
        const T ip = (T)1 / M[c][c];
        y1[c] *= ip;
        y2[c] *= ip;
    }
    T dp = 0;
    if (pact) {
        T num = -(b.c[0][u] - div), den = 0;
#pragma unroll
        for (int q = 0; q < 6; q++) {
            num += cc[q] * y1[q];
            den += cc[q] * y2[q];
        }
        if (den != (T)0) {
            dp = num / den;
            P[u] += omega * dp;
        }
    }
#pragma unroll
    for (int q = 0; q < 6; q++)
        if (act[q]) vout.c[fc[q]][fi[q]] = vin.c[fc[q]][fi[q]] + omega * (y1[q] - dp * y2[q]);
}

// ---------------------------------------------------------------------------
// Full cell-block smoother with stored cell factors.  The masked cell system
// of k_vanka_full depends on the viscosities and the grid only, so once per
// solve k_vanka_factor inverts the 6x6 face block M of every cell of one
// colour (Gauss-Jordan without pivoting: -M is diagonally dominant; in FP64,
// also for the FP32 cycle, whose factors are stored rounded to float).
// Scaled by the faces' control volumes the block is symmetric: with
// V'_a = ih / ihc along face a's normal (the face's control volume over the
// cell's), S = diag(V') M = S^T, so M^-1 = S^-1 diag(V') with S^-1 symmetric,
// and V'_a g_a = cc_a (the continuity coefficients).  Stored per cell,
// entry-major so that a warp's loads are coalesced:
//   entries 0..20  the upper triangle of S^-1 row by row (rows and columns
//                  of held faces zero);
//   entry 21       1/den, den = cc . S^-1 cc (0 where the cell pressure is a
//                  boundary unknown or den = 0, which holds the pressure).
// The sweep (k_vanka_stored) assembles the residuals with cell_rows and
// applies the stored factors: y1 = S^-1 (V' r), y2 = S^-1 cc,
// dp = (cc . y1 - r_p) / den, v += omega (y1 - dp y2), p += omega dp; the
// same update as k_vanka_full up to rounding, without building and
// eliminating the 6x6 block on every sweep.
constexpr int kBlkEntries = 22;
// minimum resident blocks per SM asked of the compiler for k_vanka_stored
// (FP32 cycle; the FP64 cycle's kernel needs more registers)
#ifndef P2_STORED_MIN_BLOCKS
#define P2_STORED_MIN_BLOCKS 7
#endif

// packed upper-triangle index of (a, c), a <= c
__host__ __device__ constexpr int tri_index(int a, int c) { return a * 6 - a * (a - 1) / 2 + (c - a); }

template <typename T>
__device__ __forceinline__ T face_ratio(T ih, T ihc) { return ih / ihc; }
template <>
__device__ __forceinline__ float face_ratio<float>(float ih, float ihc) { return __fdividef(ih, ihc); }

template <typename T>
__device__ __forceinline__ void face_volumes(const LevelView<T> &L, int i, int j, int k, T v[6])
{
    const T hx = L.ax.ih[i], hy = L.ay.ih[j], hz = L.az.ih[k];
    v[0] = face_ratio(hx, L.ax.ihc[i - 1]);
    v[1] = face_ratio(hx, L.ax.ihc[i]);
    v[2] = face_ratio(hy, L.ay.ihc[j - 1]);
    v[3] = face_ratio(hy, L.ay.ihc[j]);
    v[4] = face_ratio(hz, L.az.ihc[k - 1]);
    v[5] = face_ratio(hz, L.az.ihc[k]);
}

template <typename T, typename S>
__global__ void __launch_bounds__(128) k_vanka_factor(LevelView<T> L, int col, S *blk, long stride)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!colour_cell(L, col, t, i, j, k)) return;
    const int u = P2IDX(L, i, j, k);
    int fi[6];
    const int fc[6] = {1, 1, 2, 2, 3, 3};
    cell_faces(L, i, j, k, fi);
    const T hx = L.ax.ih[i], hy = L.ay.ih[j], hz = L.az.ih[k];
    const T cc[6] = {-hx, hx, -hy, hy, -hz, hz};
    T M[6][6];
    face_block(L, i, j, k, M);
    M[0][0] = diag_vx(L, i - 1, j - 1, k - 1);
    M[1][1] = diag_vx(L, i, j - 1, k - 1);
    M[2][2] = diag_vy(L, i - 1, j - 1, k - 1);
    M[3][3] = diag_vy(L, i - 1, j, k - 1);
    M[4][4] = diag_vz(L, i - 1, j - 1, k - 1);
    M[5][5] = diag_vz(L, i - 1, j - 1, k);
    bool act[6];
#pragma unroll
    for (int q = 0; q < 6; q++) act[q] = !(L.bcm[fi[q]] & (1 << fc[q]));
#pragma unroll
    for (int a = 0; a < 6; a++)
#pragma unroll
        for (int c = 0; c < 6; c++)
            if (!(act[a] && act[c])) M[a][c] = a == c ? (T)1 : (T)0;
    // in-place Gauss-Jordan inverse
#pragma unroll
    for (int c = 0; c < 6; c++) {
        const T ip = (T)1 / M[c][c];
        M[c][c] = (T)1;
#pragma unroll
        for (int e = 0; e < 6; e++) M[c][e] *= ip;
#pragma unroll
        for (int a = 0; a < 6; a++) {
            if (a != c) {
                const T f = M[a][c];
                M[a][c] = (T)0;
#pragma unroll
                for (int e = 0; e < 6; e++) M[a][e] -= f * M[c][e];
            }
        }
    }
    // S^-1 = M^-1 diag(V')^-1, symmetrised; held rows and columns zero
    T v[6];
    face_volumes(L, i, j, k, v);
#pragma unroll
    for (int a = 0; a < 6; a++)
#pragma unroll
        for (int c = 0; c < 6; c++)
            M[a][c] = (act[a] && act[c]) ? M[a][c] / v[c] : (T)0;
    T den = 0;
#pragma unroll
    for (int a = 0; a < 6; a++) {
        T y2 = 0;
#pragma unroll
        for (int c = 0; c < 6; c++) y2 += (T)0.5 * (M[a][c] + M[c][a]) * cc[c];
        den += cc[a] * y2;
    }
#pragma unroll
    for (int a = 0; a < 6; a++)
#pragma unroll
        for (int c = a; c < 6; c++) blk[(long)tri_index(a, c) * stride + t] = to_factor<S>((T)0.5 * (M[a][c] + M[c][a]));
    const bool pact = (L.bcm[u] & BC_P) == 0;
    blk[21L * stride + t] = to_factor<S>((pact && den != (T)0) ? (T)1 / den : (T)0);
}

template <typename T>
__device__ __forceinline__ void vanka_stored_item(const LevelView<T> &L, T *P, const Vec4<T> &vin,
                                                  const Vec4<T> &vout, const Vec4<T> &b, T omega, int col,
                                                  const factor_t<T> *__restrict__ blk, long stride, long t)
{
    int i, j, k;
    if (!colour_cell(L, col, t, i, j, k)) return;
    Fields<T, T> x{P, vin.c[1], vin.c[2], vin.c[3]};
    const int u = P2IDX(L, i, j, k);
    int fi[6];
    const int fc[6] = {1, 1, 2, 2, 3, 3};
    cell_faces(L, i, j, k, fi);
    T ax[6], div;
    cell_rows(L, x, i, j, k, fi, ax, div);
    const T hx = L.ax.ih[i], hy = L.ay.ih[j], hz = L.az.ih[k];
    const T cc[6] = {-hx, hx, -hy, hy, -hz, hz};
    T v[6];
    face_volumes(L, i, j, k, v);
    bool act[6];
    T vr[6];
#pragma unroll
    for (int q = 0; q < 6; q++) {
        act[q] = !(L.bcm[fi[q]] & (1 << fc[q]));
        vr[q] = act[q] ? (b.c[fc[q]][fi[q]] - ax[q]) * v[q] : (T)0;
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
    T dp = 0;
    if (inv != (T)0) {
        T num = -(b.c[0][u] - div);
#pragma unroll
        for (int q = 0; q < 6; q++) num += cc[q] * y1[q];
        dp = num * inv;
        P[u] += omega * dp;
    }
#pragma unroll
    for (int q = 0; q < 6; q++)
        if (act[q]) vout.c[fc[q]][fi[q]] = vin.c[fc[q]][fi[q]] + omega * (y1[q] - dp * y2[q]);
}
template <typename T>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? P2_STORED_MIN_BLOCKS : 3) k_vanka_stored(
    LevelView<T> L, T *P, Vec4<T> vin, Vec4<T> vout, Vec4<T> b, T omega, int col,
    const factor_t<T> *__restrict__ blk, long stride)
{
    pdl_enter();
    vanka_stored_item(L, P, vin, vout, b, omega, col, blk, stride, (long)blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------------------
// Transfers.  Per-axis tables (host-built from the reference's index rules,
// move3mgNew.c:3562-3575 and the corresponding blocks of vprestrict and
// vpprolong): for a fine index m, the coarse interval lo[m] and the weights
// w0 (coarse lo) and w1 (coarse lo+1).  Restriction uses the inverse lists.
__device__ __forceinline__ int ax_type(int comp, int axis)
{
    if (comp == 0) return 2;
    return (comp == axis + 1) ? 0 : 1;
}

__device__ __forceinline__ double block_sum(double v, double *sh);  // below (norms)

// tv.m[axis][type] for a runtime type without copying the parameter struct
__device__ __forceinline__ AxisMap pick_map(const AxisMap (&m)[3], int type)
{
    return type == 0 ? m[0] : (type == 1 ? m[1] : m[2]);
}

// Restriction (vprestrict, move3mgNew.c:3965-4353): b_c = sum_f w r_f / sum_f w
// over the non-boundary fine rows (pressure residuals scaled by eta_f/eta_c,
// 4308), for non-boundary coarse rows (0 otherwise); x_c = 0 (4351).  One
// thread per (coarse node, component), components in consecutive blocks of
// nodes.  Fused with the first half of the coarse
// right-hand-side compatibility shift: every block adds its volume-weighted
// continuity rows into partial[block]; the last block to finish (ticket
// counter, reset by that block) sums the partials in block order and writes
// sums[0] = sum of vol * b_P and sums[1] = vol_total (fixed per level).
constexpr int kRestrictList = 5;  // longest inverse list of one axis (host-checked)

template <typename T>
__device__ __forceinline__ double restrict_item(const LevelView<T> &F, const Vec4<T> &rf, const LevelView<T> &Cl,
                                               const Vec4<T> &bc, const Vec4<T> &xc, const TransferView &tv,
                                               int scale_p, long t)
{
    const int n = Cl.n;
    double contrib = 0;
    if (t < 4L * n) {
        const int c = (int)(t / n), v = (int)(t % n);
        const int J = v % Cl.ny, I = (v / Cl.ny) % Cl.nx, K = v / (Cl.nx * Cl.ny);
        // component pointers by constant-index selects (no local copy of the parameters)
        auto comp = [c](const Vec4<T> &V) { return c == 0 ? V.c[0] : (c == 1 ? V.c[1] : (c == 2 ? V.c[2] : V.c[3])); };
        T *xcc = comp(xc), *bcc = comp(bc);
        xcc[v] = 0;
        T out = 0;
        if (valid_pos(c, I, J, K, Cl.nx, Cl.ny, Cl.nz) && !(Cl.bcm[v] & (1 << c))) {
            const AxisMap mx = pick_map(tv.m[0], ax_type(c, 0)), my = pick_map(tv.m[1], ax_type(c, 1)),
                          mz = pick_map(tv.m[2], ax_type(c, 2));
            T acc = 0, ws = 0;
            const T etac = c == 0 ? (T)Cl.ec[v] : (T)1;
            const int x0 = mx.ptr[I], nxq = mx.ptr[I + 1] - x0, y0 = my.ptr[J], nyq = my.ptr[J + 1] - y0;
            const T *rfc = comp(rf);
            // the x and y lists (at most kRestrictList entries each, checked on
            // the host) in registers, the x and y loops unrolled with fixed trip
            // counts: the fine-node loads of one z line are independent of each
            // other, so they are issued together rather than one after another
            int xi[kRestrictList], yi[kRestrictList];
            T xw[kRestrictList], yw[kRestrictList];
#pragma unroll
            for (int a = 0; a < kRestrictList; a++) {
                xi[a] = a < nxq ? mx.idx[x0 + a] : 0;
                xw[a] = a < nxq ? (T)mx.w[x0 + a] : (T)0;
                yi[a] = a < nyq ? my.idx[y0 + a] : 0;
                yw[a] = a < nyq ? (T)my.w[y0 + a] : (T)0;
            }
            // the value, mask and viscosity loads of a fine node do not depend
            // on each other or on a branch: a boundary row contributes with
            // weight 0 (its value times 0 adds nothing), so every load of a z
            // line can be in flight at once
            for (int qz = mz.ptr[K]; qz < mz.ptr[K + 1]; qz++) {
                const int fk = mz.idx[qz];
                const T wz = (T)mz.w[qz];
#pragma unroll
                for (int ax = 0; ax < kRestrictList; ax++) {
                    if (ax < nxq) {
                        const T wzx = wz * xw[ax];
                        const int base = fk * (F.nx * F.ny) + xi[ax] * F.ny;
#pragma unroll
                        for (int ay = 0; ay < kRestrictList; ay++) {
                            if (ay < nyq) {
                                const int f = base + yi[ay];
                                const bool bnd = __ldg(F.bcm + f) & (1 << c);
                                T val = __ldg(rfc + f);
                                if (c == 0 && scale_p) val *= (T)__ldg(F.ec + f);
                                const T w = bnd ? (T)0 : wzx * yw[ay];
                                acc += val * w;
                                ws += w;
                            }
                        }
                    }
                }
            }
            // the pressure residuals' viscosity ratio eta_f / eta_c: eta_f per
            // fine node above, the division by eta_c once here
            if (c == 0 && scale_p) acc /= etac;
            out = ws != (T)0 ? acc / ws : (T)0;
            if (c == 0 && I > 0 && J > 0 && K > 0)
                contrib = (double)out / ((double)Cl.ax.ih[I] * (double)Cl.ay.ih[J] * (double)Cl.az.ih[K]);
        }
        bcc[v] = out;
    }
    return contrib;
}
template <typename T>
__global__ void k_restrict_compat(LevelView<T> F, Vec4<T> rf, LevelView<T> Cl, Vec4<T> bc, Vec4<T> xc,
                                  TransferView tv, int scale_p, double vol_total, double *partial,
                                  unsigned *ticket, double *sums)
{
    pdl_enter();
    __shared__ double sh[32];
    __shared__ bool last;
    const double contrib =
        restrict_item(F, rf, Cl, bc, xc, tv, scale_p, (long)blockIdx.x * blockDim.x + threadIdx.x);
    const double bsum = block_sum(contrib, sh);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = bsum;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last) {
        __threadfence();
        double s = 0;
        for (int q = threadIdx.x; q < (int)gridDim.x; q += blockDim.x) s += ((volatile double *)partial)[q];
        s = block_sum(s, sh);
        if (threadIdx.x == 0) {
            sums[0] = s;
            sums[1] = vol_total;
            *ticket = 0;
        }
    }
}

// x_f += sum_c w x_c * (p1koef | v1koef) over every fine unknown position.
template <typename T>
__device__ __forceinline__ void prolong_item(const LevelView<T> &F, const Vec4<T> &xf, const LevelView<T> &Cl,
                                             const Vec4<T> &xc, const TransferView &tv, T p1, T v1, int u)
{
    if (u >= F.n) return;
    int j = u % F.ny, i = (u / F.ny) % F.nx, k = u / (F.nx * F.ny);
    for (int c = 0; c < 4; c++) {
        if (!valid_pos(c, i, j, k, F.nx, F.ny, F.nz)) continue;
        const AxisMap &mx = tv.m[0][ax_type(c, 0)], &my = tv.m[1][ax_type(c, 1)], &mz = tv.m[2][ax_type(c, 2)];
        int lx = mx.lo[i], ly = my.lo[j], lz = mz.lo[k];
        T wx0 = (T)mx.w0[i], wx1 = (T)mx.w1[i], wy0 = (T)my.w0[j], wy1 = (T)my.w1[j];
        T wz0 = (T)mz.w0[k], wz1 = (T)mz.w1[k];
        T s = 0;
#pragma unroll
        for (int d = 0; d < 2; d++)
#pragma unroll
            for (int a = 0; a < 2; a++)
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    T w = (d ? wz1 : wz0) * (a ? wx1 : wx0) * (e ? wy1 : wy0);
                    s += xc.c[c][P2IDX(Cl, lx + a, ly + e, lz + d)] * w;
                }
        xf.c[c][u] += s * (c == 0 ? p1 : v1);
    }
}
template <typename T>
__global__ void k_prolong(LevelView<T> F, Vec4<T> xf, LevelView<T> Cl, Vec4<T> xc, TransferView tv, T p1, T v1)
{
    pdl_enter();
    prolong_item(F, xf, Cl, xc, tv, p1, v1, blockIdx.x * blockDim.x + threadIdx.x);
}

// ronurestrict (move3mgNew.c:3386-3527): coarse nu, ro as weighted averages
// of the fine node values (nu averaged as nu, log nu or 1/nu per viscmod).
__global__ void k_ronurestrict(int fnx, int fny, int fnz, const float *fnu, const float *fro, int cnx, int cny,
                               int cnz, float *cnu, float *cro, AxisMap mx, AxisMap my, AxisMap mz, int viscmod)
{
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= cnx * cny * cnz) return;
    int J = v % cny, I = (v / cny) % cnx, K = v / (cnx * cny);
    double sn = 0, sr = 0, sw = 0;
    for (int qz = mz.ptr[K]; qz < mz.ptr[K + 1]; qz++)
        for (int qx = mx.ptr[I]; qx < mx.ptr[I + 1]; qx++)
            for (int qy = my.ptr[J]; qy < my.ptr[J + 1]; qy++) {
                int f = mz.idx[qz] * fnx * fny + mx.idx[qx] * fny + my.idx[qy];
                double w = mz.w[qz] * mx.w[qx] * my.w[qy];
                double nv = fnu[f];
                double fv = viscmod == 0 ? nv : (viscmod == 1 ? log(nv) : 1.0 / nv);
                sn += fv * w;
                sr += (double)fro[f] * w;
                sw += w;
            }
    double nv = sn / sw;
    if (viscmod == 1) nv = exp(nv);
    if (viscmod == 2) nv = 1.0 / nv;
    cnu[v] = (float)nv;
    cro[v] = (float)(sr / sw);
}

__device__ __forceinline__ double vmean(int viscmod, const double *v, int n)
{
    double s = 0;
    if (viscmod == 0) {
        for (int i = 0; i < n; i++) s += v[i];
        return s / n;
    }
    if (viscmod == 1) {
        for (int i = 0; i < n; i++) s += log(v[i]);
        return exp(s / n);
    }
    for (int i = 0; i < n; i++) s += 1.0 / v[i];
    return 1.0 / (s / n);
}

__device__ __forceinline__ double clampd(double v, double lo, double hi)
{
    if (v > hi) v = hi;
    if (v < lo) v = lo;
    return v;
}

// Per-stencil viscosities of one level, clamped to [nubeg, nuend]: level 0
// from nxx..nyz (sxxcalc:36-38, sxycalc:433-435, ...); coarse levels from the
// 8 cell-corner (sxx) or 2 edge-end (sxy, sxz, syz) nu values (41-47, 438-444).
__global__ void k_level_eta(int nx, int ny, int nz, const float *nu, const float *nxx, const float *nxy,
                            const float *nxz, const float *nyz, float *ec, float *exy, float *exz, float *eyz,
                            double lo, double hi, int viscmod, int level0)
{
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nx * ny * nz) return;
    if (level0) {
        ec[u] = (float)clampd(nxx[u], lo, hi);
        exy[u] = (float)clampd(nxy[u], lo, hi);
        exz[u] = (float)clampd(nxz[u], lo, hi);
        eyz[u] = (float)clampd(nyz[u], lo, hi);
        return;
    }
    int j = u % ny, i = (u / ny) % nx, k = u / (nx * ny);
    int xy = nx * ny;
    if (i > 0 && j > 0 && k > 0) {
        double v[8] = {nu[u - xy - ny - 1], nu[u - xy - ny], nu[u - xy - 1], nu[u - xy],
                       nu[u - ny - 1],      nu[u - ny],      nu[u - 1],      nu[u]};
        ec[u] = (float)clampd(vmean(viscmod, v, 8), lo, hi);
    } else {
        ec[u] = (float)lo;
    }
    double v2[2];
    v2[0] = nu[u];
    v2[1] = k + 1 < nz ? nu[u + xy] : nu[u];
    exy[u] = (float)clampd(vmean(viscmod, v2, 2), lo, hi);
    v2[1] = j + 1 < ny ? nu[u + 1] : nu[u];
    exz[u] = (float)clampd(vmean(viscmod, v2, 2), lo, hi);
    v2[1] = i + 1 < nx ? nu[u + ny] : nu[u];
    eyz[u] = (float)clampd(vmean(viscmod, v2, 2), lo, hi);
}

// Level-0 right-hand sides of the Stokes rows (xstokserr:845, ystokserr:1060,
// zstokserr:1279): -g * (sum of 4 float densities, summed in float) / 4.
template <typename T>
__global__ void k_rhs0(int nx, int ny, int nz, const float *ro, const uint8_t *bcm, Vec4<T> b, double gxk, double gyk,
                       double gzk)
{
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nx * ny * nz) return;
    int j = u % ny, i = (u / ny) % nx, k = u / (nx * ny);
    int xy = nx * ny;
    uint8_t m = bcm[u];
    b.c[0][u] = 0;
    T vx = 0, vy = 0, vz = 0;
    if (valid_pos(1, i, j, k, nx, ny, nz) && !(m & BC_VX)) {
        float s = ro[u] + ro[u + 1] + ro[u + xy] + ro[u + xy + 1];
        vx = (T)(-gxk * (double)s / 4.0);
    }
    if (valid_pos(2, i, j, k, nx, ny, nz) && !(m & BC_VY)) {
        float s = ro[u] + ro[u + ny] + ro[u + xy] + ro[u + xy + ny];
        vy = (T)(-gyk * (double)s / 4.0);
    }
    if (valid_pos(3, i, j, k, nx, ny, nz) && !(m & BC_VZ)) {
        float s = ro[u] + ro[u + 1] + ro[u + ny] + ro[u + ny + 1];
        vz = (T)(-gzk * (double)s / 4.0);
    }
    b.c[1][u] = vx;
    b.c[2][u] = vy;
    b.c[3][u] = vz;
}

// Boundary-row constants into the level-0 right-hand side.
template <typename T>
__global__ void k_bc_consts(int nbc, const int *bu, const float *bconst, Vec4<T> b)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nbc) return;
    int uc = bu[q];
    b.c[uc & 3][uc >> 2] = (T)bconst[q];
}

// ---------------------------------------------------------------------------
// Deterministic reductions: fixed grid, grid-stride, block tree, then one
// block sums the partials in order.

__device__ __forceinline__ double block_sum(double v, double *sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double s = 0;
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    __syncthreads();
    return s;
}

// nd dot products of 4-field vectors: out[q] = sum a_q . b_q (pairs given by
// pointer tables), skipping the pinned pressure cell when skip_node >= 0.
// One sweep over the nodes for all pairs: a vector shared by several pairs
// (the new direction against every stored one) comes from DRAM once and is
// re-read from L1.
// ND, the number of pairs, is a template parameter: the accumulators stay in
// registers whatever ND is, and the node loop is unrolled so that each thread
// has several independent loads in flight (one load at a time per thread left
// the sweep latency-bound at a fraction of the HBM bandwidth).
template <int ND>
__global__ void k_dots_partial(DotJobs jobs, int n, int skip_node, double *partial)
{
    __shared__ double sh[32];
    double s[ND];
#pragma unroll
    for (int q = 0; q < ND; q++) s[q] = 0;
    const int stride = gridDim.x * blockDim.x;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const double *a[ND], *b[ND];
#pragma unroll
        for (int q = 0; q < ND; q++) { a[q] = jobs.j[q].a[c]; b[q] = jobs.j[q].b[c]; }
#pragma unroll 4
        for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride) {
            if (c == 0 && u == skip_node) continue;
#pragma unroll
            for (int q = 0; q < ND; q++) s[q] += __ldg(a[q] + u) * __ldg(b[q] + u);
        }
    }
#pragma unroll
    for (int q = 0; q < ND; q++) {
        const double t = block_sum(s[q], sh);
        if (threadIdx.x == 0) partial[q * gridDim.x + blockIdx.x] = t;
    }
}

// k_dots_partial<jobs.nd> on kRedBlocks blocks of kThreads threads
inline cudaError_t launch_dots(cudaStream_t st, const DotJobs &jobs, int n, int skip_node, double *partial)
{
    switch (jobs.nd) {
#define P2_DOTS_CASE(N) \
    case N: k_dots_partial<N><<<kRedBlocks, kThreads, 0, st>>>(jobs, n, skip_node, partial); break;
        P2_DOTS_CASE(1) P2_DOTS_CASE(2) P2_DOTS_CASE(3) P2_DOTS_CASE(4) P2_DOTS_CASE(5) P2_DOTS_CASE(6)
        P2_DOTS_CASE(7) P2_DOTS_CASE(8) P2_DOTS_CASE(9) P2_DOTS_CASE(10) P2_DOTS_CASE(11) P2_DOTS_CASE(12)
        P2_DOTS_CASE(13) P2_DOTS_CASE(14) P2_DOTS_CASE(15) P2_DOTS_CASE(16) P2_DOTS_CASE(17) P2_DOTS_CASE(18)
        P2_DOTS_CASE(19) P2_DOTS_CASE(20)
#undef P2_DOTS_CASE
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

__global__ void k_dots_final(int nd, int nparts, const double *partial, double *out)
{
    __shared__ double sh[32];
    for (int q = 0; q < nd; q++) {
        double s = 0;
        for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += partial[q * nparts + i];
        double t = block_sum(s, sh);
        if (threadIdx.x == 0) out[q] = t;
    }
}

// Sum of volume * b_P over continuity rows and of the volumes (compatibility).
template <typename T>
__device__ __forceinline__ void compat_apply_item(const LevelView<T> &L, T *bp, double s0, double s1, int u)
{
    if (u >= L.n || s1 <= 0) return;
    int j = u % L.ny, i = (u / L.ny) % L.nx, k = u / (L.nx * L.ny);
    if (i == 0 || j == 0 || k == 0 || (L.bcm[u] & BC_P)) return;
    bp[u] -= (T)(s0 / s1);
}
template <typename T>
__global__ void k_compat_apply(LevelView<T> L, T *bp, const double *sums)
{
    pdl_enter();
    compat_apply_item(L, bp, sums[0], sums[1], blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------------------
// Small vector kernels.
__global__ void k_axpy4(int n, const double *alpha, double sign, Vec4<double> y, Vec4<double> x)
{
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    double a = sign * alpha[0];
#pragma unroll
    for (int c = 0; c < 4; c++) y.c[c][u] += a * x.c[c][u];
}

// GCR scalars kept on the device (no host round trip inside an iteration):
// coef[j] = (q, Q_j) / (Q_j, Q_j) for the k stored directions.
__global__ void k_gcr_coef(int k, const double *dots, const double *qq, double *coef)
{
    const int j = threadIdx.x;
    if (j < k) coef[j] = dots[j] / qq[j];
}
// qq_k = (q', q') and alpha = (r, q') / qq_k from dots[0], dots[1]; a
// direction without a positive norm sets flag[0] = 1 and alpha = 0.
__global__ void k_gcr_alpha(const double *dots, double *qqk, double *alpha, double *flag)
{
    if (threadIdx.x != 0) return;
    const double qq = dots[0];
    qqk[0] = qq;
    if (qq > 0) {
        alpha[0] = dots[1] / qq;
    } else {
        alpha[0] = 0;
        flag[0] = 1;
    }
}

// Classical Gram-Schmidt update of the new direction with its dot products:
//   q' = q - sum_j coef_j Q_j (in place), z' = z - sum_j coef_j Z_j (z read
//   from zs, stored as S; z' written to zo, which may be zs),
// and per block the partial sums of (q', q') and (r, q'), in the node loop
// of k_dots_partial (kRedBlocks blocks of kThreads threads, components outer,
// nodes strided, the pinned pressure cell skipped), so the sums are the ones
// a separate dot-product pass over q' would give.  NV, the number of stored
// directions, is a template parameter: the coefficients stay in registers and
// the loads of all directions of a node are issued together.
template <int NV, typename S>
__global__ void k_cgs_update_dots(int n, const double *coef, Vec4<double> q, VecList X, Vec4<S> zs,
                                  Vec4<double> zo, VecList Z, Vec4<double> r, int skip_node, double *partial)
{
    __shared__ double sh[32];
    double cf[NV > 0 ? NV : 1];
#pragma unroll
    for (int j = 0; j < NV; j++) cf[j] = coef[j];
    double sqq = 0, srq = 0;
    const int stride = gridDim.x * blockDim.x;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride) {
            double sy = q.c[c][u], sz = (double)zs.c[c][u];
#pragma unroll
            for (int j = 0; j < NV; j++) {
                sy -= cf[j] * X.v[j][c][u];
                sz -= cf[j] * Z.v[j][c][u];
            }
            q.c[c][u] = sy;
            zo.c[c][u] = sz;
            if (c == 0 && u == skip_node) continue;
            sqq += sy * sy;
            srq += r.c[c][u] * sy;
        }
    }
    const double t0 = block_sum(sqq, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = t0;
    const double t1 = block_sum(srq, sh);
    if (threadIdx.x == 0) partial[gridDim.x + blockIdx.x] = t1;
}

// k_cgs_update_dots<nv, S> on kRedBlocks blocks of kThreads threads
template <typename S>
inline cudaError_t launch_cgs_update_dots(cudaStream_t st, int nv, int n, const double *coef, const Vec4<double> &q,
                                          const VecList &X, const Vec4<S> &zs, const Vec4<double> &zo,
                                          const VecList &Z, const Vec4<double> &r, int skip_node, double *partial)
{
    switch (nv) {
#define P2_CGS_CASE(N)                                                                                          \
    case N:                                                                                                     \
        k_cgs_update_dots<N, S><<<kRedBlocks, kThreads, 0, st>>>(n, coef, q, X, zs, zo, Z, r, skip_node, partial); \
        break;
        P2_CGS_CASE(0) P2_CGS_CASE(1) P2_CGS_CASE(2) P2_CGS_CASE(3) P2_CGS_CASE(4) P2_CGS_CASE(5) P2_CGS_CASE(6)
        P2_CGS_CASE(7) P2_CGS_CASE(8) P2_CGS_CASE(9) P2_CGS_CASE(10) P2_CGS_CASE(11) P2_CGS_CASE(12)
        P2_CGS_CASE(13) P2_CGS_CASE(14) P2_CGS_CASE(15) P2_CGS_CASE(16) P2_CGS_CASE(17)
#undef P2_CGS_CASE
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

__global__ void k_f32_to_f64(int n, Vec4<float> a, Vec4<double> b)
{
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
#pragma unroll
    for (int c = 0; c < 4; c++) b.c[c][u] = (double)a.c[c][u];
}

// Pressure shift so that the pinned cell holds pin_value (move3mgNew.c:2834-2855).
__global__ void k_pressure_shift_value(const double *p, int pin, double pin_value, double *shift)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) shift[0] = pin >= 0 ? pin_value - p[pin] : 0.0;
}
__global__ void k_pressure_shift(int nx, int ny, int nz, double *p, const double *shift)
{
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nx * ny * nz) return;
    int j = u % ny, i = (u / ny) % nx, k = u / (nx * ny);
    if (i > 0 && j > 0 && k > 0) p[u] += shift[0];
}

}  // namespace p2
