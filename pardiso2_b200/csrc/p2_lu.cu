// Coarsest-level direct solve: FP64 LU with partial pivoting and its explicit
// inverse, all on the device.
//
// Replaces the MKL PARDISO call of the reference (pardiso/gaus3mg_SerieMG.c:
// 64-309; phases 11/22/33 at 170/185/198).  The coarsest operator is reduced
// to its free unknowns (boundary rows, ghosts and the pinned pressure cell are
// eliminated).  In that ordering it is banded: row r has non-zeros only in
// columns [r - kl, r + ku], about one z-plane of unknowns either side.  The
// factorisation is the right-looking blocked LU of LAPACK's gbtrf, restricted
// to the band and kept in dense column-major storage:
//   per panel of kPB columns at k0 (rows [k0, r1), r1 = k0 + kPB + kl):
//     1. factor the panel in registers or shared memory (pivot = largest |a|,
//        smallest row on ties), row interchanges applied inside the panel only;
//     2. apply the interchanges to the columns [k0 + kPB, c1) (c1 = r1 + ku,
//        the reach of U after pivoting) and solve U12 = L11^-1 A12;
//     3. A22 -= L21 U12 on rows [k0 + kPB, r1) x columns [k0 + kPB, c1).
// Interchanges are not applied to earlier columns, so L is the product of the
// panels' (P_k, L_k) in order.  The inverse X = A^-1 replays them on the
// identity (forward) and then solves with the banded U (backward), so each
// V-cycle applies the coarsest solve as one GEMV.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "p2_internal.cuh"

namespace p2 {

constexpr int kPB = 32;                                  // panel width
constexpr int kMaxPanelBytes = 200 * 1024;               // shared-memory panel
constexpr int kMaxPanelRows = kMaxPanelBytes / (8 * kPB);  // 800 rows

// ---------------------------------------------------------------------------
// Panel in shared memory with one thread per panel row and the pivot order
// tracked instead of rows swapped: at step jj every row not yet chosen
// competes (largest |a|, lowest storage row on ties), the chosen row stays
// where it is and the others are eliminated against it.  Two barriers per
// column.  At the end the LAPACK-style interchange sequence (swap logical rows
// jj and ipiv[jj]) that produces the same final row order is rebuilt, and the
// rows are written back in that order: the result of a row-swapping panel
// factorisation (partial pivoting, LAPACK getf2) of the same columns.
constexpr int kTrackThreads = 1024;
static_assert(kMaxPanelRows <= kTrackThreads, "one thread per panel row");

__global__ void __launch_bounds__(kTrackThreads) k_panel_track(double *A, int lda, int k0, int nb, int r1, int *ipiv,
                                                               int *info)
{
    extern __shared__ double P[];
    __shared__ double wv[32];
    __shared__ int wi[32];
    __shared__ int prow[kPB];
    __shared__ int lmap[kMaxPanelRows], linv[kMaxPanelRows];
    const int m = r1 - k0;
    for (int t = threadIdx.x; t < m * nb; t += blockDim.x) {
        int r = t % m, c = t / m;
        P[t] = A[(size_t)(k0 + c) * lda + k0 + r];
    }
    __syncthreads();
    const int row = threadIdx.x, lane = row & 31, w = row >> 5;
    bool live = row < m;  // not yet chosen as a pivot
    for (int jj = 0; jj < nb; jj++) {
        double best = live ? fabs(P[(size_t)jj * m + row]) : -1.0;
        int bi = live ? row : 0x7fffffff;
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_down_sync(0xffffffffu, best, o);
            int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        if (lane == 0) { wv[w] = best; wi[w] = bi; }
        __syncthreads();
        // every warp reduces the per-warp candidates itself (butterfly: all lanes agree)
        best = lane < (int)(blockDim.x >> 5) ? wv[lane] : -1.0;
        bi = lane < (int)(blockDim.x >> 5) ? wi[lane] : 0x7fffffff;
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_xor_sync(0xffffffffu, best, o);
            int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        const int p = bi;
        if (row == 0) {
            prow[jj] = p;
            if (!(best > 0.0) && *info == 0) *info = k0 + jj + 1;
        }
        const double pv = P[(size_t)jj * m + p];
        const double inv = pv != 0.0 ? 1.0 / pv : 0.0;
        if (row == p) live = false;
        if (live) {
            const double l = P[(size_t)jj * m + row] * inv;
            P[(size_t)jj * m + row] = l;
#pragma unroll
            for (int c = 0; c < kPB; c++)
                if (c > jj && c < nb) P[(size_t)c * m + row] -= l * P[(size_t)c * m + p];
        }
        __syncthreads();
    }
    // interchange sequence and final row order
    for (int r = threadIdx.x; r < m; r += blockDim.x) { lmap[r] = r; linv[r] = r; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int jj = 0; jj < nb; jj++) {
            const int p = prow[jj], q = linv[p];   // logical position of the chosen row (q >= jj)
            ipiv[k0 + jj] = k0 + q;
            const int a = lmap[jj];
            lmap[jj] = p; linv[p] = jj;
            lmap[q] = a;  linv[a] = q;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < m * nb; t += blockDim.x) {
        int r = t % m, c = t / m;
        A[(size_t)(k0 + c) * lda + k0 + r] = P[(size_t)c * m + lmap[r]];
    }
}

// The same panel factorisation with each row held in the registers of one
// thread (the column loop fully unrolled, so every index is static), for
// panels of at most kRegPanelRows rows.  Per column one barrier: every warp
// reduces its candidates with shuffles and the winning lane of each warp
// writes its whole row to shared memory; after the barrier every thread picks
// the overall winner from the per-warp candidates and eliminates against the
// copy of the pivot row.  Pivot choice (largest |a|, lowest row on ties), the
// rebuilt interchange sequence and the output are those of k_panel_track.
constexpr int kRegPanelRows = 640;

__global__ void __launch_bounds__(kRegPanelRows) k_panel_reg(double *A, int lda, int k0, int r1, int *ipiv,
                                                             int *info)
{
    __shared__ double cand[kRegPanelRows / 32][2][kPB];  // per-warp candidate row, double-buffered by column parity
    __shared__ double cval[kRegPanelRows / 32][2];
    __shared__ int cidx[kRegPanelRows / 32][2];
    __shared__ int prow[kPB];
    __shared__ int lmap[kRegPanelRows], linv[kRegPanelRows];
    const int m = r1 - k0;
    const int row = threadIdx.x, lane = row & 31, w = row >> 5, nw = blockDim.x >> 5;
    double v[kPB];
#pragma unroll
    for (int c = 0; c < kPB; c++) v[c] = row < m ? A[(size_t)(k0 + c) * lda + k0 + row] : 0.0;
    bool live = row < m;
#pragma unroll
    for (int jj = 0; jj < kPB; jj++) {
        const int buf = jj & 1;
        double best = live ? fabs(v[jj]) : -1.0;
        int bi = live ? row : 0x7fffffff;
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_xor_sync(0xffffffffu, best, o);
            int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        if (row == bi) {  // this warp's candidate publishes its row
            cval[w][buf] = best;
            cidx[w][buf] = bi;
#pragma unroll
            for (int c = 0; c < kPB; c++)
                if (c >= jj) cand[w][buf][c] = v[c];
        }
        if (lane == 0 && bi == 0x7fffffff) {  // warp without live rows
            cval[w][buf] = -1.0;
            cidx[w][buf] = 0x7fffffff;
        }
        __syncthreads();
        double gb = lane < nw ? cval[lane][buf] : -1.0;
        int gi = lane < nw ? cidx[lane][buf] : 0x7fffffff;
        int gw = lane;
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_xor_sync(0xffffffffu, gb, o);
            int oi = __shfl_xor_sync(0xffffffffu, gi, o);
            int ow = __shfl_xor_sync(0xffffffffu, gw, o);
            if (ov > gb || (ov == gb && oi < gi)) { gb = ov; gi = oi; gw = ow; }
        }
        const int p = gi;
        if (row == 0) {
            prow[jj] = p;
            if (!(gb > 0.0) && *info == 0) *info = k0 + jj + 1;
        }
        const double pv = cand[gw][buf][jj];
        const double inv = pv != 0.0 ? 1.0 / pv : 0.0;
        if (row == p) live = false;
        if (live) {
            const double l = v[jj] * inv;
            v[jj] = l;
#pragma unroll
            for (int c = jj + 1; c < kPB; c++) v[c] -= l * cand[gw][buf][c];
        }
        // the next column writes the other buffer, so one barrier per column suffices
    }
    // interchange sequence and final row order (as k_panel_track)
    for (int r = threadIdx.x; r < m; r += blockDim.x) { lmap[r] = r; linv[r] = r; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int jj = 0; jj < kPB; jj++) {
            const int p = prow[jj], q = linv[p];
            ipiv[k0 + jj] = k0 + q;
            const int a = lmap[jj];
            lmap[jj] = p; linv[p] = jj;
            lmap[q] = a;  linv[a] = q;
        }
    }
    __syncthreads();
    // rows go back to their final positions: the destination of physical row r is linv[r]
    if (row < m) {
        const int dst = linv[row];
#pragma unroll
        for (int c = 0; c < kPB; c++) A[(size_t)(k0 + c) * lda + k0 + dst] = v[c];
    }
}

// Same factorisation in global memory, one block, for bands too wide for the
// shared-memory panel.
__global__ void k_panel_global(double *A, int lda, int k0, int nb, int r1, int *ipiv, int *info)
{
    __shared__ double sv[32];
    __shared__ int si[32];
    __shared__ int piv;
    for (int jj = 0; jj < nb; jj++) {
        int j = k0 + jj;
        double *colj = A + (size_t)j * lda;
        double best = -1.0;
        int bi = r1;
        for (int i = j + threadIdx.x; i < r1; i += blockDim.x) {
            double v = fabs(colj[i]);
            if (v > best) { best = v; bi = i; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_down_sync(0xffffffffu, best, o);
            int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane == 0) { sv[w] = best; si[w] = bi; }
        __syncthreads();
        if (threadIdx.x < 32) {
            int nw = blockDim.x >> 5;
            best = threadIdx.x < nw ? sv[threadIdx.x] : -1.0;
            bi = threadIdx.x < nw ? si[threadIdx.x] : r1;
            for (int o = 16; o > 0; o >>= 1) {
                double ov = __shfl_down_sync(0xffffffffu, best, o);
                int oi = __shfl_down_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
            }
            if (threadIdx.x == 0) {
                if (!(best > 0.0)) {
                    if (*info == 0) *info = j + 1;
                    bi = j;
                }
                piv = bi;
                ipiv[j] = bi;
            }
        }
        __syncthreads();
        int p = piv;
        if (p != j)
            for (int c = k0 + threadIdx.x; c < k0 + nb; c += blockDim.x) {
                double t = A[(size_t)c * lda + j];
                A[(size_t)c * lda + j] = A[(size_t)c * lda + p];
                A[(size_t)c * lda + p] = t;
            }
        __syncthreads();
        double d = colj[j];
        if (d != 0.0) {
            double inv = 1.0 / d;
            for (int i = j + 1 + threadIdx.x; i < r1; i += blockDim.x) colj[i] *= inv;
        }
        __syncthreads();
        for (int i = j + 1 + threadIdx.x; i < r1; i += blockDim.x) {
            double l = colj[i];
            for (int c = j + 1; c < k0 + nb; c++) A[(size_t)c * lda + i] -= l * A[(size_t)c * lda + j];
        }
        __syncthreads();
    }
}

// Triangular solves on the columns c in [c0, c1) of B, one warp per column:
//   lower: apply the panel's interchanges (rows k0..) to the column, then
//          B[k0:k0+nb, c] = L11^-1 B[k0:k0+nb, c], L11 unit lower from A;
//   upper: B[k0:k0+nb, c] = U11^-1 B[k0:k0+nb, c], U11 non-unit upper from A.
// Lane r owns row k0 + r; the solved value of each row is broadcast with a
// shuffle and the lanes below (lower) or above (upper) subtract its multiple.
// The interchange sequence is first turned into one permutation: warp 0
// replays the nb swaps on the set of rows they touch (rows k0..k0+nb and the
// pivot rows below, at most 2 nb), recording for each slot the row whose
// value ends there; every column then gathers that set with independent
// loads, solves, and stores the set back.  kTrsmWarps columns per block.
constexpr int kTrsmWarps = 8;

__global__ void __launch_bounds__(32 * kTrsmWarps) k_perm_trsm_lower_w(const double *A, int lda, int k0, int nb,
                                                                       const int *ipiv, double *B, int ldb, int c0,
                                                                       int c1)
{
    __shared__ double L[kPB][kPB + 1];
    __shared__ int S[2 * kPB], src[2 * kPB];
    __shared__ int nS;
    for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
        int r = t % nb, s = t / nb;
        L[r][s] = A[(size_t)(k0 + s) * lda + k0 + r];
    }
    if (threadIdx.x < 32) {  // the panel's interchanges as one permutation
        const int lane = threadIdx.x;
        int cnt = nb;
        if (lane < nb) { S[lane] = k0 + lane; src[lane] = k0 + lane; }
        __syncwarp();
        for (int jj = 0; jj < nb; jj++) {
            const int p = ipiv[k0 + jj];
            int sp;
            if (p < k0 + nb) {
                sp = p - k0;
            } else {
                const int idx = nb + lane;
                const bool hit = idx < cnt && S[idx] == p;
                const unsigned bal = __ballot_sync(0xffffffffu, hit);
                if (bal) {
                    sp = nb + __ffs(bal) - 1;
                } else {
                    sp = cnt;
                    if (lane == 0) { S[cnt] = p; src[cnt] = p; }
                    cnt++;
                }
            }
            __syncwarp();
            if (lane == 0 && sp != jj) { int t = src[jj]; src[jj] = src[sp]; src[sp] = t; }
            __syncwarp();
        }
        if (lane == 0) nS = cnt;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int c = c0 + blockIdx.x * kTrsmWarps + (threadIdx.x >> 5);
    if (c >= c1) return;
    double *col = B + (size_t)c * ldb;
    const int ne = nS - nb;
    // gather everything the permutation moves before writing any of it
    double x = lane < nb ? col[src[lane]] : 0.0;
    double e = lane < ne ? col[src[nb + lane]] : 0.0;
    for (int r = 0; r < nb; r++) {
        const double xr = __shfl_sync(0xffffffffu, x, r);
        if (lane > r && lane < nb) x -= L[lane][r] * xr;
    }
    e = __shfl_sync(0xffffffffu, e, lane);  // consumes every gathered value before the first store
    __syncwarp();
    if (lane < nb) col[k0 + lane] = x;
    if (lane < ne) col[S[nb + lane]] = e;
}

__global__ void __launch_bounds__(32 * kTrsmWarps) k_trsm_upper_w(const double *A, int lda, int k0, int nb, double *B,
                                                                  int ldb, int c0, int c1)
{
    __shared__ double U[kPB][kPB + 1];
    __shared__ double Ur[kPB];
    for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
        int r = t % nb, s = t / nb;
        U[r][s] = A[(size_t)(k0 + s) * lda + k0 + r];
    }
    __syncthreads();
    if (threadIdx.x < nb) Ur[threadIdx.x] = 1.0 / U[threadIdx.x][threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int c = c0 + blockIdx.x * kTrsmWarps + (threadIdx.x >> 5);
    if (c >= c1) return;
    double *col = B + (size_t)c * ldb + k0;
    double x = lane < nb ? col[lane] : 0.0;
    for (int r = nb - 1; r >= 0; r--) {
        if (lane == r) x *= Ur[r];
        const double xr = __shfl_sync(0xffffffffu, x, r);
        if (lane < r) x -= U[lane][r] * xr;
    }
    if (lane < nb) col[lane] = x;
}

// C[m x nn] -= A[m x kk] * B[kk x nn], column-major, FP64.  64x64 tile per
// block of 256 threads, 4x4 outputs per thread, kk-step 16 through shared memory.
__global__ void __launch_bounds__(256) k_dgemm_sub(int m, int nn, int kk, const double *A, int lda,
                                                   const double *B, int ldb, double *C, int ldc)
{
    __shared__ double As[16][64 + 1];
    __shared__ double Bs[16][64 + 1];
    int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    int row0 = blockIdx.x * 64, col0 = blockIdx.y * 64;
    double acc[4][4] = {};
    for (int k0 = 0; k0 < kk; k0 += 16) {
        for (int t = threadIdx.x; t < 16 * 64; t += 256) {
            int r = t % 64, s = t / 64;  // A tile: rows r, k s
            int gr = row0 + r, gk = k0 + s;
            As[s][r] = (gr < m && gk < kk) ? A[(size_t)gk * lda + gr] : 0.0;
            int kc = t % 16, cc = t / 16;  // B tile: k kc, cols cc
            int gk2 = k0 + kc, gc = col0 + cc;
            Bs[kc][cc] = (gk2 < kk && gc < nn) ? B[(size_t)gc * ldb + gk2] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < 16; s++) {
            double a[4], b[4];
#pragma unroll
            for (int q = 0; q < 4; q++) { a[q] = As[s][tx + 16 * q]; b[q] = Bs[s][ty + 16 * q]; }
#pragma unroll
            for (int q = 0; q < 4; q++)
#pragma unroll
                for (int r = 0; r < 4; r++) acc[q][r] += a[q] * b[r];
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
        for (int r = 0; r < 4; r++) {
            int gr = row0 + tx + 16 * q, gc = col0 + ty + 16 * r;
            if (gr < m && gc < nn) C[(size_t)gc * ldc + gr] -= acc[q][r];
        }
}

__global__ void k_identity(double *B, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) B[(size_t)i * n + i] = 1.0;
}

__global__ void k_d2f(size_t n, const double *a, float *b)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

// C[m x nn] -= A[m x kk] * B[kk x nn] for kk <= kPB (every update of the
// blocked LU has kk = panel width): the whole kk slab of A and B in shared
// memory with one barrier, the block's C values fetched into registers before
// the products so their latency overlaps the tile loads.  TM x TN tile per
// block of 256 threads (16 x 16 grid, TM/16 x TN/16 outputs per thread).
template <int TM, int TN>
__global__ void __launch_bounds__(256) k_dgemm_k32(int m, int nn, int kk, const double *A, int lda, const double *B,
                                                   int ldb, double *C, int ldc)
{
    constexpr int RM = TM / 16, RN = TN / 16;
    __shared__ double As[kPB][TM + 1];
    __shared__ double Bs[kPB][TN + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int row0 = blockIdx.x * TM, col0 = blockIdx.y * TN;
    double cv[RM][RN];
#pragma unroll
    for (int q = 0; q < RM; q++)
#pragma unroll
        for (int r = 0; r < RN; r++) {
            const int gr = row0 + tx + 16 * q, gc = col0 + ty + 16 * r;
            cv[q][r] = (gr < m && gc < nn) ? C[(size_t)gc * ldc + gr] : 0.0;
        }
    for (int t = threadIdx.x; t < kPB * TM; t += 256) {
        const int r = t % TM, s = t / TM;
        As[s][r] = (row0 + r < m && s < kk) ? A[(size_t)s * lda + row0 + r] : 0.0;
    }
    for (int t = threadIdx.x; t < kPB * TN; t += 256) {
        const int kc = t % kPB, cc = t / kPB;
        Bs[kc][cc] = (kc < kk && col0 + cc < nn) ? B[(size_t)(col0 + cc) * ldb + kc] : 0.0;
    }
    __syncthreads();
    double acc[RM][RN];
#pragma unroll
    for (int q = 0; q < RM; q++)
#pragma unroll
        for (int r = 0; r < RN; r++) acc[q][r] = 0.0;
#pragma unroll 8
    for (int s = 0; s < kPB; s++) {
        double a[RM], b[RN];
#pragma unroll
        for (int q = 0; q < RM; q++) a[q] = As[s][tx + 16 * q];
#pragma unroll
        for (int r = 0; r < RN; r++) b[r] = Bs[s][ty + 16 * r];
#pragma unroll
        for (int q = 0; q < RM; q++)
#pragma unroll
            for (int r = 0; r < RN; r++) acc[q][r] += a[q] * b[r];
    }
#pragma unroll
    for (int q = 0; q < RM; q++)
#pragma unroll
        for (int r = 0; r < RN; r++) {
            const int gr = row0 + tx + 16 * q, gc = col0 + ty + 16 * r;
            if (gr < m && gc < nn) C[(size_t)gc * ldc + gr] = cv[q][r] - acc[q][r];
        }
}

static void dgemm_sub(cudaStream_t st, int m, int nn, int kk, const double *A, int lda, const double *B, int ldb,
                      double *C, int ldc)
{
    if (m <= 0 || nn <= 0 || kk <= 0) return;
    if (kk <= kPB) {
        const long big = (long)((m + 63) / 64) * ((nn + 63) / 64);
        if (big >= 2 * 148) {
            dim3 grid((m + 63) / 64, (nn + 63) / 64);
            k_dgemm_k32<64, 64><<<grid, 256, 0, st>>>(m, nn, kk, A, lda, B, ldb, C, ldc); P2_COUNT_LAUNCH();
        } else {
            dim3 grid((m + 31) / 32, (nn + 31) / 32);
            k_dgemm_k32<32, 32><<<grid, 256, 0, st>>>(m, nn, kk, A, lda, B, ldb, C, ldc); P2_COUNT_LAUNCH();
        }
        return;
    }
    dim3 grid((m + 63) / 64, (nn + 63) / 64);
    k_dgemm_sub<<<grid, 256, 0, st>>>(m, nn, kk, A, lda, B, ldb, C, ldc); P2_COUNT_LAUNCH();
}


// Diagnostic per-kernel-type device times of the LU (environment variable
// P2CUDA_LU_TIMING=1): every launch is bracketed by events and waited for, so
// the totals are exact per kernel but the run itself is slower.
struct LuTimer {
    bool on = false;
    cudaEvent_t a = nullptr, b = nullptr;
    double ms[4] = {0, 0, 0, 0};  // panel, lower TRSM, GEMM, upper TRSM
    int cnt[4] = {0, 0, 0, 0};
    cudaStream_t st = nullptr;
    void begin()
    {
        if (on) cudaEventRecord(a, st);
    }
    void end(int kind)
    {
        if (!on) return;
        cudaEventRecord(b, st);
        cudaEventSynchronize(b);
        float t = 0;
        cudaEventElapsedTime(&t, a, b);
        ms[kind] += t;
        cnt[kind]++;
    }
};

// Factor the banded A (n x n, column-major, lower/upper half-bandwidths kl,
// ku) in place and write its inverse into Ainv.  Returns 0 or the first
// zero-pivot column + 1.  marks (optional, 2 events) are recorded after the
// factorisation and after the forward half of the inverse.
// panels per group in the backward half of the inverse
constexpr int kInvGroup = 4;

static void lu_issue(cudaStream_t st, double *A, int n, int kl, int ku, double *Ainv, int *d_ipiv, int *d_info,
                     cudaEvent_t *marks, LuTimer &T)
{
    const bool smem = kPB + kl <= kMaxPanelRows;
    P2_CUDA_TRY(cudaMemsetAsync(d_info, 0, sizeof(int), st));
    for (int k0 = 0; k0 < n; k0 += kPB) {
        const int nb = std::min(kPB, n - k0);
        const int r1 = std::min(n, k0 + nb + kl);
        const int c1 = std::min(n, r1 + ku);
        if (smem) {
            size_t bytes = sizeof(double) * (size_t)(r1 - k0) * nb;
            const int thr = ((r1 - k0) + 31) / 32 * 32;  // one thread per panel row
            T.begin();
            if (nb == kPB && r1 - k0 <= kRegPanelRows) {
                k_panel_reg<<<1, thr, 0, st>>>(A, n, k0, r1, d_ipiv, d_info); P2_COUNT_LAUNCH();
            } else {
                k_panel_track<<<1, thr, bytes, st>>>(A, n, k0, nb, r1, d_ipiv, d_info); P2_COUNT_LAUNCH();
            }
            T.end(0);
        } else {
            k_panel_global<<<1, 1024, 0, st>>>(A, n, k0, nb, r1, d_ipiv, d_info); P2_COUNT_LAUNCH();
        }
        const int cb = k0 + nb;
        if (c1 > cb) {
            T.begin();
            k_perm_trsm_lower_w<<<(c1 - cb + kTrsmWarps - 1) / kTrsmWarps, 32 * kTrsmWarps, 0, st>>>(
                A, n, k0, nb, d_ipiv, A, n, cb, c1); P2_COUNT_LAUNCH();
            T.end(1);
            T.begin();
            dgemm_sub(st, r1 - cb, c1 - cb, nb, A + (size_t)k0 * n + cb, n, A + (size_t)cb * n + k0, n,
                      A + (size_t)cb * n + cb, n);
            T.end(2);
        }
    }
    if (marks) P2_CUDA_TRY(cudaEventRecord(marks[0], st));
    // forward: replay (P_k, L_k) on the identity; rows [k0, r1) of the partial
    // product only have non-zeros in columns [0, r1)
    P2_CUDA_TRY(cudaMemsetAsync(Ainv, 0, sizeof(double) * (size_t)n * n, st));
    k_identity<<<(n + 255) / 256, 256, 0, st>>>(Ainv, n); P2_COUNT_LAUNCH();
    for (int k0 = 0; k0 < n; k0 += kPB) {
        const int nb = std::min(kPB, n - k0);
        const int r1 = std::min(n, k0 + nb + kl);
        T.begin();
        k_perm_trsm_lower_w<<<(r1 + kTrsmWarps - 1) / kTrsmWarps, 32 * kTrsmWarps, 0, st>>>(A, n, k0, nb, d_ipiv,
                                                                                         Ainv, n, 0, r1); P2_COUNT_LAUNCH();
        T.end(1);
        const int cb = k0 + nb;
        T.begin();
        if (r1 > cb) dgemm_sub(st, r1 - cb, r1, nb, A + (size_t)k0 * n + cb, n, Ainv + k0, n, Ainv + cb, n);
        T.end(2);
    }
    if (marks) P2_CUDA_TRY(cudaEventRecord(marks[1], st));
    // backward: U X = Y with U's band (kl + ku above the diagonal), in groups
    // of kInvGroup panels: inside a group every panel's rows are solved and
    // propagated to the group's rows above it; then the rows above the group
    // that U couples to it (within kl + ku) get one update with K = the
    // group's height, instead of one K = kPB update per panel
    const int kuu = std::min(n - 1, kl + ku);
    const int G = kInvGroup * kPB;
    for (int g0 = ((n - 1) / G) * G; g0 >= 0; g0 -= G) {
        const int g1 = std::min(n, g0 + G);
        for (int k0 = g0 + ((g1 - 1 - g0) / kPB) * kPB; k0 >= g0; k0 -= kPB) {
            const int nb = std::min(kPB, n - k0);
            T.begin();
            k_trsm_upper_w<<<(n + kTrsmWarps - 1) / kTrsmWarps, 32 * kTrsmWarps, 0, st>>>(A, n, k0, nb, Ainv, n, 0,
                                                                                       n); P2_COUNT_LAUNCH();
            T.end(3);
            const int a = std::max(g0, k0 - kuu);
            T.begin();
            if (k0 > a) dgemm_sub(st, k0 - a, n, nb, A + (size_t)k0 * n + a, n, Ainv + k0, n, Ainv + a, n);
            T.end(2);
        }
        const int a = std::max(0, g0 - kuu);
        T.begin();
        if (g0 > a) dgemm_sub(st, g0 - a, n, g1 - g0, A + (size_t)g0 * n + a, n, Ainv + g0, n, Ainv + a, n);
        T.end(2);
    }
    P2_CUDA_TRY(cudaGetLastError());
}

int band_lu_inverse(cudaStream_t st, double *A, int n, int kl, int ku, double *Ainv, int *d_ipiv, int *d_info,
                    cudaEvent_t *marks, LuGraph *cache, bool wait)
{
    kl = std::max(0, std::min(kl, n - 1));
    ku = std::max(0, std::min(ku, n - 1));
    // a per-device attribute, set on the current device (a host-side call)
    if (kPB + kl <= kMaxPanelRows)
        P2_CUDA_TRY(cudaFuncSetAttribute(k_panel_track, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxPanelBytes));
    LuTimer T;
    {
        const char *e = std::getenv("P2CUDA_LU_TIMING");
        T.on = e && e[0] == '1';
        T.st = st;
        if (T.on) {
            P2_CUDA_TRY(cudaEventCreate(&T.a));
            P2_CUDA_TRY(cudaEventCreate(&T.b));
        }
    }
    if (cache && !T.on && !marks) {
        // the ~800 dependent launches replayed as one graph; captured again
        // only when the size, the band or the buffers change
        const bool hit = cache->exec && cache->n == n && cache->kl == kl && cache->ku == ku && cache->A == A &&
                         cache->Ainv == Ainv && cache->ipiv == d_ipiv && cache->info == d_info;
        if (!hit) {
            if (cache->exec) cudaGraphExecDestroy(cache->exec);
            cache->exec = nullptr;
            cudaGraph_t graph;
            long long before = g_launches;
            P2_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            lu_issue(st, A, n, kl, ku, Ainv, d_ipiv, d_info, nullptr, T);
            P2_CUDA_TRY(cudaStreamEndCapture(st, &graph));
            cache->kernels = g_launches - before;
            g_launches = before;
            cudaError_t e = cudaGraphInstantiate(&cache->exec, graph, 0);
            cudaGraphDestroy(graph);
            P2_CUDA_TRY(e);
            cache->n = n; cache->kl = kl; cache->ku = ku; cache->A = A; cache->Ainv = Ainv;
            cache->ipiv = d_ipiv; cache->info = d_info;
        }
        P2_CUDA_TRY(cudaGraphLaunch(cache->exec, st));
        g_launches += cache->kernels;
    } else {
        lu_issue(st, A, n, kl, ku, Ainv, d_ipiv, d_info, marks, T);
    }
    if (T.on) {
        std::fprintf(stderr, "p2cuda LU timing: panel %.3f ms (%d), lower TRSM %.3f ms (%d), GEMM %.3f ms (%d), "
                     "upper TRSM %.3f ms (%d)\n", T.ms[0], T.cnt[0], T.ms[1], T.cnt[1], T.ms[2], T.cnt[2], T.ms[3],
                     T.cnt[3]);
        cudaEventDestroy(T.a);
        cudaEventDestroy(T.b);
    }
    int info = 0;
    if (!wait) return 0;  // the caller reads d_info once the stream has finished
    P2_CUDA_TRY(cudaMemcpyAsync(&info, d_info, sizeof(int), cudaMemcpyDeviceToHost, st));
    P2_CUDA_TRY(cudaStreamSynchronize(st));
    return info;
}

void d2f(cudaStream_t st, size_t n, const double *a, float *b)
{
    k_d2f<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, a, b); P2_COUNT_LAUNCH();
}

}  // namespace p2
