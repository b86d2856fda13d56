// Coarsest-level direct solve: dense FP64 LU with partial pivoting and its
// explicit inverse, all on the device.
//
// Replaces the MKL PARDISO call of the reference (pardiso/gaus3mg_SerieMG.c:
// 64-309; phases 11/22/33 at 170/185/198).  The coarsest operator is reduced
// to its free unknowns (boundary rows, ghosts and the pinned pressure cell are
// eliminated), factored once per solve (P A = L U, right-looking, panel width
// kNB), and inverted (X = U^-1 L^-1 P) so that each V-cycle applies it as one
// GEMV on the B200.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "p2_internal.cuh"

namespace p2 {

constexpr int kNB = 32;

// ---------------------------------------------------------------------------
// Panel factorisation of columns [k0, k0+nb) over rows [k0, n) (column-major,
// leading dimension n), one block.  Pivot: largest |a|, smallest row on ties.
__global__ void k_lu_panel(double *A, int n, int k0, int nb, int *ipiv, int *info)
{
    __shared__ double sv[32];
    __shared__ int si[32];
    __shared__ int piv;
    for (int jj = 0; jj < nb; jj++) {
        int j = k0 + jj;
        double *colj = A + (size_t)j * n;
        double best = -1.0;
        int bi = n;
        for (int i = j + threadIdx.x; i < n; i += blockDim.x) {
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
            bi = threadIdx.x < nw ? si[threadIdx.x] : n;
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
                double t = A[(size_t)c * n + j];
                A[(size_t)c * n + j] = A[(size_t)c * n + p];
                A[(size_t)c * n + p] = t;
            }
        __syncthreads();
        double d = colj[j];
        if (d != 0.0) {
            double inv = 1.0 / d;
            for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) colj[i] *= inv;
        }
        __syncthreads();
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
            double l = colj[i];
            for (int c = j + 1; c < k0 + nb; c++) A[(size_t)c * n + i] -= l * A[(size_t)c * n + j];
        }
        __syncthreads();
    }
}

// Apply the panel's row interchanges to the columns outside the panel.
__global__ void k_lu_swap(double *A, int n, int k0, int nb, const int *ipiv)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n || (c >= k0 && c < k0 + nb)) return;
    double *col = A + (size_t)c * n;
    for (int jj = 0; jj < nb; jj++) {
        int j = k0 + jj, p = ipiv[j];
        if (p != j) { double t = col[j]; col[j] = col[p]; col[p] = t; }
    }
}

// B[k0:k0+nb, c] = L11^-1 B[k0:k0+nb, c] (unit lower) for columns c in [c0, c1);
// L11 = A[k0:k0+nb, k0:k0+nb].
__global__ void k_trsm_lower(const double *A, int lda, int k0, int nb, double *B, int ldb, int c0, int c1)
{
    __shared__ double L[kNB][kNB + 1];
    for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
        int r = t % nb, s = t / nb;
        L[r][s] = A[(size_t)(k0 + s) * lda + k0 + r];
    }
    __syncthreads();
    int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= c1) return;
    double x[kNB];
    double *col = B + (size_t)c * ldb + k0;
    for (int r = 0; r < nb; r++) {
        double v = col[r];
        for (int s = 0; s < r; s++) v -= L[r][s] * x[s];
        x[r] = v;
    }
    for (int r = 0; r < nb; r++) col[r] = x[r];
}

// B[k0:k0+nb, c] = U11^-1 B[k0:k0+nb, c] (non-unit upper).
__global__ void k_trsm_upper(const double *A, int lda, int k0, int nb, double *B, int ldb, int c0, int c1)
{
    __shared__ double U[kNB][kNB + 1];
    for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
        int r = t % nb, s = t / nb;
        U[r][s] = A[(size_t)(k0 + s) * lda + k0 + r];
    }
    __syncthreads();
    int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= c1) return;
    double x[kNB];
    double *col = B + (size_t)c * ldb + k0;
    for (int r = nb - 1; r >= 0; r--) {
        double v = col[r];
        for (int s = r + 1; s < nb; s++) v -= U[r][s] * x[s];
        x[r] = v / U[r][r];
    }
    for (int r = 0; r < nb; r++) col[r] = x[r];
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

__global__ void k_perm_identity(double *B, int n, const int *perm)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    B[(size_t)perm[i] * n + i] = 1.0;  // row i of P*I is e_{perm[i]}
}

__global__ void k_d2f(size_t n, const double *a, float *b)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

static void dgemm_sub(cudaStream_t st, int m, int nn, int kk, const double *A, int lda, const double *B, int ldb,
                      double *C, int ldc)
{
    if (m <= 0 || nn <= 0 || kk <= 0) return;
    dim3 grid((m + 63) / 64, (nn + 63) / 64);
    k_dgemm_sub<<<grid, 256, 0, st>>>(m, nn, kk, A, lda, B, ldb, C, ldc); P2_COUNT_LAUNCH();
}

// Factor A (n x n, column-major, overwritten by L\U) and write its inverse
// into Ainv (n x n).  Returns 0 or the first zero-pivot column + 1.
int dense_lu_inverse(cudaStream_t st, double *A, int n, double *Ainv, int *d_ipiv, int *d_info)
{
    P2_CUDA_TRY(cudaMemsetAsync(d_info, 0, sizeof(int), st));
    for (int k0 = 0; k0 < n; k0 += kNB) {
        int nb = std::min(kNB, n - k0);
        k_lu_panel<<<1, 1024, 0, st>>>(A, n, k0, nb, d_ipiv, d_info); P2_COUNT_LAUNCH();
        k_lu_swap<<<(n + 255) / 256, 256, 0, st>>>(A, n, k0, nb, d_ipiv); P2_COUNT_LAUNCH();
        int rest = n - (k0 + nb);
        if (rest > 0) {
            k_trsm_lower<<<(rest + 127) / 128, 128, 0, st>>>(A, n, k0, nb, A, n, k0 + nb, n); P2_COUNT_LAUNCH();
            dgemm_sub(st, rest, rest, nb, A + (size_t)k0 * n + k0 + nb, n, A + (size_t)(k0 + nb) * n + k0, n,
                      A + (size_t)(k0 + nb) * n + k0 + nb, n);
        }
    }
    int info = 0;
    std::vector<int> ipiv(n);
    P2_CUDA_TRY(cudaMemcpyAsync(&info, d_info, sizeof(int), cudaMemcpyDeviceToHost, st));
    P2_CUDA_TRY(cudaMemcpyAsync(ipiv.data(), d_ipiv, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    P2_CUDA_TRY(cudaStreamSynchronize(st));
    if (info) return info;
    std::vector<int> perm(n);
    for (int i = 0; i < n; i++) perm[i] = i;
    for (int j = 0; j < n; j++) std::swap(perm[j], perm[ipiv[j]]);
    // d_ipiv is reused to hold perm
    P2_CUDA_TRY(cudaMemcpyAsync(d_ipiv, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
    P2_CUDA_TRY(cudaMemsetAsync(Ainv, 0, sizeof(double) * (size_t)n * n, st));
    k_perm_identity<<<(n + 255) / 256, 256, 0, st>>>(Ainv, n, d_ipiv); P2_COUNT_LAUNCH();
    // forward: L Y = P I
    for (int k0 = 0; k0 < n; k0 += kNB) {
        int nb = std::min(kNB, n - k0);
        k_trsm_lower<<<(n + 127) / 128, 128, 0, st>>>(A, n, k0, nb, Ainv, n, 0, n); P2_COUNT_LAUNCH();
        int rest = n - (k0 + nb);
        if (rest > 0)
            dgemm_sub(st, rest, n, nb, A + (size_t)k0 * n + k0 + nb, n, Ainv + k0, n, Ainv + k0 + nb, n);
    }
    // backward: U X = Y
    int last = ((n - 1) / kNB) * kNB;
    for (int k0 = last; k0 >= 0; k0 -= kNB) {
        int nb = std::min(kNB, n - k0);
        k_trsm_upper<<<(n + 127) / 128, 128, 0, st>>>(A, n, k0, nb, Ainv, n, 0, n); P2_COUNT_LAUNCH();
        if (k0 > 0) dgemm_sub(st, k0, n, nb, A + (size_t)k0 * n, n, Ainv + k0, n, Ainv, n);
    }
    P2_CUDA_TRY(cudaGetLastError());
    return 0;
}

void d2f(cudaStream_t st, size_t n, const double *a, float *b)
{
    k_d2f<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, a, b); P2_COUNT_LAUNCH();
}

}  // namespace p2
