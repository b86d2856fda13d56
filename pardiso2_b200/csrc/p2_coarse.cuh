// The coarsest level's direct solve as three kernels: gather the free
// unknowns' right-hand side, multiply by the stored inverse (GEMV), scatter
// the solution back (the reference calls MKL PARDISO here,
// gaus3mg_SerieMG.c:170-216; the inverse comes from p2_lu.cu).
#pragma once

#include "p2_kernels.cuh"

namespace p2 {

// b_F = b on the free unknowns of the coarsest level
template <typename T>
__device__ __forceinline__ void coarse_gather_item(int nF, const int *fre, const Vec4<T> &b, T *bF, int q)
{
    if (q >= nF) return;
    int uc = fre[q];
    bF[q] = b.c[uc & 3][uc >> 2];
}
template <typename T>
__global__ void k_coarse_gather(int nF, const int *fre, Vec4<T> b, T *bF)
{
    pdl_enter();
    coarse_gather_item(nF, fre, b, bF, blockIdx.x * blockDim.x + threadIdx.x);
}
template <typename T>
__device__ __forceinline__ void coarse_scatter_item(int nF, const int *fre, const T *xF, const Vec4<T> &x, int q)
{
    if (q >= nF) return;
    int uc = fre[q];
    x.c[uc & 3][uc >> 2] = xF[q];
}
template <typename T>
__global__ void k_coarse_scatter(int nF, const int *fre, const T *xF, Vec4<T> x)
{
    pdl_enter();
    coarse_scatter_item(nF, fre, xF, x, blockIdx.x * blockDim.x + threadIdx.x);
}
// y = Ainv b (column-major n x n) for the rows 32 vb .. 32 vb + 31: a block
// of 256 threads, its 8 warps split the columns, partial sums in part.
template <typename T>
__device__ __forceinline__ void gemv_block(int n, const T *A, const T *b, T *y, int vb, T (*part)[33])
{
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int r = vb * 32 + lane;
    T s = 0;
    if (r < n)
        for (int c = w; c < n; c += 8) s += A[(size_t)c * n + r] * __ldg(b + c);
    part[w][lane] = s;
    __syncthreads();
    if (w == 0 && r < n) {
        T t = 0;
        for (int q = 0; q < 8; q++) t += part[q][lane];
        y[r] = t;
    }
    __syncthreads();
}
template <typename T>
__global__ void k_gemv(int n, const T *A, const T *b, T *y)
{
    pdl_enter();
    __shared__ T part[8][33];
    gemv_block(n, A, b, y, blockIdx.x, part);
}

}  // namespace p2
