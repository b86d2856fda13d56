// Marker -> node interpolation (ronurecalc, pardiso/mark3mg.c:630-1133) on the
// device, deterministic and with no floating-point atomics:
//   1. per marker: validity (inside the box, type < 50: mark3mg.c:692) and
//      cell (binary search on the gridlines, m1serch..m3serch 1138-1204);
//   2. stable LSD radix sort of (cell, marker index) — own kernels;
//   3. per cell: the [start, end) range in the sorted order;
//   4. per node: the markers of the <= 8 adjacent cells are merged by marker
//      index and accumulated in that order with the reference's arithmetic
//      (float accumulators, double weights, no fused multiply-add), so the
//      node fields equal those of the reference run on one thread.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <vector>

#include "p2_internal.cuh"
#include "p2_interp.cuh"
#include "p2_solver.h"

namespace p2 {

static inline unsigned nb(long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

__global__ void k_mark_keys(long nmark, const float *mx, const float *my, const float *mz, const signed char *mt,
                            const double *gx, const double *gy, const double *gz, int nx, int ny, int nz,
                            double xsize, double ysize, double zsize, unsigned sentinel, unsigned *key,
                            unsigned *val)
{
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nmark) return;
    float x = mx[q], y = my[q], z = mz[q];
    int t = mt[q];
    unsigned kk = sentinel;
    if (x > 0 && y > 0 && z > 0 && (double)x < xsize && (double)y < ysize && (double)z < zsize && t < 50) {
        int c1 = serch(gx, nx, (double)x), c2 = serch(gy, ny, (double)y), c3 = serch(gz, nz, (double)z);
        kk = (unsigned)c3 * (unsigned)((nx - 1) * (ny - 1)) + (unsigned)c1 * (unsigned)(ny - 1) + (unsigned)c2;
    }
    key[q] = kk;
    val[q] = (unsigned)q;
}

// ---------------------------------------------------------------------------
// Stable LSD radix sort, 8-bit digits.  A tile of kTile keys per block of 256
// threads (8 warps x 16 chunks of 32); per pass: tile histograms, exclusive
// scan in digit-major order, stable scatter (warp match + running counters).
constexpr int kRadixBits = 8, kBuckets = 256, kChunks = 16, kTile = 8 * kChunks * 32;

__global__ void k_radix_hist(long n, const unsigned *key, int shift, unsigned *hist, int ntiles)
{
    __shared__ unsigned h[kBuckets];
    for (int i = threadIdx.x; i < kBuckets; i += blockDim.x) h[i] = 0;
    __syncthreads();
    long base = (long)blockIdx.x * kTile;
    for (int i = threadIdx.x; i < kTile; i += blockDim.x) {
        long q = base + i;
        if (q < n) atomicAdd(&h[(key[q] >> shift) & (kBuckets - 1)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kBuckets; d += blockDim.x) hist[(long)d * ntiles + blockIdx.x] = h[d];
}

// exclusive scan of hist (kBuckets * ntiles entries) in one block
__global__ void k_radix_scan(unsigned *hist, long len)
{
    __shared__ unsigned long long carry;
    __shared__ unsigned long long part[1024];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long base = 0; base < len; base += 1024) {
        long q = base + threadIdx.x;
        unsigned long long v = q < len ? hist[q] : 0;
        part[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            unsigned long long t = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
            __syncthreads();
            part[threadIdx.x] += t;
            __syncthreads();
        }
        unsigned long long incl = part[threadIdx.x];
        if (q < len) hist[q] = (unsigned)(carry + incl - v);
        __syncthreads();
        if (threadIdx.x == 1023) carry += incl;
        __syncthreads();
    }
}

// Device-wide exclusive scan of the histograms (kBuckets * ntiles entries, up
// to millions at 10^8 markers) in three launches: every block scans
// kScanChunk consecutive entries and records its total; one block scans the
// totals (k_radix_scan); every block adds its offset.
constexpr int kScanThreads = 1024, kScanPer = 4, kScanChunk = kScanThreads * kScanPer;

__global__ void __launch_bounds__(kScanThreads) k_scan_local(unsigned *a, long len, unsigned *block_total)
{
    __shared__ unsigned wsum[kScanThreads / 32];
    const long base = (long)blockIdx.x * kScanChunk + (long)threadIdx.x * kScanPer;
    unsigned v[kScanPer], s = 0;
#pragma unroll
    for (int e = 0; e < kScanPer; e++) {
        v[e] = base + e < len ? a[base + e] : 0u;
        s += v[e];
    }
    // inclusive scan of the thread sums: warp shuffles, then the warp totals
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned inc = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {
        unsigned x = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned t = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += t;
        }
        wsum[lane] = x;  // inclusive over warps
    }
    __syncthreads();
    unsigned run = inc - s + (w > 0 ? wsum[w - 1] : 0u);  // exclusive prefix of this thread
#pragma unroll
    for (int e = 0; e < kScanPer; e++) {
        if (base + e < len) a[base + e] = run;
        run += v[e];
    }
    if (threadIdx.x == kScanThreads - 1) block_total[blockIdx.x] = wsum[31];
}

__global__ void __launch_bounds__(kScanThreads) k_scan_add(unsigned *a, long len, const unsigned *block_offset)
{
    const unsigned off = block_offset[blockIdx.x];
    const long base = (long)blockIdx.x * kScanChunk + (long)threadIdx.x * kScanPer;
#pragma unroll
    for (int e = 0; e < kScanPer; e++)
        if (base + e < len) a[base + e] += off;
}

__global__ void k_radix_scatter(long n, const unsigned *key, const unsigned *val, unsigned *key2, unsigned *val2,
                                int shift, const unsigned *offs, int ntiles)
{
    __shared__ unsigned wcnt[8][kBuckets];   // per-warp digit counts, then exclusive offsets
    __shared__ unsigned boff[kBuckets];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < 8 * kBuckets; i += blockDim.x) (&wcnt[0][0])[i] = 0;
    for (int d = threadIdx.x; d < kBuckets; d += blockDim.x) boff[d] = offs[(long)d * ntiles + blockIdx.x];
    __syncthreads();
    long wbase = (long)blockIdx.x * kTile + (long)w * kChunks * 32;
    // pass 1: per-warp counts
    for (int ch = 0; ch < kChunks; ch++) {
        long q = wbase + ch * 32 + lane;
        bool ok = q < n;
        unsigned d = ok ? (key[q] >> shift) & (kBuckets - 1) : 0xffffffffu;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        if (ok && lane == __ffs(peers) - 1) wcnt[w][d] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // exclusive prefix over warps per digit
    for (int d = threadIdx.x; d < kBuckets; d += blockDim.x) {
        unsigned s = boff[d];
        for (int ww = 0; ww < 8; ww++) {
            unsigned c = wcnt[ww][d];
            wcnt[ww][d] = s;
            s += c;
        }
    }
    __syncthreads();
    // pass 2: stable placement
    for (int ch = 0; ch < kChunks; ch++) {
        long q = wbase + ch * 32 + lane;
        bool ok = q < n;
        unsigned kk = ok ? key[q] : 0, vv = ok ? val[q] : 0;
        unsigned d = ok ? (kk >> shift) & (kBuckets - 1) : 0xffffffffu;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        unsigned lt = peers & ((1u << lane) - 1u);
        unsigned pos = 0;
        if (ok) pos = wcnt[w][d] + __popc(lt);
        __syncwarp();
        if (ok && lane == __ffs(peers) - 1) wcnt[w][d] += __popc(peers);
        __syncwarp();
        if (ok) { key2[pos] = kk; val2[pos] = vv; }
    }
}

// cell ranges from the sorted keys (cells without markers keep [0, 0))
__global__ void k_cell_bounds(long n, const unsigned *key, unsigned sentinel, int *start, int *end)
{
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    unsigned k = key[q];
    if (k == sentinel) return;
    if (q == 0 || key[q - 1] != k) start[k] = (int)q;
    if (q == n - 1 || key[q + 1] != k) end[k] = (int)(q + 1);
}

__global__ void k_permute(long n, const unsigned *idx, const float *mx, const float *my, const float *mz,
                          const signed char *mt, float4 *sorted)
{
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    unsigned m = idx[q];
    sorted[q] = make_float4(mx[m], my[m], mz[m], __int_as_float((int)mt[m]));
}

// ---------------------------------------------------------------------------
struct Rock {
    double nu, ro;  // clamped viscosity, density
};

// power-law table per rock type: {flag, marknu, (1 - n) / n, markn0, markn1}
constexpr int kPowerLawStride = 5;

__global__ void k_node_gather(int nx, int ny, int nz, const double *gx, const double *gy, const double *gz,
                              const int *start, const int *end, const unsigned *idx, const float4 *mk,
                              const double *rock_f, const double *rock_ro, double nukoef, int viscmod,
                              double nubeg, double nuend, float *nu, float *ro, float *nxx, float *nxy, float *nxz,
                              float *nyz, const double *pl = nullptr, const double *val1 = nullptr)
{
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nx * ny * nz) return;
    int m2 = u % ny, m1 = (u / ny) % nx, m3 = u / (nx * ny);
    int nx1 = nx - 1, ny1 = ny - 1;
    // the up-to-8 adjacent cells and their cursors
    int cur[8], lim[8], cz[8], cx[8], cy[8], nc = 0;
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++)
            for (int c = 0; c < 2; c++) {
                int c3 = m3 - 1 + a, c1 = m1 - 1 + b, c2 = m2 - 1 + c;
                if (c3 < 0 || c1 < 0 || c2 < 0 || c3 >= nz - 1 || c1 >= nx - 1 || c2 >= ny - 1) continue;
                int cell = c3 * nx1 * ny1 + c1 * ny1 + c2;
                int s = start[cell], e = end[cell];
                if (s >= e) continue;
                cur[nc] = s; lim[nc] = e; cz[nc] = c3; cx[nc] = c1; cy[nc] = c2;
                nc++;
            }
    // float accumulators (the reference's per-thread float buffers) and double weights
    float aN = 0.f, aR = 0.f, aXX = 0.f, aXY = 0.f, aXZ = 0.f, aYZ = 0.f;
    double wN = 0, wR = 0, wXX = 0, wXY = 0, wXZ = 0, wYZ = 0;
    const double gxm = gx[m1], gym = gy[m2], gzm = gz[m3];
    for (;;) {
        int best = -1;
        unsigned bidx = 0xffffffffu;
        for (int q = 0; q < nc; q++)
            if (cur[q] < lim[q]) {
                unsigned v = idx[cur[q]];
                if (v < bidx) { bidx = v; best = q; }
            }
        if (best < 0) break;
        float4 m = mk[cur[best]];
        cur[best]++;
        int t = __float_as_int(m.w);
        int m10 = cx[best], m20 = cy[best], m30 = cz[best];
        double dx = __dsub_rn(gx[m10 + 1], gx[m10]);
        double dy = __dsub_rn(gy[m20 + 1], gy[m20]);
        double dz = __dsub_rn(gz[m30 + 1], gz[m30]);
        double ddz = __dsub_rn(1.0, fabs(__ddiv_rn(__dsub_rn(gzm, (double)m.z), dz)));
        double ddx = __dsub_rn(1.0, fabs(__ddiv_rn(__dsub_rn(gxm, (double)m.x), dx)));
        double ddy = __dsub_rn(1.0, fabs(__ddiv_rn(__dsub_rn(gym, (double)m.y), dy)));
        double swt = __dmul_rn(__dmul_rn(ddx, ddy), ddz);
        double f = rock_f[t];
        if (pl && pl[kPowerLawStride * t] != 0) {
            // power-law rock (viscalc, mark3mg.c:1489-1498): marknu * val1^((1-n)/n) clamped to
            // [markn0, markn1], then to [nubeg, nuend]
            const double *r = pl + kPowerLawStride * t;
            double mnu = __dmul_rn(r[1], pow(val1[bidx], r[2]));
            if (mnu < r[3]) mnu = r[3];
            if (mnu > r[4]) mnu = r[4];
            if (mnu < nubeg) mnu = nubeg;
            if (mnu > nuend) mnu = nuend;
            f = viscmod == 0 ? mnu : (viscmod == 1 ? log(mnu) : __ddiv_rn(1.0, mnu));
        }
        if (ddx > nukoef && ddy > nukoef && ddz > nukoef) {
            aN = __double2float_rn(__dadd_rn((double)aN, __dmul_rn(f, swt)));
            wN = __dadd_rn(wN, swt);
        }
        if (m1 > m10 && m2 > m20 && m3 > m30) {
            double s1 = __dmul_rn(__dmul_rn(__dmul_rn(8.0, __dsub_rn(0.5, fabs(__dsub_rn(ddx, 0.5)))),
                                            __dsub_rn(0.5, fabs(__dsub_rn(ddy, 0.5)))),
                                  __dsub_rn(0.5, fabs(__dsub_rn(ddz, 0.5))));
            aXX = __double2float_rn(__dadd_rn((double)aXX, __dmul_rn(f, s1)));
            wXX = __dadd_rn(wXX, s1);
        }
        if (m3 == m30 && ddx > 0.5 && ddy > 0.5) {
            double s1 = __dmul_rn(__dmul_rn(__dmul_rn(8.0, __dsub_rn(ddx, 0.5)), __dsub_rn(ddy, 0.5)),
                                  __dsub_rn(0.5, fabs(__dsub_rn(ddz, 0.5))));
            aXY = __double2float_rn(__dadd_rn((double)aXY, __dmul_rn(f, s1)));
            wXY = __dadd_rn(wXY, s1);
        }
        if (m2 == m20 && ddx > 0.5 && ddz > 0.5) {
            double s1 = __dmul_rn(__dmul_rn(__dmul_rn(8.0, __dsub_rn(ddx, 0.5)),
                                            __dsub_rn(0.5, fabs(__dsub_rn(ddy, 0.5)))),
                                  __dsub_rn(ddz, 0.5));
            aXZ = __double2float_rn(__dadd_rn((double)aXZ, __dmul_rn(f, s1)));
            wXZ = __dadd_rn(wXZ, s1);
        }
        if (m1 == m10 && ddy > 0.5 && ddz > 0.5) {
            double s1 = __dmul_rn(__dmul_rn(__dmul_rn(8.0, __dsub_rn(0.5, fabs(__dsub_rn(ddx, 0.5)))),
                                            __dsub_rn(ddy, 0.5)),
                                  __dsub_rn(ddz, 0.5));
            aYZ = __double2float_rn(__dadd_rn((double)aYZ, __dmul_rn(f, s1)));
            wYZ = __dadd_rn(wYZ, s1);
        }
        if (ddx > 0.5 && ddy > 0.5 && ddz > 0.5) {
            double s1 = __dmul_rn(__dmul_rn(__dmul_rn(8.0, __dsub_rn(ddx, 0.5)), __dsub_rn(ddy, 0.5)),
                                  __dsub_rn(ddz, 0.5));
            aR = __double2float_rn(__dadd_rn((double)aR, __dmul_rn(rock_ro[t], s1)));
            wR = __dadd_rn(wR, s1);
        }
    }
    // normalise (mark3mg.c:958-1014), keep old values where no marker contributed, clamp viscosities
    auto fin = [&](float a, double w, float old) -> float {
        if (!(w > 0)) return old;
        float v = __double2float_rn(__ddiv_rn((double)a, w));
        if (viscmod == 1) v = __double2float_rn(exp((double)v));
        if (viscmod == 2) v = __double2float_rn(__ddiv_rn(1.0, (double)v));
        return v;
    };
    auto clampf = [&](float v) -> float {
        if ((double)v < nubeg) v = __double2float_rn(nubeg);
        if ((double)v > nuend) v = __double2float_rn(nuend);
        return v;
    };
    nu[u] = clampf(fin(aN, wN, nu[u]));
    nxx[u] = clampf(fin(aXX, wXX, nxx[u]));
    nxy[u] = clampf(fin(aXY, wXY, nxy[u]));
    nxz[u] = clampf(fin(aXZ, wXZ, nxz[u]));
    nyz[u] = clampf(fin(aYZ, wYZ, nyz[u]));
    if (wR > 0) ro[u] = __double2float_rn(__ddiv_rn((double)aR, wR));
}

// gridlines in shared memory when they fit (kMoveShBytes), else read in place
// Strain rate at a point (epscalc1, mark3mg.c:3244-3642, non-periodic box):
// the normal components from the cell centres, exy / exz / eyz from their
// edges, each by trilinear weights with the reference's clamping per axis and
// accumulation order (z outer, x, y inner).  Three axis kinds:
//   centre  normal strain rates, stored at the cell's upper corner node;
//   line    the edge direction's nodes (clamped to [1, n-3]);
//   mid     an axis across the edge: between cell mid-points.
struct StrainF {
    const float *e[6];  // exx eyy ezz exy exz eyz, node layout
};

__device__ __forceinline__ void ax_centre(const double *g, int n, int cell, double x, int &lo, double &w0,
                                          double &w1)
{
    int m = cell;
    double X = x;
    if (X > dmid(g, m)) m += 1;
    if (m < 1) { m = 1; X = __dmul_rn(__dadd_rn(g[1], g[0]), 0.5); }
    if (m > n - 2) { m = n - 2; X = __dmul_rn(__dadd_rn(g[m], g[m + 1]), 0.5); }
    const double d = __dmul_rn(__dsub_rn(g[m + 1], g[m - 1]), 0.5);
    lo = m;
    w0 = __dsub_rn(1.0, -__ddiv_rn(__dsub_rn(__dmul_rn(__dadd_rn(g[m], g[m - 1]), 0.5), X), d));
    w1 = __dsub_rn(1.0, __ddiv_rn(__dsub_rn(__dmul_rn(__dadd_rn(g[m + 1], g[m]), 0.5), X), d));
}

__device__ __forceinline__ void ax_line(const double *g, int n, int cell, double x, int &lo, double &w0, double &w1)
{
    int m = cell;
    double X = x;
    if (m < 1) { m = 1; X = g[1]; }
    if (m > n - 3) { m = n - 3; X = g[m + 1]; }
    const double d = __dsub_rn(g[m + 1], g[m]);
    lo = m;
    w0 = __dsub_rn(1.0, -__ddiv_rn(__dsub_rn(g[m], X), d));
    w1 = __dsub_rn(1.0, __ddiv_rn(__dsub_rn(g[m + 1], X), d));
}

// as ax_mid, but the lower clamp also applies at m == 0 (mark3mg.c:3408, 3485, 3559)
__device__ __forceinline__ void ax_mid_eps(const double *g, int n, int cell, double x, int &lo, double &w0,
                                           double &w1)
{
    int m = cell;
    double X = x;
    if (X < dmid(g, m)) m -= 1;
    if (m < 1) { m = 0; X = dmid(g, 0); }
    if (m > n - 3) { m = n - 3; X = dmid(g, m + 1); }
    const double d = __dmul_rn(__dsub_rn(g[m + 2], g[m]), 0.5);
    lo = m;
    w0 = __dsub_rn(1.0, -__ddiv_rn(__dsub_rn(dmid(g, m), X), d));
    w1 = __dsub_rn(1.0, __ddiv_rn(__dsub_rn(dmid(g, m + 1), X), d));
}

// weighted sum over the 8 nodes, z outer, x, y inner
__device__ __forceinline__ double trilin(const float *f, const int lo[3], const double w[3][2], long nxy, int ny)
{
    double s = 0;
#pragma unroll
    for (int c = 0; c < 2; c++)
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++) {
                const long idx = (long)(lo[2] + c) * nxy + (long)(lo[0] + a) * ny + (lo[1] + b);
                s = __dadd_rn(s, __dmul_rn((double)__ldg(f + idx), __dmul_rn(__dmul_rn(w[0][a], w[1][b]), w[2][c])));
            }
    return s;
}

// second invariant sqrt(0.5 (exx^2 + eyy^2 + ezz^2) + exy^2 + exz^2 + eyz^2)
// of the strain rate at (x, y, z) (mark3mg.c:219, 361)
__device__ double strain_ii(const GridSh &G, const StrainF &S, double x, double y, double z)
{
    const double p[3] = {x < 0 ? 0.0 : (x > G.size[0] ? G.size[0] : x), y < 0 ? 0.0 : (y > G.size[1] ? G.size[1] : y),
                         z < 0 ? 0.0 : (z > G.size[2] ? G.size[2] : z)};
    int cell[3];
    for (int a = 0; a < 3; a++) cell[a] = serch(G.g[a], G.n[a], p[a]);
    const long nxy = (long)G.n[0] * G.n[1];
    const int ny = G.n[1];
    int loC[3], loL[3], loM[3];
    double wC[3][2], wL[3][2], wM[3][2];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        ax_centre(G.g[a], G.n[a], cell[a], p[a], loC[a], wC[a][0], wC[a][1]);
        ax_line(G.g[a], G.n[a], cell[a], p[a], loL[a], wL[a][0], wL[a][1]);
        ax_mid_eps(G.g[a], G.n[a], cell[a], p[a], loM[a], wM[a][0], wM[a][1]);
    }
    const double exx = trilin(S.e[0], loC, wC, nxy, ny), eyy = trilin(S.e[1], loC, wC, nxy, ny),
                 ezz = trilin(S.e[2], loC, wC, nxy, ny);
    // exy: x, y along the edge's nodes, z between mid-points; exz: x, z lines,
    // y mid; eyz: y, z lines, x mid
    int lo[3];
    double w[3][2];
    lo[0] = loL[0]; lo[1] = loL[1]; lo[2] = loM[2];
    w[0][0] = wL[0][0]; w[0][1] = wL[0][1]; w[1][0] = wL[1][0]; w[1][1] = wL[1][1]; w[2][0] = wM[2][0]; w[2][1] = wM[2][1];
    const double exy = trilin(S.e[3], lo, w, nxy, ny);
    lo[1] = loM[1]; lo[2] = loL[2];
    w[1][0] = wM[1][0]; w[1][1] = wM[1][1]; w[2][0] = wL[2][0]; w[2][1] = wL[2][1];
    const double exz = trilin(S.e[4], lo, w, nxy, ny);
    lo[0] = loM[0]; lo[1] = loL[1];
    w[0][0] = wM[0][0]; w[0][1] = wM[0][1]; w[1][0] = wL[1][0]; w[1][1] = wL[1][1];
    const double eyz = trilin(S.e[5], lo, w, nxy, ny);
    const double nn = __dadd_rn(__dadd_rn(__dmul_rn(exx, exx), __dmul_rn(eyy, eyy)), __dmul_rn(ezz, ezz));
    double q = __dmul_rn(0.5, nn);
    q = __dadd_rn(q, __dmul_rn(exy, exy));
    q = __dadd_rn(q, __dmul_rn(exz, exz));
    q = __dadd_rn(q, __dmul_rn(eyz, eyz));
    return __dsqrt_rn(q);
}

constexpr int kMoveThreads = 256;
constexpr int kMoveShBytes = 96 * 1024;

// kStrain: also val1 (strain-rate invariant at the marker before the move) and
// the brittle strain marke (RK4 of the invariant over the stages, for markers
// with marke > 0), as movemark does (mark3mg.c:218-220, 358-410, 488).
template <bool kStrain>
__global__ void __launch_bounds__(kMoveThreads, 3) k_movemark(long nmark, Grid3 G3, bool shared_grid, const float *vx,
                                                           const float *vy, const float *vz, float *mx, float *my,
                                                           float *mz, const signed char *mt, double dt, int markmod,
                                                           int outgrid, StrainF S, double *val1, float *marke)
{
    extern __shared__ double gsh[];
    GridSh G;
    if (shared_grid) {
        int off = 0;
        for (int a = 0; a < 3; a++) {
            for (int q = threadIdx.x; q < G3.n[a]; q += blockDim.x) gsh[off + q] = G3.g[a][q];
            G.g[a] = gsh + off;
            off += G3.n[a];
        }
        __syncthreads();
    } else {
        for (int a = 0; a < 3; a++) G.g[a] = G3.g[a];
    }
    for (int a = 0; a < 3; a++) { G.n[a] = G3.n[a]; G.size[a] = G3.size[a]; }
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nmark) return;
    const float fx = mx[q], fy = my[q], fz = mz[q];
    const int t = mt[q];
    const bool inside = fx >= 0 && fy >= 0 && fz >= 0 && (double)fx <= G.size[0] && (double)fy <= G.size[1] &&
                        (double)fz <= G.size[2];
    if (!(inside || (outgrid != 1 && (t < 50 || t >= 100)))) return;
    double v1[3], v2[3], v3[3], v4[3], v[3];
    double ee0 = 0;
    bool brittle = false;
    vxyz_at(G, vx, vy, vz, fx, fy, fz, v1);
    if constexpr (kStrain) {
        const double e1 = strain_ii(G, S, fx, fy, fz);
        val1[q] = e1;
        brittle = marke[q] > 0;
        ee0 = e1;  // the single-velocity branch keeps the marker's own rate
    }
    if (markmod == 1) {  // velocity at the marker (mark3mg.c:317-323)
        for (int a = 0; a < 3; a++) v[a] = v1[a];
    } else {
        // (v dt) / 2 of the reference is v dt rounded, then halved exactly
        double X[3];
        for (int a = 0; a < 3; a++) X[a] = __dadd_rn((double)(a == 0 ? fx : a == 1 ? fy : fz), __dmul_rn(__dmul_rn(v1[a], dt), 0.5));
        vxyz_at(G, vx, vy, vz, X[0], X[1], X[2], v2);
        double e2 = 0, e3 = 0, e4 = 0;
        if constexpr (kStrain) {
            if (brittle) e2 = strain_ii(G, S, X[0], X[1], X[2]);
        }
        for (int a = 0; a < 3; a++) X[a] = __dadd_rn((double)(a == 0 ? fx : a == 1 ? fy : fz), __dmul_rn(__dmul_rn(v2[a], dt), 0.5));
        vxyz_at(G, vx, vy, vz, X[0], X[1], X[2], v3);
        if constexpr (kStrain) {
            if (brittle) e3 = strain_ii(G, S, X[0], X[1], X[2]);
        }
        for (int a = 0; a < 3; a++) X[a] = __dadd_rn((double)(a == 0 ? fx : a == 1 ? fy : fz), __dmul_rn(v3[a], dt));
        vxyz_at(G, vx, vy, vz, X[0], X[1], X[2], v4);
        if constexpr (kStrain) {
            if (brittle) {
                e4 = strain_ii(G, S, X[0], X[1], X[2]);
                ee0 = __ddiv_rn(__dadd_rn(__dadd_rn(__dadd_rn(ee0, __dmul_rn(2.0, e2)), __dmul_rn(2.0, e3)), e4), 6.0);
            }
        }
        for (int a = 0; a < 3; a++)
            v[a] = __ddiv_rn(__dadd_rn(__dadd_rn(__dadd_rn(v1[a], __dmul_rn(2.0, v2[a])), __dmul_rn(2.0, v3[a])), v4[a]),
                             6.0);
    }
    if (outgrid == 2) {  // orthogonal motion only outside the box (mark3mg.c:437-459, non-periodic)
        if (fx < 0 || (double)fx > G.size[0]) v[1] = v[2] = 0;
        if (fy < 0 || (double)fy > G.size[1]) v[0] = v[2] = 0;
        if (fz < 0 || (double)fz > G.size[2]) v[0] = v[1] = 0;
    }
    mx[q] = __double2float_rn(__dadd_rn((double)fx, __dmul_rn(dt, v[0])));
    my[q] = __double2float_rn(__dadd_rn((double)fy, __dmul_rn(dt, v[1])));
    mz[q] = __double2float_rn(__dadd_rn((double)fz, __dmul_rn(dt, v[2])));
    if constexpr (kStrain) {
        // brittle strain of normal markers (mark3mg.c:488)
        if (brittle && t < 100) marke[q] = __fadd_rn(marke[q], __double2float_rn(__dmul_rn(ee0, dt)));
    }
}

static void launch_movemark(cudaStream_t st, long nmark, const Grid3 &G, const float *const vel[3], float *const pos[3],
                            const signed char *mt, double dt, int markmod, int outgrid, const StrainF *S = nullptr,
                            double *val1 = nullptr, float *marke = nullptr)
{
    const size_t bytes = sizeof(double) * ((size_t)G.n[0] + G.n[1] + G.n[2]);
    const bool sh = bytes <= (size_t)kMoveShBytes;
    const unsigned grid = nb(nmark, kMoveThreads);
    if (S) {
        if (sh && bytes > 48 * 1024)
            P2_CUDA_TRY(cudaFuncSetAttribute(k_movemark<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
        k_movemark<true><<<grid, kMoveThreads, sh ? bytes : 0, st>>>(nmark, G, sh, vel[0], vel[1], vel[2], pos[0],
                                                                     pos[1], pos[2], mt, dt, markmod, outgrid, *S,
                                                                     val1, marke); P2_COUNT_LAUNCH();
    } else {
        if (sh && bytes > 48 * 1024)
            P2_CUDA_TRY(cudaFuncSetAttribute(k_movemark<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
        k_movemark<false><<<grid, kMoveThreads, sh ? bytes : 0, st>>>(nmark, G, sh, vel[0], vel[1], vel[2], pos[0],
                                                                      pos[1], pos[2], mt, dt, markmod, outgrid,
                                                                      StrainF{}, nullptr, nullptr); P2_COUNT_LAUNCH();
    }
    P2_CUDA_TRY(cudaGetLastError());
}

// float velocities of the resident FP64 solution, zero at positions that are
// not unknowns (what p2_get_solution hands back)
__global__ void k_velocity_f32(int nx, int ny, int nz, const double *vx, const double *vy, const double *vz,
                               float *ox, float *oy, float *oz)
{
    long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= (long)nx * ny * nz) return;
    int j = (int)(u % ny), i = (int)((u / ny) % nx), k = (int)(u / ((long)nx * ny));
    ox[u] = valid_pos(1, i, j, k, nx, ny, nz) ? (float)vx[u] : 0.f;
    oy[u] = valid_pos(2, i, j, k, nx, ny, nz) ? (float)vy[u] : 0.f;
    oz[u] = valid_pos(3, i, j, k, nx, ny, nz) ? (float)vz[u] : 0.f;
}

Grid3 Solver::grid3() const
{
    const Level &L0 = L[0];
    Grid3 G;
    for (int a = 0; a < 3; a++) {
        G.g[a] = d_g[a];
        G.size[a] = L0.g[a].back() - L0.g[a].front();
    }
    G.n[0] = L0.nx; G.n[1] = L0.ny; G.n[2] = L0.nz;
    return G;
}

void Solver::ensure_move_buffers(long nmark)
{
    const Level &L0 = L[0];
    if (!d_g[0]) {
        for (int q = 0; q < 3; q++) {
            d_g[q] = (double *)grid_arena.alloc(sizeof(double) * L0.g[q].size());
            P2_CUDA_TRY(cudaMemcpy(d_g[q], L0.g[q].data(), sizeof(double) * L0.g[q].size(), cudaMemcpyHostToDevice));
        }
    }
    if (!mv_vel[0]) {
        for (int q = 0; q < 3; q++) mv_vel[q] = (float *)grid_arena.alloc(sizeof(float) * L0.n);
    }
    if (nmark > mv_cap) {
        move_arena.release();
        mv_val1 = nullptr;
        mv_marke = nullptr;
        mv_cap = std::max<long>(nmark, 1);
        for (int q = 0; q < 3; q++) mv_pos[q] = (float *)move_arena.alloc(sizeof(float) * mv_cap);
        mv_type = (signed char *)move_arena.alloc(mv_cap);
    }
}

// movemark() with its strain-rate outputs, on host arrays: velocities and the
// strain-rate fields exx..eyz (float, node layout, as vpiterate leaves them),
// markers in/out, val1 (double per marker) out, marke (float) in/out.
void Solver::movemark_strain_host(double dt, int markmod, int outgrid, const float *vx, const float *vy,
                                  const float *vz, const float *const e[6], long nmark, float *mx, float *my, float *mz,
                                  const signed char *mt, double *val1, float *marke)
{
    if (!grid_ready) throw Error(P2_ERR_STATE, "movemark before p2_set_grid");
    if (nmark < 0 || nmark > 0x7fffffffL) throw Error(P2_ERR_ARG, "marker count out of range");
    if (!(dt >= 0) || !std::isfinite(dt)) throw Error(P2_ERR_ARG, "time step must be finite and >= 0");
    if (outgrid < 0 || outgrid > 2) throw Error(P2_ERR_ARG, "outgrid must be 0, 1 or 2");
    if (markmod != 1 && markmod != 2) throw Error(P2_ERR_ARG, "markmod must be 1 (simple) or 2 (Runge-Kutta 4)");
    ensure_move_buffers(nmark);
    const Level &L0 = L[0];
    if (!mv_e[0])
        for (int q = 0; q < 6; q++) mv_e[q] = (float *)grid_arena.alloc(sizeof(float) * L0.n);
    if (!mv_val1) {
        mv_val1 = (double *)move_arena.alloc(sizeof(double) * mv_cap);
        mv_marke = (float *)move_arena.alloc(sizeof(float) * mv_cap);
    }
    const float *src[3] = {vx, vy, vz};
    for (int q = 0; q < 3; q++)
        P2_CUDA_TRY(cudaMemcpyAsync(mv_vel[q], src[q], sizeof(float) * L0.n, cudaMemcpyHostToDevice, st));
    for (int q = 0; q < 6; q++)
        P2_CUDA_TRY(cudaMemcpyAsync(mv_e[q], e[q], sizeof(float) * L0.n, cudaMemcpyHostToDevice, st));
    if (nmark > 0) {
        float *pos[3] = {mx, my, mz};
        for (int q = 0; q < 3; q++)
            P2_CUDA_TRY(cudaMemcpyAsync(mv_pos[q], pos[q], sizeof(float) * nmark, cudaMemcpyHostToDevice, st));
        P2_CUDA_TRY(cudaMemcpyAsync(mv_type, mt, nmark, cudaMemcpyHostToDevice, st));
        P2_CUDA_TRY(cudaMemcpyAsync(mv_val1, val1, sizeof(double) * nmark, cudaMemcpyHostToDevice, st));
        P2_CUDA_TRY(cudaMemcpyAsync(mv_marke, marke, sizeof(float) * nmark, cudaMemcpyHostToDevice, st));
        StrainF S;
        for (int q = 0; q < 6; q++) S.e[q] = mv_e[q];
        launch_movemark(st, nmark, grid3(), mv_vel, mv_pos, mv_type, dt, markmod, outgrid, &S, mv_val1, mv_marke);
        for (int q = 0; q < 3; q++)
            P2_CUDA_TRY(cudaMemcpyAsync(pos[q], mv_pos[q], sizeof(float) * nmark, cudaMemcpyDeviceToHost, st));
        P2_CUDA_TRY(cudaMemcpyAsync(val1, mv_val1, sizeof(double) * nmark, cudaMemcpyDeviceToHost, st));
        P2_CUDA_TRY(cudaMemcpyAsync(marke, mv_marke, sizeof(float) * nmark, cudaMemcpyDeviceToHost, st));
    }
    P2_CUDA_TRY(cudaStreamSynchronize(st));
}

// float copies of the resident solution velocities into mv_vel
void Solver::velocity_f32()
{
    const Level &L0 = L[0];
    k_velocity_f32<<<nb(L0.n), 256, 0, st>>>(L0.nx, L0.ny, L0.nz, gx.c[1], gx.c[2], gx.c[3], mv_vel[0],
                                             mv_vel[1], mv_vel[2]); P2_COUNT_LAUNCH();
}

// movemark() on host arrays: velocities vx, vy, vz (float, node layout) and
// markers in/out.
void Solver::movemark_host(double dt, int markmod, int outgrid, const float *vx, const float *vy, const float *vz, long nmark,
                           float *mx, float *my, float *mz, const signed char *mt)
{
    if (!grid_ready) throw Error(P2_ERR_STATE, "movemark before p2_set_grid");
    if (nmark < 0 || nmark > 0x7fffffffL) throw Error(P2_ERR_ARG, "marker count out of range");
    if (!(dt >= 0) || !std::isfinite(dt)) throw Error(P2_ERR_ARG, "time step must be finite and >= 0");
    if (outgrid < 0 || outgrid > 2) throw Error(P2_ERR_ARG, "outgrid must be 0, 1 or 2");
    if (markmod != 1 && markmod != 2) throw Error(P2_ERR_ARG, "markmod must be 1 (simple) or 2 (Runge-Kutta 4)");
    ensure_move_buffers(nmark);
    const Level &L0 = L[0];
    const float *src[3] = {vx, vy, vz};
    for (int q = 0; q < 3; q++)
        P2_CUDA_TRY(cudaMemcpyAsync(mv_vel[q], src[q], sizeof(float) * L0.n, cudaMemcpyHostToDevice, st));
    if (nmark > 0) {
        float *pos[3] = {mx, my, mz};
        for (int q = 0; q < 3; q++)
            P2_CUDA_TRY(cudaMemcpyAsync(mv_pos[q], pos[q], sizeof(float) * nmark, cudaMemcpyHostToDevice, st));
        P2_CUDA_TRY(cudaMemcpyAsync(mv_type, mt, nmark, cudaMemcpyHostToDevice, st));
        launch_movemark(st, nmark, grid3(), mv_vel, mv_pos, mv_type, dt, markmod, outgrid);
        for (int q = 0; q < 3; q++)
            P2_CUDA_TRY(cudaMemcpyAsync(pos[q], mv_pos[q], sizeof(float) * nmark, cudaMemcpyDeviceToHost, st));
    }
    P2_CUDA_TRY(cudaStreamSynchronize(st));
}

// movemark() on the resident markers with the resident solution.
void Solver::movemark_device(double dt, int markmod, int outgrid)
{
    if (!markers_ready) throw Error(P2_ERR_STATE, "movemark before markers were uploaded");
    if (!solution_ready) throw Error(P2_ERR_STATE, "movemark before a solve");
    if (!(dt >= 0) || !std::isfinite(dt)) throw Error(P2_ERR_ARG, "time step must be finite and >= 0");
    if (outgrid < 0 || outgrid > 2) throw Error(P2_ERR_ARG, "outgrid must be 0, 1 or 2");
    if (markmod != 1 && markmod != 2) throw Error(P2_ERR_ARG, "markmod must be 1 (simple) or 2 (Runge-Kutta 4)");
    ensure_move_buffers(0);
    velocity_f32();
    if (nmk > 0) {
        float *const pos[3] = {mk_x, mk_y, mk_z};
        launch_movemark(st, nmk, grid3(), mv_vel, pos, mk_t, dt, markmod, outgrid);
    }
    P2_CUDA_TRY(cudaGetLastError());
}

void Solver::get_markers(float *mx, float *my, float *mz)
{
    if (!markers_ready) throw Error(P2_ERR_STATE, "no resident markers");
    float *dst[3] = {mx, my, mz}, *src[3] = {mk_x, mk_y, mk_z};
    for (int q = 0; q < 3; q++)
        if (dst[q] && nmk > 0)
            P2_CUDA_TRY(cudaMemcpyAsync(dst[q], src[q], sizeof(float) * nmk, cudaMemcpyDeviceToHost, st));
    P2_CUDA_TRY(cudaStreamSynchronize(st));
}

// ---------------------------------------------------------------------------
void Solver::upload_markers(long nmark, const float *mx, const float *my, const float *mz, const signed char *mt,
                            int nrock, const double *n0, const double *n1, const double *rho, const double *marknu,
                            const double *markmm, const double *val1)
{
    if (!grid_ready) throw Error(P2_ERR_STATE, "markers before p2_set_grid");
    if (nmark < 0 || nmark > 0x7fffffffL) throw Error(P2_ERR_ARG, "marker count out of range");
    if (nrock <= 0 || nrock > 256) throw Error(P2_ERR_ARG, "rock table size out of range");
    const bool have_pl = marknu && markmm && (val1 || nmark == 0);
    // per-type viscosity (viscalc, mark3mg.c:1479-1482: types above 20 and
    // types with markn0 == markn1 are constant) and density (dencalc1, 1429);
    // power-law types (markn0 != markn1, type <= 20) need marknu, markmm and
    // every marker's strain-rate invariant val1
    std::vector<double> f(256, 1.0), r(256, 0.0), pl(kPowerLawStride * 256, 0.0);
    bool any_pl = false;
    for (int t = 0; t < nrock && t < 50; t++) {
        if (n0[t] != n1[t] && t <= 20) {
            if (!have_pl)
                throw Error(P2_ERR_UNSUPPORTED, "rock type " + std::to_string(t) +
                                                    " has a power-law viscosity (markn0 != markn1): use "
                                                    "p2_ronurecalc_powerlaw");
            if (!(markmm[t] != 0)) throw Error(P2_ERR_ARG, "markmm must be nonzero for power-law rock types");
            double *e = &pl[kPowerLawStride * t];
            e[0] = 1.0;
            e[1] = marknu[t];
            e[2] = (1 - markmm[t]) / markmm[t];
            e[3] = n0[t];
            e[4] = n1[t];
            any_pl = true;
        }
        double mnu = n0[t];
        if (mnu < prm.nubeg) mnu = prm.nubeg;
        if (mnu > prm.nuend) mnu = prm.nuend;
        f[t] = prm.viscmod == 0 ? mnu : (prm.viscmod == 1 ? std::log(mnu) : 1.0 / mnu);
        r[t] = rho[t];
    }
    // every marker with type < 50 must have a rock entry
    marker_arena.release();
    nmk = nmark;
    long cap = std::max<long>(nmark, 1);
    mk_x = (float *)marker_arena.alloc(sizeof(float) * cap);
    mk_y = (float *)marker_arena.alloc(sizeof(float) * cap);
    mk_z = (float *)marker_arena.alloc(sizeof(float) * cap);
    mk_t = (signed char *)marker_arena.alloc(cap);
    if (nmark) {
        P2_CUDA_TRY(cudaMemcpyAsync(mk_x, mx, sizeof(float) * nmark, cudaMemcpyHostToDevice, st));
        P2_CUDA_TRY(cudaMemcpyAsync(mk_y, my, sizeof(float) * nmark, cudaMemcpyHostToDevice, st));
        P2_CUDA_TRY(cudaMemcpyAsync(mk_z, mz, sizeof(float) * nmark, cudaMemcpyHostToDevice, st));
        P2_CUDA_TRY(cudaMemcpyAsync(mk_t, mt, nmark, cudaMemcpyHostToDevice, st));
    }
    for (long q = 0; q < nmark; q++)
        if (mt[q] < 50 && (mt[q] < 0 || mt[q] >= nrock)) throw Error(P2_ERR_ARG, "marker type without rock entry");
    rock_f = (double *)marker_arena.alloc(sizeof(double) * 256);
    rock_ro = (double *)marker_arena.alloc(sizeof(double) * 256);
    P2_CUDA_TRY(cudaMemcpy(rock_f, f.data(), sizeof(double) * 256, cudaMemcpyHostToDevice));
    P2_CUDA_TRY(cudaMemcpy(rock_ro, r.data(), sizeof(double) * 256, cudaMemcpyHostToDevice));
    rock_pl = nullptr;
    mk_val1 = nullptr;
    if (any_pl) {
        rock_pl = (double *)marker_arena.alloc(sizeof(double) * pl.size());
        P2_CUDA_TRY(cudaMemcpy(rock_pl, pl.data(), sizeof(double) * pl.size(), cudaMemcpyHostToDevice));
        mk_val1 = (double *)marker_arena.alloc(sizeof(double) * cap);
        if (nmark) P2_CUDA_TRY(cudaMemcpyAsync(mk_val1, val1, sizeof(double) * nmark, cudaMemcpyHostToDevice, st));
    }
    // sort and node buffers
    int ntiles = (int)((cap + kTile - 1) / kTile);
    mk_key[0] = (unsigned *)marker_arena.alloc(sizeof(unsigned) * cap);
    mk_key[1] = (unsigned *)marker_arena.alloc(sizeof(unsigned) * cap);
    mk_val[0] = (unsigned *)marker_arena.alloc(sizeof(unsigned) * cap);
    mk_val[1] = (unsigned *)marker_arena.alloc(sizeof(unsigned) * cap);
    mk_hist = (unsigned *)marker_arena.alloc(sizeof(unsigned) * (size_t)kBuckets * ntiles);
    mk_scan = (unsigned *)marker_arena.alloc(sizeof(unsigned) *
                                             (((size_t)kBuckets * ntiles + kScanChunk - 1) / kScanChunk));
    mk_sorted = (float4 *)marker_arena.alloc(sizeof(float4) * cap);
    const Level &L0 = L[0];
    long ncell = (long)(L0.nx - 1) * (L0.ny - 1) * (L0.nz - 1);
    cell_start = (int *)marker_arena.alloc(sizeof(int) * ncell);
    cell_end = (int *)marker_arena.alloc(sizeof(int) * ncell);
    d_g[0] = (double *)marker_arena.alloc(sizeof(double) * L0.nx);
    d_g[1] = (double *)marker_arena.alloc(sizeof(double) * L0.ny);
    d_g[2] = (double *)marker_arena.alloc(sizeof(double) * L0.nz);
    for (int q = 0; q < 3; q++)
        P2_CUDA_TRY(cudaMemcpy(d_g[q], L0.g[q].data(), sizeof(double) * L0.g[q].size(), cudaMemcpyHostToDevice));
    for (int q = 0; q < 6; q++) mk_nodes[q] = (float *)marker_arena.alloc(sizeof(float) * L0.n);
    markers_ready = true;
}

// Node fields in/out are mk_nodes[0..5] = nu, ro, nxx, nxy, nxz, nyz.
void Solver::ronurecalc_device()
{
    if (!markers_ready) throw Error(P2_ERR_STATE, "ronurecalc before markers were uploaded");
    const Level &L0 = L[0];
    long n = nmk;
    long ncell = (long)(L0.nx - 1) * (L0.ny - 1) * (L0.nz - 1);
    unsigned sentinel = (unsigned)ncell;
    int bits = 1;
    while ((1ul << bits) <= (unsigned long)sentinel) bits++;
    int passes = (bits + kRadixBits - 1) / kRadixBits;
    double xsize = L0.g[0].back() - L0.g[0].front(), ysize = L0.g[1].back() - L0.g[1].front(),
           zsize = L0.g[2].back() - L0.g[2].front();
    P2_CUDA_TRY(cudaMemsetAsync(cell_start, 0, sizeof(int) * ncell, st));
    P2_CUDA_TRY(cudaMemsetAsync(cell_end, 0, sizeof(int) * ncell, st));
    if (n > 0) {
        k_mark_keys<<<nb(n), 256, 0, st>>>(n, mk_x, mk_y, mk_z, mk_t, d_g[0], d_g[1], d_g[2], L0.nx, L0.ny, L0.nz,
                                           xsize, ysize, zsize, sentinel, mk_key[0], mk_val[0]); P2_COUNT_LAUNCH();
        int ntiles = (int)((n + kTile - 1) / kTile);
        int a = 0;
        for (int p = 0; p < passes; p++) {
            int shift = p * kRadixBits;
            k_radix_hist<<<ntiles, 256, 0, st>>>(n, mk_key[a], shift, mk_hist, ntiles); P2_COUNT_LAUNCH();
            const long hlen = (long)kBuckets * ntiles;
            const unsigned sblocks = (unsigned)((hlen + kScanChunk - 1) / kScanChunk);
            k_scan_local<<<sblocks, kScanThreads, 0, st>>>(mk_hist, hlen, mk_scan); P2_COUNT_LAUNCH();
            k_radix_scan<<<1, 1024, 0, st>>>(mk_scan, (long)sblocks); P2_COUNT_LAUNCH();
            k_scan_add<<<sblocks, kScanThreads, 0, st>>>(mk_hist, hlen, mk_scan); P2_COUNT_LAUNCH();
            k_radix_scatter<<<ntiles, 256, 0, st>>>(n, mk_key[a], mk_val[a], mk_key[1 - a], mk_val[1 - a], shift,
                                                    mk_hist, ntiles); P2_COUNT_LAUNCH();
            a = 1 - a;
        }
        mk_cur = a;
        k_cell_bounds<<<nb(n), 256, 0, st>>>(n, mk_key[a], sentinel, cell_start, cell_end); P2_COUNT_LAUNCH();
        k_permute<<<nb(n), 256, 0, st>>>(n, mk_val[a], mk_x, mk_y, mk_z, mk_t, mk_sorted); P2_COUNT_LAUNCH();
    }
    k_node_gather<<<nb(L0.n, 128), 128, 0, st>>>(L0.nx, L0.ny, L0.nz, d_g[0], d_g[1], d_g[2], cell_start, cell_end,
                                            mk_val[mk_cur], mk_sorted, rock_f, rock_ro, prm.nukoef, prm.viscmod,
                                            prm.nubeg, prm.nuend, mk_nodes[0], mk_nodes[1], mk_nodes[2],
                                            mk_nodes[3], mk_nodes[4], mk_nodes[5], rock_pl, mk_val1); P2_COUNT_LAUNCH();
    P2_CUDA_TRY(cudaGetLastError());
    // the result becomes the solver's resident node fields
    if (bc_ready) {
        float *dst[6] = {L[0].nu, L[0].ro, f0.nxx, f0.nxy, f0.nxz, f0.nyz};
        for (int q = 0; q < 6; q++)
            P2_CUDA_TRY(cudaMemcpyAsync(dst[q], mk_nodes[q], sizeof(float) * L0.n, cudaMemcpyDeviceToDevice, st));
        nodes_ready = true;
    }
}

}  // namespace p2

// ---------------------------------------------------------------------------
// p2_ronurecalc_noalloc: the interpolation above for callers that must not
// allocate device memory (a host code whose device memory is all handed out
// by its own pool at start-up, or one that cannot afford the device-wide
// synchronisation cudaMalloc/cudaFree imply inside its time loop).  The sort
// keys, indices, histograms, permuted markers, cell ranges, gridlines and rock
// tables live in one file-scope device array of fixed size instead of a
// context's buffers; markers and node fields are the caller's device arrays.
// The kernels are the ones above, unchanged.
namespace p2na {

constexpr long kMaxMarkers = 1L << 18;  // 262144 markers
constexpr long kMaxCells = 1L << 17;    // 131072 cells, e.g. 50 x 50 x 52
constexpr int kMaxLines = 1024;         // gridlines per axis
constexpr int kMaxTiles = (int)((kMaxMarkers + p2::kTile - 1) / p2::kTile);
constexpr size_t up(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t kKeyBytes = up(sizeof(unsigned) * kMaxMarkers);
constexpr size_t kOffKeys = 0;  // key[0], key[1], idx[0], idx[1]
constexpr size_t kOffSorted = kOffKeys + 4 * kKeyBytes;
constexpr size_t kOffHist = kOffSorted + up(sizeof(float4) * kMaxMarkers);
constexpr size_t kOffCells = kOffHist + up(sizeof(unsigned) * p2::kBuckets * kMaxTiles);
constexpr size_t kCellBytes = up(sizeof(int) * kMaxCells);
constexpr size_t kOffLines = kOffCells + 2 * kCellBytes;
constexpr size_t kLineBytes = up(sizeof(double) * kMaxLines);
constexpr size_t kOffRocks = kOffLines + 3 * kLineBytes;
constexpr size_t kOffFlag = kOffRocks + 2 * up(sizeof(double) * 256);
constexpr size_t kBytes = kOffFlag + 256;  // 9531648 bytes (9.1 MiB)
constexpr int kMaxDevices = 64;

}  // namespace p2na

// Held by every GPU that loads this library, until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[p2na::kBytes];

namespace p2na {

static std::mutex g_mu;
static unsigned char *g_addr[kMaxDevices];  // device address of the array, per device

// markers the gather would read a rock entry for (type < 50) without one
__global__ void k_count_bad_types(long nmark, const signed char *mt, int nrock, unsigned *bad)
{
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nmark) return;
    int t = mt[q];
    if (t < 50 && (t < 0 || t >= nrock)) atomicAdd(bad, 1u);
}

static p2_status fail(char *err, long errlen, p2_status code, const char *fmt, ...)
{
    if (err && errlen > 0) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(err, (size_t)errlen, fmt, ap);
        va_end(ap);
    }
    return code;
}

// device (or managed) memory that the current device `dev` can use: a device
// array of another GPU is refused (its kernels would read peer memory)
static bool on_device(const void *p, int dev)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

static bool increasing(const double *g, int n)
{
    for (int i = 1; i < n; i++)
        if (!(g[i] > g[i - 1])) return false;
    return true;
}

}  // namespace p2na

extern "C" p2_status p2_ronurecalc_noalloc(int nx, int ny, int nz, const double *gx, const double *gy,
                                           const double *gz, const p2_params *prm, int nrock, const double *markn0,
                                           const double *markn1, const double *markro, long nmark,
                                           const float *markx, const float *marky, const float *markz,
                                           const signed char *markt, float *nu, float *ro, float *nxx, float *nxy,
                                           float *nxz, float *nyz, void *stream, char *err, long errlen)
{
    using namespace p2na;
    using p2::nb;
    if (err && errlen > 0) err[0] = 0;
    if (!prm || !gx || !gy || !gz || !markn0 || !markn1 || !markro)
        return fail(err, errlen, P2_ERR_ARG, "null parameter, gridline or rock-table pointer");
    if (nx < 2 || ny < 2 || nz < 2 || nx > kMaxLines || ny > kMaxLines || nz > kMaxLines)
        return fail(err, errlen, P2_ERR_ARG, "grid %d x %d x %d: each axis needs 2..%d gridlines", nx, ny, nz,
                    kMaxLines);
    long ncell = (long)(nx - 1) * (ny - 1) * (nz - 1);
    if (ncell > kMaxCells)
        return fail(err, errlen, P2_ERR_ARG, "%ld cells exceed the maximum of %ld for the static scratch", ncell,
                    kMaxCells);
    if (nmark < 0 || nmark > kMaxMarkers)
        return fail(err, errlen, P2_ERR_ARG, "%ld markers: the static scratch holds 0..%ld", nmark, kMaxMarkers);
    if (!increasing(gx, nx) || !increasing(gy, ny) || !increasing(gz, nz))
        return fail(err, errlen, P2_ERR_ARG, "gridlines must be strictly increasing");
    if (prm->viscmod < 0 || prm->viscmod > 2) return fail(err, errlen, P2_ERR_ARG, "viscmod must be 0, 1 or 2");
    if (nrock <= 0 || nrock > 256) return fail(err, errlen, P2_ERR_ARG, "rock table size %d out of 1..256", nrock);
    // rock tables as in upload_markers: constant per-type viscosity (mark3mg.c:1481-1482) and density (1429)
    double f[256], r[256];
    for (int t = 0; t < 256; t++) { f[t] = 1.0; r[t] = 0.0; }
    for (int t = 0; t < nrock && t < 50; t++) {
        // only types up to 20 take the power law (mark3mg.c:1481-1498); above
        // that markn0 is the viscosity whatever markn1 holds
        if (markn0[t] != markn1[t] && t <= 20)
            return fail(err, errlen, P2_ERR_UNSUPPORTED, "rock type %d has a power-law viscosity (markn0 != markn1)",
                        t);
        double mnu = markn0[t];
        if (mnu < prm->nubeg) mnu = prm->nubeg;
        if (mnu > prm->nuend) mnu = prm->nuend;
        f[t] = prm->viscmod == 0 ? mnu : (prm->viscmod == 1 ? std::log(mnu) : 1.0 / mnu);
        r[t] = markro[t];
    }
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return fail(err, errlen, P2_ERR_CUDA, "no usable current CUDA device");
    }
    float *outs[6] = {nu, ro, nxx, nxy, nxz, nyz};
    for (int q = 0; q < 6; q++)
        if (!outs[q] || !on_device(outs[q], dev))
            return fail(err, errlen, P2_ERR_ARG, "node field %d is not a device array of the current device", q);
    if (nmark > 0 && (!markx || !marky || !markz || !markt || !on_device(markx, dev) || !on_device(marky, dev) ||
                      !on_device(markz, dev) || !on_device(markt, dev)))
        return fail(err, errlen, P2_ERR_ARG, "marker arrays must be device arrays of the current device");
    // the array's host-side name is not a device address: look the address up once per device
    unsigned char *base;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        // a cudaDeviceReset unloads the module: an address cached before it is
        // looked up again when it no longer names device memory of this device
        if (g_addr[dev] && !on_device(g_addr[dev], dev)) g_addr[dev] = nullptr;
        if (!g_addr[dev]) {
            cudaError_t e = cudaGetSymbolAddress((void **)&g_addr[dev], g_noalloc_scratch);
            if (e != cudaSuccess) {
                g_addr[dev] = nullptr;
                cudaGetLastError();
                return fail(err, errlen, P2_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
            }
        }
        base = g_addr[dev];
    }
    unsigned *key[2] = {(unsigned *)(base + kOffKeys), (unsigned *)(base + kOffKeys + kKeyBytes)};
    unsigned *val[2] = {(unsigned *)(base + kOffKeys + 2 * kKeyBytes), (unsigned *)(base + kOffKeys + 3 * kKeyBytes)};
    float4 *sorted = (float4 *)(base + kOffSorted);
    unsigned *hist = (unsigned *)(base + kOffHist);
    int *cstart = (int *)(base + kOffCells), *cend = (int *)(base + kOffCells + kCellBytes);
    double *dg[3] = {(double *)(base + kOffLines), (double *)(base + kOffLines + kLineBytes),
                     (double *)(base + kOffLines + 2 * kLineBytes)};
    double *rf = (double *)(base + kOffRocks), *rr = (double *)(base + kOffRocks + up(sizeof(double) * 256));
    unsigned *bad = (unsigned *)(base + kOffFlag);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
#define P2NA_TRY(expr)                                                                                     \
    do {                                                                                                   \
        if ((e = (expr)) != cudaSuccess) {                                                                 \
            cudaGetLastError();                                                                            \
            return fail(err, errlen, P2_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e));                 \
        }                                                                                                  \
    } while (0)
    P2NA_TRY(cudaMemcpyAsync(dg[0], gx, sizeof(double) * nx, cudaMemcpyHostToDevice, s));
    P2NA_TRY(cudaMemcpyAsync(dg[1], gy, sizeof(double) * ny, cudaMemcpyHostToDevice, s));
    P2NA_TRY(cudaMemcpyAsync(dg[2], gz, sizeof(double) * nz, cudaMemcpyHostToDevice, s));
    P2NA_TRY(cudaMemcpyAsync(rf, f, sizeof(f), cudaMemcpyHostToDevice, s));
    P2NA_TRY(cudaMemcpyAsync(rr, r, sizeof(r), cudaMemcpyHostToDevice, s));
    // the array keeps the previous call's contents: the cell ranges and the bad-type count start at zero
    P2NA_TRY(cudaMemsetAsync(cstart, 0, sizeof(int) * ncell, s));
    P2NA_TRY(cudaMemsetAsync(cend, 0, sizeof(int) * ncell, s));
    P2NA_TRY(cudaMemsetAsync(bad, 0, sizeof(unsigned), s));
    int cur = 0;
    if (nmark > 0) {
        p2na::k_count_bad_types<<<nb(nmark), 256, 0, s>>>(nmark, markt, nrock, bad);
        P2NA_TRY(cudaGetLastError());
        unsigned nbad = 0;
        P2NA_TRY(cudaMemcpyAsync(&nbad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        P2NA_TRY(cudaStreamSynchronize(s));
        if (nbad)
            return fail(err, errlen, P2_ERR_ARG, "%u markers have a type below 50 without a rock entry", nbad);
        unsigned sentinel = (unsigned)ncell;
        int bits = 1;
        while ((1ul << bits) <= (unsigned long)sentinel) bits++;
        int passes = (bits + p2::kRadixBits - 1) / p2::kRadixBits;
        double xsize = gx[nx - 1] - gx[0], ysize = gy[ny - 1] - gy[0], zsize = gz[nz - 1] - gz[0];
        p2::k_mark_keys<<<nb(nmark), 256, 0, s>>>(nmark, markx, marky, markz, markt, dg[0], dg[1], dg[2], nx, ny,
                                                  nz, xsize, ysize, zsize, sentinel, key[0], val[0]);
        int ntiles = (int)((nmark + p2::kTile - 1) / p2::kTile);
        for (int p = 0; p < passes; p++) {
            int shift = p * p2::kRadixBits;
            p2::k_radix_hist<<<ntiles, 256, 0, s>>>(nmark, key[cur], shift, hist, ntiles);
            p2::k_radix_scan<<<1, 1024, 0, s>>>(hist, (long)p2::kBuckets * ntiles);
            p2::k_radix_scatter<<<ntiles, 256, 0, s>>>(nmark, key[cur], val[cur], key[1 - cur], val[1 - cur], shift,
                                                       hist, ntiles);
            cur = 1 - cur;
        }
        p2::k_cell_bounds<<<nb(nmark), 256, 0, s>>>(nmark, key[cur], sentinel, cstart, cend);
        p2::k_permute<<<nb(nmark), 256, 0, s>>>(nmark, val[cur], markx, marky, markz, markt, sorted);
    }
    p2::k_node_gather<<<nb((long)nx * ny * nz, 128), 128, 0, s>>>(nx, ny, nz, dg[0], dg[1], dg[2], cstart, cend,
                                                                  val[cur], sorted, rf, rr, prm->nukoef,
                                                                  prm->viscmod, prm->nubeg, prm->nuend, nu, ro, nxx,
                                                                  nxy, nxz, nyz);
    P2NA_TRY(cudaGetLastError());
#undef P2NA_TRY
    return P2_OK;
}
