// Host side of the p2cuda Stokes multigrid: level set-up, boundary tables,
// transfer tables, the V-cycle (FP32 or FP64) and the FP64 outer loop.
//
// Solve structure (move3mgNew.c:1791 vpiterate is the reference entry point):
//   outer FP64 GCR on the level-0 system, each iteration: true residual
//   r = b - A x in FP64, z = V(r) one V-cycle (FP32 in mixed mode), q = A z,
//   Gram-Schmidt against the previous directions, x += alpha z.
//   V-cycle: on levels 0..L-1 cell-block smoothing + residual + restriction
//   (vprestrict), dense inverse on the coarsest level (replaces PARDISO),
//   prolongation (vpprolong) + smoothing back up.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "p2_kernels.cuh"
#include "p2_solver.h"
#include "p2_sweep.cuh"
#include "p2_zmarch.cuh"
#include "p2_coarse.cuh"

namespace p2 {

constexpr int kProbes = 4 * 125;  // coarsest-operator probes: 125 colour classes x 4 components
int band_lu_inverse(cudaStream_t st, double *A, int n, int kl, int ku, double *Ainv, int *d_ipiv, int *d_info,
                    cudaEvent_t *marks, LuGraph *cache, bool wait = true);
// sweeps of the diagonal cell smoother on the coarsest level standing in for
// its direct solve while the LU is still running
constexpr int kCoarseApxSweeps = 16;
// cell planes per block of the fused sweep (each block starts 3 planes early)
constexpr int kSweepChunk = 32;
// Outer iterations that use the smoothed coarsest level: kOverlapScale *
// nF / n0, the LU's latency-bound panel chain (about linear in nF) over the
// fine work of one iteration (linear in n0), fixed from the grid sizes so
// that the iterates do not depend on timing (10 at 65^3, 2 at 129^3, 0 at
// 257^3 with nF = 6912); none on grids of fewer than four levels, where the
// coarsest level is too large a part of the problem for smoothing to stand
// in for it.  The solve waits for the LU at that iteration if it is still
// running.
constexpr double kOverlapScale = 400.0;
constexpr int kOverlapMax = 16;
void d2f(cudaStream_t st, size_t n, const double *a, float *b);

static inline unsigned nblk(long n, int t = kThreads) { return (unsigned)((n + t - 1) / t); }

// Launch with programmatic stream serialization (see pdl_enter): kernels
// launched this way start with pdl_enter().
template <typename... KArgs, typename... Args>
static void pdl_launch(cudaStream_t st, dim3 grid, dim3 block, void (*kern)(KArgs...), Args &&...args)
{
#ifdef P2_NO_PDL
    kern<<<grid, block, 0, st>>>(std::forward<Args>(args)...);
#else
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    P2_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...));
#endif
    P2_COUNT_LAUNCH();
}

void *DeviceArena::alloc(size_t bytes)
{
    void *p = nullptr;
    if (bytes == 0) bytes = 16;
    bytes += guard;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(P2_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
    }
    ptrs.push_back(p);
    // Zero-fill on the legacy stream and wait for it: the library's own
    // streams are non-blocking, so without the wait a fill still in flight
    // could land after a copy that the caller queues on its stream.
    P2_CUDA_TRY(cudaMemsetAsync(p, 0, bytes, 0));
    P2_CUDA_TRY(cudaStreamSynchronize(0));
    return p;
}
void DeviceArena::release()
{
    for (void *p : ptrs) cudaFree(p);
    ptrs.clear();
}

// ---------------------------------------------------------------------------
// Transfer tables along one axis (oracle p2oracle.c axis_node/axis_mid/
// axis_cell; reference move3mgNew.c:3562-3575 and the Vy/Vz/P blocks).
static int cmin_common(int m, int nf, int nc)
{
    int r = (m - 2) / 2 + 2;
    if (m < 3) r = m;
    if (m > nf - 4) r = nc - (nf - m);
    return r;
}

static void axis_table(const std::vector<double> &gf, const std::vector<double> &gc, int type, HostAxis &t)
{
    int nf = (int)gf.size(), nc = (int)gc.size();
    t.lo.assign(nf, 0);
    t.w0.assign(nf, 0.0);
    t.w1.assign(nf, 0.0);
    int m0 = 0, m1 = nf;
    if (type == 1) m1 = nf - 1;   // mid-located: 0..nf-2
    if (type == 2) m0 = 1;        // pressure cell: 1..nf-1
    std::vector<std::vector<std::pair<int, double>>> inv(nc);
    for (int m = m0; m < m1; m++) {
        int lo = cmin_common(m, nf, nc);
        double w0, w1;
        if (type == 0) {
            if (lo > nc - 2) lo = nc - 2;
            double d = gc[lo + 1] - gc[lo];
            w0 = 1.0 + (gc[lo] - gf[m]) / d;
            w1 = 1.0 - (gc[lo + 1] - gf[m]) / d;
        } else if (type == 1) {
            if (lo > nc - 3) lo = nc - 3;
            if ((gf[m] + gf[m + 1]) / 2.0 < (gc[lo] + gc[lo + 1]) / 2.0 && lo > 0) lo -= 1;
            double d = (gc[lo + 2] - gc[lo]) / 2.0, xf = gf[m] + gf[m + 1];
            w0 = 1.0 + (gc[lo] + gc[lo + 1] - xf) / 2.0 / d;
            w1 = 1.0 - (gc[lo + 1] + gc[lo + 2] - xf) / 2.0 / d;
        } else {
            if (lo > nc - 2) lo = nc - 2;
            if ((gf[m] + gf[m - 1]) / 2.0 < (gc[lo] + gc[lo - 1]) / 2.0 && lo > 1) lo -= 1;
            double d = (gc[lo + 1] - gc[lo - 1]) / 2.0, xf = gf[m] + gf[m - 1];
            w0 = 1.0 + (gc[lo] + gc[lo - 1] - xf) / 2.0 / d;
            w1 = 1.0 - (gc[lo + 1] + gc[lo] - xf) / 2.0 / d;
        }
        t.lo[m] = lo;
        t.w0[m] = w0;
        t.w1[m] = w1;
        inv[lo].push_back({m, w0});
        inv[lo + 1].push_back({m, w1});
    }
    t.ptr.assign(nc + 1, 0);
    t.idx.clear();
    t.w.clear();
    for (int I = 0; I < nc; I++) {
        for (auto &pr : inv[I]) { t.idx.push_back(pr.first); t.w.push_back(pr.second); }
        t.ptr[I + 1] = (int)t.idx.size();
    }
}

// ronurestrict weights 1 - |x_c - x_f| / dx (move3mgNew.c:3442-3484)
static void axis_table_ronu(const std::vector<double> &gf, const std::vector<double> &gc, HostAxis &t)
{
    int nf = (int)gf.size(), nc = (int)gc.size();
    std::vector<std::vector<std::pair<int, double>>> inv(nc);
    t.lo.assign(nf, 0);
    t.w0.assign(nf, 0.0);
    t.w1.assign(nf, 0.0);
    for (int m = 0; m < nf; m++) {
        int lo = cmin_common(m, nf, nc);
        if (lo > nc - 2) lo = nc - 2;
        double d = gc[lo + 1] - gc[lo];
        double w0 = 1.0 - std::fabs((gc[lo] - gf[m]) / d);
        double w1 = 1.0 - std::fabs((gc[lo + 1] - gf[m]) / d);
        t.lo[m] = lo;
        t.w0[m] = w0;
        t.w1[m] = w1;
        inv[lo].push_back({m, w0});
        inv[lo + 1].push_back({m, w1});
    }
    t.ptr.assign(nc + 1, 0);
    t.idx.clear();
    t.w.clear();
    for (int I = 0; I < nc; I++) {
        for (auto &pr : inv[I]) { t.idx.push_back(pr.first); t.w.push_back(pr.second); }
        t.ptr[I + 1] = (int)t.idx.size();
    }
}

template <typename V>
static V *upload(DeviceArena &A, const std::vector<V> &h)
{
    V *d = (V *)A.alloc(sizeof(V) * std::max<size_t>(h.size(), 1));
    if (!h.empty()) P2_CUDA_TRY(cudaMemcpy(d, h.data(), sizeof(V) * h.size(), cudaMemcpyHostToDevice));
    return d;
}

static AxisMap upload_axis(DeviceArena &A, const HostAxis &h, bool restriction = false)
{
    for (size_t I = 0; restriction && I + 1 < h.ptr.size(); I++)
        if (h.ptr[I + 1] - h.ptr[I] > kRestrictList)
            throw Error(P2_ERR_UNSUPPORTED, "restriction list longer than " + std::to_string(kRestrictList) +
                                                " fine nodes (grid coarsening not by factors of about 2)");
    AxisMap m;
    m.lo = upload(A, h.lo);
    m.w0 = upload(A, h.w0);
    m.w1 = upload(A, h.w1);
    m.ptr = upload(A, h.ptr);
    m.idx = upload(A, h.idx);
    m.w = upload(A, h.w);
    return m;
}

// ---------------------------------------------------------------------------
Solver::Solver(int device) : dev(device)
{
    P2_CUDA_TRY(cudaSetDevice(dev));
    P2_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    {
        // the coarsest LU's panel chain is latency-bound: its kernels go first
        // when they share the device with the V-cycles
        int lo = 0, hi = 0;
        P2_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        P2_CUDA_TRY(cudaStreamCreateWithPriority(&st_lu, cudaStreamNonBlocking, hi));
    }
    P2_CUDA_TRY(cudaEventCreateWithFlags(&ev_lu, cudaEventDisableTiming));
    for (int i = 0; i < 8; i++) P2_CUDA_TRY(cudaEventCreate(&ev[i]));
}

Solver::~Solver()
{
    cudaSetDevice(dev);
    if (st_lu) cudaStreamSynchronize(st_lu);
    drop_graphs();
    if (lu_graph.exec) cudaGraphExecDestroy(lu_graph.exec);
    arena.release();
    grid_arena.release();
    marker_arena.release();
    move_arena.release();
    post_arena.release();
    heat_arena.release();
    heat_mk_arena.release();
    heat = HeatState{};
    for (int i = 0; i < 8; i++) cudaEventDestroy(ev[i]);
    for (auto e : vc_ev) cudaEventDestroy(e);
    if (ev_lu) cudaEventDestroy(ev_lu);
    if (st_lu) cudaStreamDestroy(st_lu);
    if (st) cudaStreamDestroy(st);
}

void Solver::drop_graphs()
{
    for (auto &g : graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
    }
    for (auto &g : graphs_apx) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
    }
}

template <typename T>
LevelView<T> Solver::view(int l, bool raw_clamp) const
{
    const Level &Lv = L[l];
    LevelView<T> v;
    v.nx = Lv.nx; v.ny = Lv.ny; v.nz = Lv.nz; v.n = Lv.n;
    const T *tab = (const T *)(std::is_same<T, double>::value ? (const void *)Lv.tabd : (const void *)Lv.tabf);
    int mx = Lv.tabstride;
    v.ax = Axis<T>{tab + 0 * mx, tab + 1 * mx, tab + 2 * mx, tab + 3 * mx};
    v.ay = Axis<T>{tab + 4 * mx, tab + 5 * mx, tab + 6 * mx, tab + 7 * mx};
    v.az = Axis<T>{tab + 8 * mx, tab + 9 * mx, tab + 10 * mx, tab + 11 * mx};
    if (raw_clamp) {
        v.ec = f0.nxx; v.exy = f0.nxy; v.exz = f0.nxz; v.eyz = f0.nyz;
        v.do_clamp = 1;
    } else {
        v.ec = Lv.ec; v.exy = Lv.exy; v.exz = Lv.exz; v.eyz = Lv.eyz;
        v.do_clamp = 0;
    }
    v.clamp_lo = prm.nubeg;
    v.clamp_hi = prm.nuend;
    v.bcm = Lv.bcm;
    v.pin = Lv.pin;
    return v;
}

void Solver::set_grid(long nx, long ny, long nz, const double *gx, const double *gy, const double *gz,
                      const p2_params &p)
{
    if (nx < 8 || ny < 8 || nz < 8) throw Error(P2_ERR_ARG, "grid too small (need >= 8 nodes per axis)");
    if ((double)nx * ny * nz * 4.0 > 2.0e9) throw Error(P2_ERR_ARG, "grid too large for 32-bit unknown indices");
    if (p.multinum < 0 || p.multinum + 1 > P2_MAX_LEVELS) throw Error(P2_ERR_ARG, "multinum out of range");
    if (p.p2koef != 0.0) throw Error(P2_ERR_UNSUPPORTED, "p2koef != 0 (grad-div term) is not supported");
    drop_graphs();
    arena.release();
    // The cell-block smoothers load the neighbour cells of every cell,
    // including the cell layer above the top one (its values are masked,
    // since the top faces are boundary rows): one plane past the end of a
    // level array.  Every level allocation carries a zero-filled plane of
    // the finest level (the largest) after its end, so those loads stay in
    // the allocation.
    arena.guard = sizeof(double) * ((size_t)nx * ny + ny + 2);
    grid_arena.release();
    marker_arena.release();  // markers and their buffers belong to the previous grid
    move_arena.release();
    post_arena.release();
    heat_arena.release();  // heat rows and fields belong to the previous grid
    heat_mk_arena.release();
    heat = HeatState{};
    for (int q = 0; q < 12; q++) post_out[q] = nullptr;
    post_partial = nullptr;
    post_range = nullptr;
    for (int q = 0; q < 17; q++) bulk_in[q] = nullptr;
    bulk_partial = bulk_out = nullptr;
    mv_cap = 0;
    for (int q = 0; q < 3; q++) { d_g[q] = nullptr; mv_vel[q] = nullptr; mv_pos[q] = nullptr; }
    for (int q = 0; q < 6; q++) mv_e[q] = nullptr;
    mv_val1 = nullptr;
    mv_marke = nullptr;
    for (int q = 0; q < 6; q++) mk_nodes[q] = nullptr;
    mv_type = nullptr;
    prm = p;
    bc_ready = nodes_ready = markers_ready = solution_ready = false;
    L.clear();
    int nl = p.multinum + 1;
    L.resize(nl);
    long off = 0;
    std::vector<double> g0[3] = {std::vector<double>(gx, gx + nx), std::vector<double>(gy, gy + ny),
                                 std::vector<double>(gz, gz + nz)};
    for (int q = 0; q < 3; q++)
        for (size_t i = 1; i < g0[q].size(); i++)
            if (!(g0[q][i] > g0[q][i - 1])) throw Error(P2_ERR_ARG, "gridlines must increase strictly");
    for (int l = 0; l < nl; l++) {
        Level &Lv = L[l];
        if (l == 0) { Lv.nx = (int)nx; Lv.ny = (int)ny; Lv.nz = (int)nz; }
        else {
            Lv.nx = (L[l - 1].nx - 5) / 2 + 5;
            Lv.ny = (L[l - 1].ny - 5) / 2 + 5;
            Lv.nz = (L[l - 1].nz - 5) / 2 + 5;
        }
        if (Lv.nx < 6 || Lv.ny < 6 || Lv.nz < 6) throw Error(P2_ERR_ARG, "too many levels for this grid");
        Lv.n = Lv.nx * Lv.ny * Lv.nz;
        Lv.off = off;
        off += Lv.n;
        int s = 1 << l;
        // gridcheck(): outer three lines copied, interior (n2-2)*2^l+2 (load3mg.c:2079-2194)
        for (int q = 0; q < 3; q++) {
            int n = q == 0 ? Lv.nx : q == 1 ? Lv.ny : Lv.nz;
            const std::vector<double> &g = g0[q];
            int nf = (int)g.size();
            std::vector<double> &o = Lv.g[q];
            o.assign(n, 0.0);
            o[0] = g[0]; o[1] = g[1]; o[2] = g[2];
            o[n - 1] = g[nf - 1]; o[n - 2] = g[nf - 2]; o[n - 3] = g[nf - 3];
            for (int n2 = 3; n2 < n - 3; n2++) o[n2] = g[(n2 - 2) * s + 2];
        }
        // spacing tables, 12 arrays of stride max(n)
        int mx = std::max(Lv.nx, std::max(Lv.ny, Lv.nz));
        Lv.tabstride = mx;
        std::vector<double> td(12 * mx, 0.0);
        for (int q = 0; q < 3; q++) {
            const std::vector<double> &g = Lv.g[q];
            int n = (int)g.size();
            double *ih = &td[(4 * q + 0) * mx], *ihc = &td[(4 * q + 1) * mx], *ihe = &td[(4 * q + 2) * mx],
                   *ihv = &td[(4 * q + 3) * mx];
            for (int i = 1; i < n; i++) ih[i] = 1.0 / (g[i] - g[i - 1]);
            for (int i = 1; i < n - 1; i++) { ihc[i] = 2.0 / (g[i + 1] - g[i - 1]); ihe[i] = 1.0 / (g[i + 1] - g[i - 1]); }
            for (int i = 0; i < n - 1; i++) ihv[i] = 1.0 / (g[i + 1] - g[i]);
        }
        std::vector<float> tf(td.begin(), td.end());
        Lv.tabd = upload(grid_arena, td);
        Lv.tabf = upload(grid_arena, tf);
    }
    total_nodes = off;
    // transfer tables between consecutive levels
    for (int l = 0; l + 1 < nl; l++) {
        Level &F = L[l], &Cl = L[l + 1];
        for (int q = 0; q < 3; q++) {
            for (int t = 0; t < 3; t++) {
                HostAxis h;
                axis_table(F.g[q], Cl.g[q], t, h);
                F.tv.m[q][t] = upload_axis(grid_arena, h, true);
            }
            HostAxis hr;
            axis_table_ronu(F.g[q], Cl.g[q], hr);
            F.ronu[q] = upload_axis(grid_arena, hr);
        }
    }
    grid_ready = true;
}

void Solver::set_bc(const int *bondm, long bondm_len, const float *bondv1, const int *bondn1, long bondnum)
{
    if (!grid_ready) throw Error(P2_ERR_STATE, "p2_set_bc before p2_set_grid");
    if (bondm_len < 4 * total_nodes) throw Error(P2_ERR_ARG, "bondm shorter than 4 * (sum of level nodes)");
    drop_graphs();
    arena.release();
    for (size_t l = 0; l < L.size(); l++) {
        Level &Lv = L[l];
        std::vector<uint8_t> m(Lv.n, 0);
        Lv.pin = -1;
        Lv.pinval = 0.0;
        int npin = 0, pin_node = -1;
        double pin_value = 0;
        // rows of this level: (unknown, const, koef, target unknown or -1)
        struct Row { int uc; float cst, k; int t; };
        std::vector<Row> rows;
        std::map<int, int> row_of;  // uc -> row index
        for (int u = 0; u < Lv.n; u++)
            for (int c = 0; c < 4; c++) {
                long gidx = (Lv.off + u) * 4 + c;
                int bi = bondm[gidx];
                if (!bi) continue;
                if (bi < 0 || bi > bondnum) throw Error(P2_ERR_ARG, "bondm entry out of range");
                int j = u % Lv.ny, i = (u / Lv.ny) % Lv.nx, k = u / (Lv.nx * Lv.ny);
                if (!valid_pos(c, i, j, k, Lv.nx, Lv.ny, Lv.nz)) continue;  // no equation there
                Row r;
                r.uc = u * 4 + c;
                r.cst = bondv1[2 * bi];
                r.k = bondv1[2 * bi + 1];
                r.t = -1;
                long tg = bondn1[bi];
                if (tg) {
                    tg -= 1;
                    long tn = tg / 4 - Lv.off;
                    if (tn < 0 || tn >= Lv.n) throw Error(P2_ERR_ARG, "boundary row couples across levels");
                    r.t = (int)(tn * 4 + tg % 4);
                } else if (c == 0) {
                    npin++;
                    pin_node = u;
                    pin_value = r.cst;
                }
                row_of[r.uc] = (int)rows.size();
                rows.push_back(r);
                m[u] |= (uint8_t)(1 << c);
            }
        if (npin == 1) {
            Lv.pin = pin_node;
            Lv.pinval = pin_value;
            m[pin_node] &= (uint8_t)~BC_P;
            rows.erase(rows.begin() + row_of[pin_node * 4]);
            row_of.clear();
            for (size_t q = 0; q < rows.size(); q++) row_of[rows[q].uc] = (int)q;
        }
        // every non-boundary velocity row must keep its stencil inside the grid
        for (int u = 0; u < Lv.n; u++) {
            int j = u % Lv.ny, i = (u / Lv.ny) % Lv.nx, k = u / (Lv.nx * Lv.ny);
            int nx = Lv.nx, ny = Lv.ny, nz = Lv.nz;
            bool okx = i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 3 && k >= 1 && k <= nz - 3;
            bool oky = i >= 1 && i <= nx - 3 && j >= 1 && j <= ny - 2 && k >= 1 && k <= nz - 3;
            bool okz = i >= 1 && i <= nx - 3 && j >= 1 && j <= ny - 3 && k >= 1 && k <= nz - 2;
            if (valid_pos(1, i, j, k, nx, ny, nz) && !(m[u] & BC_VX) && !okx)
                throw Error(P2_ERR_UNSUPPORTED, "open boundary row (Vx) on level " + std::to_string(l) +
                                                    ": periodic or missing boundary conditions are not supported");
            if (valid_pos(2, i, j, k, nx, ny, nz) && !(m[u] & BC_VY) && !oky)
                throw Error(P2_ERR_UNSUPPORTED, "open boundary row (Vy) on level " + std::to_string(l));
            if (valid_pos(3, i, j, k, nx, ny, nz) && !(m[u] & BC_VZ) && !okz)
                throw Error(P2_ERR_UNSUPPORTED, "open boundary row (Vz) on level " + std::to_string(l));
        }
        // chain depth: rows whose target is itself a boundary row run later
        std::vector<int> depth(rows.size(), 0);
        for (size_t q = 0; q < rows.size(); q++) {
            int d = 0, t = rows[q].t;
            while (t >= 0) {
                auto it = row_of.find(t);
                if (it == row_of.end()) break;
                if (++d > 16) throw Error(P2_ERR_ARG, "cyclic boundary-row chain");
                t = rows[it->second].t;
            }
            depth[q] = d;
        }
        std::vector<size_t> order(rows.size());
        for (size_t q = 0; q < order.size(); q++) order[q] = q;
        std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return depth[a] < depth[b]; });
        std::vector<int> bu, bt;
        std::vector<float> bk, bcst;
        Lv.bc_groups.clear();
        Lv.bc_groups.push_back(0);
        int cur = 0;
        for (size_t q : order) {
            while (depth[q] > cur) { Lv.bc_groups.push_back((int)bu.size()); cur++; }
            bu.push_back(rows[q].uc);
            bt.push_back(rows[q].t);
            bk.push_back(rows[q].k);
            bcst.push_back(rows[q].cst);
        }
        Lv.bc_groups.push_back((int)bu.size());
        Lv.nbc = (int)bu.size();
        // per row, the boundary row owning its target (-1: the target is a
        // regular unknown or none), so one launch can evaluate whole chains
        std::vector<int> bnext(bu.size(), -1);
        {
            std::map<int, int> pos;
            for (size_t q = 0; q < bu.size(); q++) pos[bu[q]] = (int)q;
            for (size_t q = 0; q < bu.size(); q++) {
                auto it = bt[q] >= 0 ? pos.find(bt[q]) : pos.end();
                if (it != pos.end()) bnext[q] = it->second;
            }
            for (size_t q = 0; q < bu.size(); q++) {
                int d = 0;
                for (int r = bnext[q]; r >= 0; r = bnext[r])
                    if (++d >= kMaxBcChain)
                        throw Error(P2_ERR_UNSUPPORTED, "boundary-row copy chain longer than " +
                                                            std::to_string(kMaxBcChain));
            }
        }
        // resolved chains (target non-boundary, product of koefs) for the coarse elimination
        Lv.h_bu = bu;
        Lv.h_rt.assign(bu.size(), -1);
        Lv.h_rk.assign(bu.size(), 0.0);
        for (size_t q = 0; q < bu.size(); q++) {
            int t = bt[q];
            double kk = bk[q];
            while (t >= 0) {
                auto it = row_of.find(t);
                if (it == row_of.end()) break;
                kk *= rows[it->second].k;
                t = rows[it->second].t;
            }
            Lv.h_rt[q] = t;
            Lv.h_rk[q] = t >= 0 ? kk : 0.0;
        }
        // fused sweeps: boundary rows by node, and whether every resolved
        // target lies within one node of its unknown
        {
            Lv.fuse_ok = true;
            for (size_t q = 0; q < bu.size() && Lv.fuse_ok; q++) {
                const int t = Lv.h_rt[q];
                if (t < 0) continue;
                const int u = bu[q] >> 2, v = t >> 2;
                const int du[3] = {u / (Lv.nx * Lv.ny), (u / Lv.ny) % Lv.nx, u % Lv.ny};
                const int dv[3] = {v / (Lv.nx * Lv.ny), (v / Lv.ny) % Lv.nx, v % Lv.ny};
                for (int a = 0; a < 3; a++)
                    if (std::abs(du[a] - dv[a]) > 1) Lv.fuse_ok = false;
            }
            std::vector<int> order(bu.size());
            for (size_t q = 0; q < order.size(); q++) order[q] = (int)q;
            std::sort(order.begin(), order.end(), [&](int a, int b2) { return bu[a] < bu[b2]; });
            std::vector<int> first(Lv.n, 0);
            for (size_t r = order.size(); r-- > 0;) first[bu[order[r]] >> 2] = (int)r;
            Lv.sw_first = upload(arena, first);
            if (order.empty()) order.push_back(0);
            Lv.sw_order = upload(arena, order);
        }
        Lv.h_bcm = m;
        Lv.bcm = upload(arena, m);
        Lv.bu = upload(arena, bu);
        Lv.bt = upload(arena, bt);
        Lv.bk = upload(arena, bk);
        Lv.bconst = upload(arena, bcst);
        Lv.bnext = upload(arena, bnext);
    }
    allocate_work();
    bc_ready = true;
}

void Solver::allocate_work()
{
    int nl = (int)L.size();
    for (int l = 0; l < nl; l++) {
        Level &Lv = L[l];
        long n = Lv.n;
        Lv.nu = (float *)arena.alloc(sizeof(float) * n);
        Lv.ro = (float *)arena.alloc(sizeof(float) * n);
        Lv.ec = (float *)arena.alloc(sizeof(float) * n);
        Lv.exy = (float *)arena.alloc(sizeof(float) * n);
        Lv.exz = (float *)arena.alloc(sizeof(float) * n);
        Lv.eyz = (float *)arena.alloc(sizeof(float) * n);
        auto v32 = [&](Vec4<float> &v) {
            float *p = (float *)arena.alloc(sizeof(float) * 4 * n);
            for (int c = 0; c < 4; c++) v.c[c] = p + c * n;
            v.n = (int)n;
        };
        auto v64 = [&](Vec4<double> &v) {
            double *p = (double *)arena.alloc(sizeof(double) * 4 * n);
            for (int c = 0; c < 4; c++) v.c[c] = p + c * n;
            v.n = (int)n;
        };
        v32(Lv.x32); v32(Lv.y32); v32(Lv.b32); v32(Lv.r32);
        {
            const long slots = (long)(Lv.nx - 1) * (Lv.nz - 1) * (Lv.ny / 2);
            Lv.blk_stride = (slots + 31) / 32 * 32;
            const size_t tsz = prm.precision == 0 ? sizeof(factor_t<float>) : sizeof(factor_t<double>);
            Lv.blk = arena.alloc(tsz * 2 * kBlkEntries * (size_t)Lv.blk_stride);
        }
        if (prm.precision == 1 || l == 0) {
            v64(Lv.x64); v64(Lv.y64); v64(Lv.r64);
            if (!(prm.precision == 1 && l == 0)) v64(Lv.b64);  // FP64 level 0: gr, set below
        }
        if (prm.precision == 1 && l > 0) {}
    }
    // level-0 raw fields
    long n0 = L[0].n;
    f0.nu = L[0].nu;
    f0.ro = L[0].ro;
    f0.nxx = (float *)arena.alloc(sizeof(float) * n0);
    f0.nxy = (float *)arena.alloc(sizeof(float) * n0);
    f0.nxz = (float *)arena.alloc(sizeof(float) * n0);
    f0.nyz = (float *)arena.alloc(sizeof(float) * n0);
    // outer loop vectors
    int m = std::max(1, std::min(prm.restart, kMaxDots - 2));
    restart = m;
    auto v64n = [&](Vec4<double> &v) {
        double *p = (double *)arena.alloc(sizeof(double) * 4 * n0);
        for (int c = 0; c < 4; c++) v.c[c] = p + c * n0;
        v.n = (int)n0;
    };
    v64n(gx); v64n(gb); v64n(gr);
    if (prm.precision == 1) L[0].b64 = gr;  // the FP64 cycle's level-0 right-hand side is the residual
    qq_dev = (double *)arena.alloc(sizeof(double) * m);
    Z.assign(m, Vec4<double>());
    Q.assign(m, Vec4<double>());
    for (int q = 0; q < m; q++) { v64n(Z[q]); v64n(Q[q]); }
    partial = (double *)arena.alloc(sizeof(double) * kRedBlocks * kMaxDots);
    {
        long maxc = 1;
        for (int l = 1; l < nl; l++) maxc = std::max<long>(maxc, L[l].n);
        rpartial = (double *)arena.alloc(sizeof(double) * nblk(4 * maxc));
        rticket = (unsigned *)arena.alloc(sizeof(unsigned) * 4);
        for (int l = 0; l < nl; l++) {
            Level &Lv = L[l];
            double vt = 0;
            for (int k = 1; k < Lv.nz; k++)
                for (int i = 1; i < Lv.nx; i++)
                    for (int j = 1; j < Lv.ny; j++) {
                        long u = (long)k * Lv.nx * Lv.ny + (long)i * Lv.ny + j;
                        if (Lv.h_bcm[u] & BC_P) continue;
                        vt += (Lv.g[0][i] - Lv.g[0][i - 1]) * (Lv.g[1][j] - Lv.g[1][j - 1]) *
                              (Lv.g[2][k] - Lv.g[2][k - 1]);
                    }
            Lv.compat_vol = vt;
        }
    }
    dots = (double *)arena.alloc(sizeof(double) * kMaxDots * 2);
    scal = (double *)arena.alloc(sizeof(double) * 64);  // [0,1] compat sums, [2] alpha, [3] shift, [8..] GS coefficients
    P2_CUDA_TRY(cudaMallocHost(&hdots_raw, sizeof(double) * kMaxDots * 2));
    hdots.reset(hdots_raw, [](double *p) { cudaFreeHost(p); });
    // coarse free-unknown set
    build_coarse_index();
}

void Solver::build_coarse_index()
{
    Level &C = L.back();
    std::vector<int> col(C.n * 4, -1);
    std::vector<int> fre;
    for (int u = 0; u < C.n; u++) {
        int j = u % C.ny, i = (u / C.ny) % C.nx, k = u / (C.nx * C.ny);
        for (int c = 0; c < 4; c++) {
            if (!valid_pos(c, i, j, k, C.nx, C.ny, C.nz)) continue;
            if (C.h_bcm[u] & (1 << c)) continue;
            if (c == 0 && u == C.pin) continue;  // pinned: fixed zero in the coarse correction
            col[u * 4 + c] = (int)fre.size();
            fre.push_back(u * 4 + c);
        }
    }
    nF = (int)fre.size();
    coarse_col = col;
    d_free = upload(arena, fre);
    d_colmap = upload(arena, col);
    // resolved boundary rows of the coarsest level as a dense per-unknown map
    std::vector<int> rt(C.n * 4, -2);
    std::vector<float> rk(C.n * 4, 0.0f);
    for (size_t q = 0; q < C.h_bu.size(); q++) {
        rt[C.h_bu[q]] = C.h_rt[q];
        rk[C.h_bu[q]] = (float)C.h_rk[q];
    }
    d_crt = upload(arena, rt);
    d_crk = upload(arena, rk);
    A_c = (double *)arena.alloc(sizeof(double) * (size_t)nF * nF);
    Ainv64 = (double *)arena.alloc(sizeof(double) * (size_t)nF * nF);
    Ainv32 = (float *)arena.alloc(sizeof(float) * (size_t)nF * nF);
    d_ipiv = (int *)arena.alloc(sizeof(int) * nF);
    d_info = (int *)arena.alloc(sizeof(int) * 4);
    probes = (double *)arena.alloc(sizeof(double) * (size_t)C.n * 4 * kProbes);
    d_bw = (int *)arena.alloc(sizeof(int) * 2);
    if (!h_bw) {
        int *p = nullptr;
        P2_CUDA_TRY(cudaMallocHost(&p, sizeof(int) * 2));
        h_bw_keep.reset(p, [](int *q) { cudaFreeHost(q); });
        h_bw = p;
    }
    cb64 = (double *)arena.alloc(sizeof(double) * nF);
    cx64 = (double *)arena.alloc(sizeof(double) * nF);
    cb32 = (float *)arena.alloc(sizeof(float) * nF);
    cx32 = (float *)arena.alloc(sizeof(float) * nF);
}

// ---------------------------------------------------------------------------
// Coarsest operator by probing: 125 colour classes (index mod 5 per axis) x 4
// components; a probe sets 1 on the free unknowns of its class and koef on the
// boundary unknowns whose resolved target is in the class, so that every
// non-zero of a row is attributed to the unique free column of that class
// within two nodes.  All kProbes probes are built and applied in one launch
// each (blockIdx.y = probe); the row kernel also records the band of the
// operator in the free-unknown ordering (bw[0] = max row - col, bw[1] = max
// col - row over the non-zeros).

__global__ void k_probe_build(int nx, int ny, int nz, const int *colmap, const int *rt, const float *rk,
                              double *probes)
{
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    int n = nx * ny * nz;
    if (u >= n) return;
    const int cls = blockIdx.y % 125, comp = blockIdx.y / 125;
    double *X = probes + (size_t)blockIdx.y * 4 * n;
    int j = u % ny, i = (u / ny) % nx, k = u / (nx * ny);
    int cx = cls % 5, cy = (cls / 5) % 5, cz = cls / 25;
    for (int c = 0; c < 4; c++) {
        double v = 0;
        int uc = u * 4 + c;
        if (colmap[uc] >= 0) {
            if (c == comp && i % 5 == cx && j % 5 == cy && k % 5 == cz) v = 1.0;
        } else if (rt[uc] >= 0) {
            int t = rt[uc], tn = t >> 2, tc = t & 3;
            int tj = tn % ny, ti = (tn / ny) % nx, tk = tn / (nx * ny);
            if (tc == comp && ti % 5 == cx && tj % 5 == cy && tk % 5 == cz && colmap[t] >= 0) v = rk[uc];
        }
        X[(size_t)c * n + u] = v;
    }
}

__global__ void k_probe_rows(LevelView<double> Lc, const double *probes, const int *colmap, double *A, int nF,
                             int *bw)
{
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= Lc.n) return;
    int n = Lc.n;
    const int cls = blockIdx.y % 125, comp = blockIdx.y / 125;
    const double *X = probes + (size_t)blockIdx.y * 4 * n;
    int j = u % Lc.ny, i = (u / Lc.ny) % Lc.nx, k = u / (Lc.nx * Lc.ny);
    Fields<double, double> x{X, X + n, X + 2 * n, X + 3 * n};
    int cx = cls % 5, cy = (cls / 5) % 5, cz = cls / 25;
    // the unique node of this class within two nodes
    int ci = i + ((cx - i) % 5 + 5) % 5, cj = j + ((cy - j) % 5 + 5) % 5, ck = k + ((cz - k) % 5 + 5) % 5;
    if (ci > i + 2) ci -= 5;
    if (cj > j + 2) cj -= 5;
    if (ck > k + 2) ck -= 5;
    if (ci < 0 || cj < 0 || ck < 0 || ci >= Lc.nx || cj >= Lc.ny || ck >= Lc.nz) return;
    int col = colmap[P2IDX(Lc, ci, cj, ck) * 4 + comp];
    if (col < 0) return;
    for (int c = 0; c < 4; c++) {
        int row = colmap[u * 4 + c];
        if (row < 0) continue;
        double a;
        if (c == 0) a = row_p(Lc, x, i, j, k);
        else if (c == 1) a = row_vx(Lc, x, i, j, k, (double *)nullptr);
        else if (c == 2) a = row_vy(Lc, x, i, j, k, (double *)nullptr);
        else a = row_vz(Lc, x, i, j, k, (double *)nullptr);
        A[(size_t)col * nF + row] = a;
        if (a != 0.0) {
            if (row > col) atomicMax(&bw[0], row - col);
            if (col > row) atomicMax(&bw[1], col - row);
        }
    }
}

void Solver::coarse_setup()
{
    // an LU left running by a solve that ended in an error still reads A_c
    P2_CUDA_TRY(cudaStreamSynchronize(st_lu));
    lu_pending = false;
    Level &C = L.back();
    int nl = (int)L.size();
    LevelView<double> Lc = view<double>(nl - 1, nl == 1);
    P2_CUDA_TRY(cudaMemsetAsync(A_c, 0, sizeof(double) * (size_t)nF * nF, st));
    P2_CUDA_TRY(cudaMemsetAsync(d_bw, 0, sizeof(int) * 2, st));
    dim3 grid(nblk(C.n), kProbes);
    k_probe_build<<<grid, kThreads, 0, st>>>(C.nx, C.ny, C.nz, d_colmap, d_crt, d_crk, probes); P2_COUNT_LAUNCH();
    k_probe_rows<<<grid, kThreads, 0, st>>>(Lc, probes, d_colmap, A_c, nF, d_bw); P2_COUNT_LAUNCH();
    P2_CUDA_TRY(cudaGetLastError());
    P2_CUDA_TRY(cudaMemcpyAsync(h_bw, d_bw, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
    P2_CUDA_TRY(cudaStreamSynchronize(st));
    if (!verbose) {
        // The LU and the inverse run on their own stream (st has no work in
        // flight after the synchronisation above); the solve goes on with a
        // smoothed coarsest level for lu_overlap_iters outer iterations.
        band_lu_inverse(st_lu, A_c, nF, h_bw[0], h_bw[1], Ainv64, d_ipiv, d_info, nullptr, &lu_graph, false);
        d2f(st_lu, (size_t)nF * nF, Ainv64, Ainv32);
        P2_CUDA_TRY(cudaEventRecord(ev_lu, st_lu));
        lu_pending = true;
        lu_overlap_iters = L.size() < 4 ? 0
                           : (int)std::min<double>(kOverlapMax, std::floor(kOverlapScale * nF / (double)L[0].n + 0.5));
        return;
    }
    P2_CUDA_TRY(cudaEventRecord(ev[5], st));
    int info = band_lu_inverse(st, A_c, nF, h_bw[0], h_bw[1], Ainv64, d_ipiv, d_info, verbose ? ev + 6 : nullptr,
                               &lu_graph);
    if (verbose) {
        float t0 = 0, t1 = 0, t2 = 0;
        P2_CUDA_TRY(cudaEventElapsedTime(&t0, ev[0], ev[5]));
        P2_CUDA_TRY(cudaEventElapsedTime(&t1, ev[5], ev[6]));
        P2_CUDA_TRY(cudaEventElapsedTime(&t2, ev[6], ev[7]));
        std::fprintf(stderr, "p2cuda: coarsest nF %d band kl %d ku %d; node fields + probing %.3f ms, "
                     "factorisation %.3f ms, inverse (forward) %.3f ms\n", nF, h_bw[0], h_bw[1], t0, t1, t2);
    }
    if (info) throw Error(P2_ERR_SINGULAR, "zero pivot in the coarsest LU at column " + std::to_string(info));
    d2f(st, (size_t)nF * nF, Ainv64, Ainv32);
}

// The overlapped LU: wait for it, check its pivots and order the solve's
// stream after it.
void Solver::lu_finish()
{
    if (!lu_pending) return;
    P2_CUDA_TRY(cudaEventSynchronize(ev_lu));
    int info = 0;
    P2_CUDA_TRY(cudaMemcpyAsync(&info, d_info, sizeof(int), cudaMemcpyDeviceToHost, st_lu));
    P2_CUDA_TRY(cudaStreamSynchronize(st_lu));
    P2_CUDA_TRY(cudaStreamWaitEvent(st, ev_lu, 0));
    lu_pending = false;
    if (info) throw Error(P2_ERR_SINGULAR, "zero pivot in the coarsest LU at column " + std::to_string(info));
}

// Stand-in for the coarsest direct solve: x = 0, then sweeps of the diagonal
// cell smoother (no stored factors needed) on the coarsest level.
template <typename T>
void Solver::coarse_approx(Vec4<T> &b, Vec4<T> &x)
{
    Level &C = L.back();
    for (int c = 0; c < 4; c++) P2_CUDA_TRY(cudaMemsetAsync(x.c[c], 0, sizeof(T) * C.n, st));
    const int keep = prm.smoother;
    prm.smoother = 0;
    smooth<T>((int)L.size() - 1, kCoarseApxSweeps);
    prm.smoother = keep;
    (void)b;
}

template <typename T>
void Solver::coarse_solve(Vec4<T> &b, Vec4<T> &x)
{
    if (coarse_mode) {
        coarse_approx<T>(b, x);
        return;
    }
    Level &C = L.back();
    T *bF = std::is_same<T, double>::value ? (T *)cb64 : (T *)cb32;
    T *xF = std::is_same<T, double>::value ? (T *)cx64 : (T *)cx32;
    const T *Ai = std::is_same<T, double>::value ? (const T *)Ainv64 : (const T *)Ainv32;
    for (int c = 0; c < 4; c++) P2_CUDA_TRY(cudaMemsetAsync(x.c[c], 0, sizeof(T) * C.n, st));
    pdl_launch(st, nblk(nF), kThreads, k_coarse_gather<T>, nF, (const int *)d_free, b, bF);
    pdl_launch(st, (nF + 31) / 32, 256, k_gemv<T>, nF, Ai, (const T *)bF, xF);
    pdl_launch(st, nblk(nF), kThreads, k_coarse_scatter<T>, nF, (const int *)d_free, (const T *)xF, x);
    bc_set<T>((int)L.size() - 1, x, b);
}

// ---------------------------------------------------------------------------
template <typename T>
void Solver::bc_set(int l, Vec4<T> &x, Vec4<T> &b)
{
    Level &Lv = L[l];
    if (Lv.nbc > 0) {
        pdl_launch(st, nblk(Lv.nbc), kThreads, k_bc_set_chain<T>, Lv.nbc, (const int *)Lv.bu, (const int *)Lv.bt,
                   (const float *)Lv.bk, (const int *)Lv.bnext, x, b);
    }
}

template <typename T>
static Vec4<T> &vx_of(Level &Lv, int which);
template <>
Vec4<float> &vx_of<float>(Level &Lv, int which) { return which ? Lv.y32 : Lv.x32; }
template <>
Vec4<double> &vx_of<double>(Level &Lv, int which) { return which ? Lv.y64 : Lv.x64; }
template <typename T>
static Vec4<T> &b_of(Level &Lv);
template <>
Vec4<float> &b_of<float>(Level &Lv) { return Lv.b32; }
template <>
Vec4<double> &b_of<double>(Level &Lv) { return Lv.b64; }
template <typename T>
static Vec4<T> &r_of(Level &Lv);
template <>
Vec4<float> &r_of<float>(Level &Lv) { return Lv.r32; }
template <>
Vec4<double> &r_of<double>(Level &Lv) { return Lv.r64; }

// FP32 rows run k_rows_zm when its grid has at least this many blocks (8
// per SM): with fewer, a block's column of planes is a long serial march and
// the device is not filled (measured at 129^3: 145 against 93 us for k_rows on
// level 0, 425 blocks; 128 us for 14 MB on level 1, 81 blocks), while at 257^3
// (2673 blocks) it beats k_rows (0.66 against 0.72 ms).
constexpr long kZmMinBlocks = 8L * 148;

static long zm_blocks(int nx, int ny, int nz)
{
    return (long)((nx + kZmTX - 1) / kZmTX) * ((ny + kZmTY - 1) / kZmTY) * ((nz + kZmKZ - 1) / kZmKZ);
}

template <typename T, typename S>
static void launch_rows(cudaStream_t st, bool pdl, const LevelView<T> &V, const Fields<T, S> &f, const Vec4<T> &b,
                        Vec4<T> &out, const Vec4<float> &o32, int mode, int variant = 0)
{
    if (variant == 0) variant = (sizeof(T) == 4 && zm_blocks(V.nx, V.ny, V.nz) >= kZmMinBlocks) ? 2 : 1;
    if (variant == 1) {
        if (pdl) pdl_launch(st, nblk(V.n), kThreads, k_rows<T, S>, V, f, b, out, o32, mode);
        else {
            k_rows<T, S><<<nblk(V.n), kThreads, 0, st>>>(V, f, b, out, o32, mode);
            P2_COUNT_LAUNCH();
        }
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    cfg.stream = st;
    if (variant == 2) {
        static bool attr_done = false;  // per instantiation (the attribute is per function)
        if (!attr_done) {
            P2_CUDA_TRY(cudaFuncSetAttribute(k_rows_zm<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)zm_smem_bytes<T, S>()));
            attr_done = true;
        }
        cfg.gridDim = dim3((V.nx + kZmTX - 1) / kZmTX, (V.ny + kZmTY - 1) / kZmTY, (V.nz + kZmKZ - 1) / kZmKZ);
        cfg.blockDim = dim3(kZmThreads);
        cfg.dynamicSmemBytes = zm_smem_bytes<T, S>();
        P2_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_rows_zm<T, S>, V, f, b, out, o32, mode));
        P2_COUNT_LAUNCH();
        return;
    }
    throw Error(P2_ERR_ARG, "rows kernel variant must be 0, 1 or 2");
}

// One colour pass of the selected smoother on level l.
template <typename T>
void Solver::smoother_pass(int l, const LevelView<T> &V, T *P, Vec4<T> &vin, Vec4<T> &vout, Vec4<T> &b, int col)
{
    Level &Lv = L[l];
    const long cells = (long)(Lv.nx - 1) * (Lv.nz - 1) * (Lv.ny / 2);
    const T om = (T)prm.omega;
    switch (prm.smoother) {
    case 1:
    case 5: {
        const factor_t<T> *blk = (const factor_t<T> *)Lv.blk + (size_t)col * kBlkEntries * Lv.blk_stride;
        pdl_launch(st, nblk(cells, 128), 128, k_vanka_stored<T>, V, P, vin, vout, b, om, col, blk, Lv.blk_stride);
        break;
    }
    case 2: pdl_launch(st, nblk(cells, 128), 128, k_vanka_full<T>, V, P, vin, vout, b, om, col); break;
    case 3: pdl_launch(st, nblk(cells, 128), 128, k_vanka_fast<T>, V, P, vin, vout, b, om, col); break;
    default: pdl_launch(st, nblk(cells), kThreads, k_vanka<T>, V, P, vin, vout, b, om, col); break;
    }
}

// Cell factors of the stored-factor smoother on every level, both colours
// (the level viscosities must be current), computed in FP64 and stored in
// the V-cycle's type T.
template <typename T>
void Solver::factor_smoother()
{
    for (int l = 0; l < (int)L.size(); l++) {
        Level &Lv = L[l];
        LevelView<double> V = view<double>(l, false);
        const long cells = (long)(Lv.nx - 1) * (Lv.nz - 1) * (Lv.ny / 2);
        for (int col = 0; col < 2; col++) {
            factor_t<T> *blk = (factor_t<T> *)Lv.blk + (size_t)col * kBlkEntries * Lv.blk_stride;
            k_vanka_factor<double, factor_t<T>><<<nblk(cells, 128), 128, 0, st>>>(V, col, blk, Lv.blk_stride); P2_COUNT_LAUNCH();
        }
    }
    P2_CUDA_TRY(cudaGetLastError());
}

void Solver::factor_cells()
{
    if (prm.smoother != 1 && prm.smoother != 5) return;
    if (prm.precision == 0) factor_smoother<float>();
    else factor_smoother<double>();
}

// Fused sweeps (smoother 5) on levels whose planes hold enough tiles to fill
// the device and whose boundary rows are local; other levels, and smoother 1,
// run the two colour passes.
constexpr long kFuseMinPlaneCells = 48L * 48L;

bool Solver::use_fused(int l) const
{
    const Level &Lv = L[l];
    return prm.smoother == 5 && Lv.fuse_ok && (long)(Lv.nx - 1) * (Lv.ny - 1) >= kFuseMinPlaneCells &&
           Lv.nz - 1 >= 8;
}

template <typename T>
static void sweep_kernel_setup()
{
    static bool done = false;  // per instantiation, per process (the attribute is per function)
    if (!done) {
        P2_CUDA_TRY(cudaFuncSetAttribute(k_vanka_sweep<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sweep_smem_bytes<T>()));
        done = true;
    }
}

// One fused sweep xin -> xout on level l (boundary rows of xout not set).
template <typename T>
void Solver::sweep_fused(int l, const LevelView<T> &V, Vec4<T> &xin, Vec4<T> &xout, Vec4<T> &b)
{
    Level &Lv = L[l];
    sweep_kernel_setup<T>();
    const int chunk = kSweepChunk;
    dim3 grid((Lv.nx - 1 + kSwTX - 1) / kSwTX, (Lv.ny - 1 + kSwTY - 1) / kSwTY, (Lv.nz - 1 + chunk - 1) / chunk);
    const factor_t<T> *blk0 = (const factor_t<T> *)Lv.blk, *blk1 = blk0 + (size_t)kBlkEntries * Lv.blk_stride;
    SweepBC bc{Lv.sw_first, Lv.sw_order, Lv.bu, Lv.bt, Lv.bnext, Lv.bk};
#ifdef P2_NO_PDL
    k_vanka_sweep<T><<<grid, kSwThreads, sweep_smem_bytes<T>(), st>>>(V, xin, xout, b, (T)prm.omega, blk0, blk1,
                                                                      Lv.blk_stride, bc, chunk);
    P2_COUNT_LAUNCH();
#else
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(kSwThreads);
    cfg.dynamicSmemBytes = sweep_smem_bytes<T>();
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    P2_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_vanka_sweep<T>, V, xin, xout, b, (T)prm.omega, blk0, blk1,
                                   Lv.blk_stride, bc, chunk));
    P2_COUNT_LAUNCH();
#endif
}

template <typename T>
void Solver::smooth(int l, int sweeps)
{
    Level &Lv = L[l];
    LevelView<T> V = view<T>(l, false);
    Vec4<T> &x = vx_of<T>(Lv, 0), &y = vx_of<T>(Lv, 1), &b = b_of<T>(Lv);
    bc_set<T>(l, x, b);
    if (sweeps <= 0) return;
    // colour 0 reads velocities from x and writes y, colour 1 goes back; the
    // pressure is updated in place in x.c[0] (yy shares it)
    Vec4<T> yy = y;
    yy.c[0] = x.c[0];
    int s0 = 0;
    if (use_fused(l)) {
        // pairs of fused sweeps x -> y -> x (y with its own pressure field);
        // an odd count starts with one sweep of colour passes
        if (sweeps & 1) {
            for (int col = 0; col < 2; col++) {
                Vec4<T> &vin = col ? yy : x, &vout = col ? x : yy;
                smoother_pass<T>(l, V, x.c[0], vin, vout, b, col);
                bc_set<T>(l, vout, b);
            }
            s0 = 1;
        }
        for (int s = s0; s < sweeps; s += 2) {
            sweep_fused<T>(l, V, x, y, b);
            bc_set<T>(l, y, b);
            sweep_fused<T>(l, V, y, x, b);
            bc_set<T>(l, x, b);
        }
        return;
    }
    for (int s = 0; s < sweeps; s++) {
        for (int col = 0; col < 2; col++) {
            Vec4<T> &vin = col ? yy : x, &vout = col ? x : yy;
            smoother_pass<T>(l, V, x.c[0], vin, vout, b, col);
            bc_set<T>(l, vout, b);
        }
    }
}

template <typename T>
void Solver::level_residual(int l)
{
    Level &Lv = L[l];
    LevelView<T> V = view<T>(l, false);
    Vec4<T> &x = vx_of<T>(Lv, 0), &b = b_of<T>(Lv), &r = r_of<T>(Lv);
    Fields<T, T> f{x.c[0], x.c[1], x.c[2], x.c[3]};
    Vec4<float> none;
    launch_rows<T, T>(st, true, V, f, b, r, none, 0, dbg_rows_variant);
    if (Lv.nbc)
        pdl_launch(st, nblk(Lv.nbc), kThreads, k_bc_rows<T, T>, Lv.nbc, (const int *)Lv.bu, (const int *)Lv.bt,
                   (const float *)Lv.bk, f, b, r, none, 0);
}

template <typename T>
void Solver::vcycle()
{
    int nl = (int)L.size();
    for (int l = 0; l < nl - 1; l++) {
        smooth<T>(l, prm.npre[l]);
        level_residual<T>(l);
        Level &F = L[l], &Cl = L[l + 1];
        LevelView<T> VF = view<T>(l, false), VC = view<T>(l + 1, false);
        pdl_launch(st, nblk(4L * Cl.n), kThreads, k_restrict_compat<T>, VF, r_of<T>(F), VC, b_of<T>(Cl),
                   vx_of<T>(Cl, 0), F.tv, 1, Cl.compat_vol, rpartial, rticket, scal);
        pdl_launch(st, nblk(Cl.n), kThreads, k_compat_apply<T>, VC, b_of<T>(Cl).c[0], (const double *)scal);
    }
    if (nl > 1) coarse_solve<T>(b_of<T>(L[nl - 1]), vx_of<T>(L[nl - 1], 0));
    else coarse_solve<T>(b_of<T>(L[0]), vx_of<T>(L[0], 0));
    for (int l = nl - 2; l >= 0; l--) {
        Level &F = L[l], &Cl = L[l + 1];
        LevelView<T> VF = view<T>(l, false), VC = view<T>(l + 1, false);
        pdl_launch(st, nblk(F.n), kThreads, k_prolong<T>, VF, vx_of<T>(F, 0), VC, vx_of<T>(Cl, 0), F.tv,
                   (T)prm.p1koef, (T)prm.v1koef);
        smooth<T>(l, prm.npost[l]);
    }
}

// ---------------------------------------------------------------------------
void Solver::set_nodes_device()
{
    // coarse nu/ro (ronurestrict), per-stencil viscosities, level-0 rhs
    int nl = (int)L.size();
    for (int l = 1; l < nl; l++) {
        Level &F = L[l - 1], &C = L[l];
        k_ronurestrict<<<nblk(C.n), kThreads, 0, st>>>(F.nx, F.ny, F.nz, F.nu, F.ro, C.nx, C.ny, C.nz, C.nu, C.ro,
                                                       F.ronu[0], F.ronu[1], F.ronu[2], prm.viscmod); P2_COUNT_LAUNCH();
    }
    for (int l = 0; l < nl; l++) {
        Level &Lv = L[l];
        k_level_eta<<<nblk(Lv.n), kThreads, 0, st>>>(Lv.nx, Lv.ny, Lv.nz, Lv.nu, f0.nxx, f0.nxy, f0.nxz, f0.nyz,
                                                     Lv.ec, Lv.exy, Lv.exz, Lv.eyz, prm.nubeg, prm.nuend,
                                                     prm.viscmod, l == 0); P2_COUNT_LAUNCH();
    }
    Level &L0 = L[0];
    k_rhs0<double><<<nblk(L0.n), kThreads, 0, st>>>(L0.nx, L0.ny, L0.nz, L0.ro, L0.bcm, gb, prm.gxkoef, prm.gykoef,
                                                    prm.gzkoef); P2_COUNT_LAUNCH();
    if (L0.nbc) k_bc_consts<double><<<nblk(L0.nbc), kThreads, 0, st>>>(L0.nbc, L0.bu, L0.bconst, gb); P2_COUNT_LAUNCH();
    P2_CUDA_TRY(cudaGetLastError());
}

void Solver::upload_nodes(const float *nu, const float *ro, const float *nxx, const float *nxy, const float *nxz,
                          const float *nyz)
{
    if (!bc_ready) throw Error(P2_ERR_STATE, "node fields before p2_set_bc");
    long n = L[0].n;
    const float *src[6] = {nu, ro, nxx, nxy, nxz, nyz};
    float *dst[6] = {L[0].nu, L[0].ro, f0.nxx, f0.nxy, f0.nxz, f0.nyz};
    for (int q = 0; q < 6; q++) {
        if (!src[q]) throw Error(P2_ERR_ARG, "null node field");
        P2_CUDA_TRY(cudaMemcpyAsync(dst[q], src[q], sizeof(float) * n, cudaMemcpyHostToDevice, st));
    }
    nodes_ready = true;
}

void Solver::dots_sync(const DotJobs &jobs)
{
    P2_CUDA_TRY(launch_dots(st, jobs, L[0].n, L[0].pin, partial)); P2_COUNT_LAUNCH();
    k_dots_final<<<1, 1024, 0, st>>>(jobs.nd, kRedBlocks, partial, dots); P2_COUNT_LAUNCH();
    P2_CUDA_TRY(cudaMemcpyAsync(hdots.get(), dots, sizeof(double) * jobs.nd, cudaMemcpyDeviceToHost, st));
    P2_CUDA_TRY(cudaStreamSynchronize(st));
}

static DotJob job(const Vec4<double> &a, const Vec4<double> &b)
{
    DotJob j;
    for (int c = 0; c < 4; c++) { j.a[c] = a.c[c]; j.b[c] = b.c[c]; }
    return j;
}

// out = b - A x (mode 0) or A x (mode 1) on level 0 in FP64 (x stored as
// S); r32 optional.
template <typename S>
void Solver::rows0(const Vec4<S> &x, Vec4<double> &out, Vec4<float> *r32, int mode)
{
    Level &L0 = L[0];
    LevelView<double> V = view<double>(0, true);
    Fields<double, S> f{x.c[0], x.c[1], x.c[2], x.c[3]};
    Vec4<float> o32 = r32 ? *r32 : Vec4<float>();
    launch_rows<double, S>(st, false, V, f, gb, out, o32, mode, dbg_rows_variant);
    if (L0.nbc) {
        k_bc_rows<double, S><<<nblk(L0.nbc), kThreads, 0, st>>>(L0.nbc, L0.bu, L0.bt, L0.bk, f, gb, out, o32, mode);
        P2_COUNT_LAUNCH();
    }
}

// One preconditioning V-cycle from zero for the level-0 right-hand side r:
// the mixed cycle reads float(r), which the true residual wrote into b32;
// the FP64 cycle's level-0 right-hand side is r itself (b64 of level 0 is
// gr).  The correction stays in x32 / x64; the Gram-Schmidt update reads it
// from there.
void Solver::precondition()
{
    Level &L0 = L[0];
    if (prm.precision == 0) {
        for (int c = 0; c < 4; c++) P2_CUDA_TRY(cudaMemsetAsync(L0.x32.c[c], 0, sizeof(float) * L0.n, st));
        run_vcycle_graph<float>();
    } else {
        for (int c = 0; c < 4; c++) P2_CUDA_TRY(cudaMemsetAsync(L0.x64.c[c], 0, sizeof(double) * L0.n, st));
        run_vcycle_graph<double>();
    }
}

// Capture (once per configuration) and upload the V-cycle graph.
template <typename T>
void Solver::capture_vcycle_graph()
{
    GraphSlot &g = (coarse_mode ? graphs_apx : graphs)[std::is_same<T, double>::value ? 1 : 0];
    if (g.exec || !prm.use_graphs) return;
    cudaGraph_t graph;
    long long before = g_launches;
    P2_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    vcycle<T>();
    P2_CUDA_TRY(cudaStreamEndCapture(st, &graph));
    g.kernels = g_launches - before;  // captured, not yet executed
    g_launches = before;
    P2_CUDA_TRY(cudaGraphInstantiate(&g.exec, graph, 0));
    cudaGraphDestroy(graph);
    P2_CUDA_TRY(cudaGraphUpload(g.exec, st));
}

template <typename T>
void Solver::run_vcycle_graph()
{
    int key = std::is_same<T, double>::value ? 1 : 0;
    GraphSlot &g = (coarse_mode ? graphs_apx : graphs)[key];
    if (!prm.use_graphs) {
        vcycle<T>();
        P2_CUDA_TRY(cudaGetLastError());
        return;
    }
    capture_vcycle_graph<T>();
    P2_CUDA_TRY(cudaGraphLaunch(g.exec, st));
    g_launches += g.kernels;
}

thread_local long long g_launches = 0;

p2_solve_info Solver::solve()
{
    const char *vb = std::getenv("P2CUDA_VERBOSE");
    verbose = vb && vb[0] == '1';
    if (!nodes_ready) throw Error(P2_ERR_STATE, "solve before node fields were set");
    p2_solve_info info{};
    long long launches0 = g_launches;
    Level &L0 = L[0];
    long n = L0.n;
    P2_CUDA_TRY(cudaEventRecord(ev[0], st));
    set_nodes_device();
    factor_cells();
    coarse_setup();
    P2_CUDA_TRY(cudaEventRecord(ev[1], st));
    if (verbose) {
        float tb = 0;
        P2_CUDA_TRY(cudaEventSynchronize(ev[1]));
        P2_CUDA_TRY(cudaEventElapsedTime(&tb, ev[7], ev[1]));
        std::fprintf(stderr, "p2cuda: inverse (backward) + FP32 copy %.3f ms; V-cycle graph %lld kernels\n", tb,
                     graphs[prm.precision == 0 ? 0 : 1].kernels);
    }
    // b-norm of the pinned system: every row but the pin cell's, plus the pin value
    DotJobs J{};
    J.j[0] = job(gb, gb);
    J.nd = 1;
    dots_sync(J);
    double bnorm2 = hdots.get()[0] + (L0.pin >= 0 ? L0.pinval * L0.pinval : 0.0);
    double bnorm = std::sqrt(bnorm2);
    if (!(bnorm > 0)) bnorm = 1.0;
    int m = restart, k = 0, it = 0;
    float vc_ms = 0;
    double rel = 0;
    if ((int)vc_ev.size() < 2) {
        vc_ev.resize(2);
        for (auto &e : vc_ev) P2_CUDA_TRY(cudaEventCreate(&e));
    }
    std::vector<std::pair<int, int>> vc_marks;  // event pairs around each V-cycle
    P2_CUDA_TRY(cudaMemsetAsync(scal + 4, 0, sizeof(double), st));  // non-positive direction norm flag
    for (;;) {
        // true FP64 residual (its float copy is the mixed cycle's right-hand side)
        rows0(gx, gr, prm.precision == 0 ? &L0.b32 : nullptr, 0);
        // the one host synchronisation of an iteration: the residual norm and
        // the flag of the previous iteration's direction
        J.nd = 1;
        J.j[0] = job(gr, gr);
        P2_CUDA_TRY(launch_dots(st, J, L0.n, L0.pin, partial)); P2_COUNT_LAUNCH();
        k_dots_final<<<1, 1024, 0, st>>>(1, kRedBlocks, partial, dots); P2_COUNT_LAUNCH();
        P2_CUDA_TRY(cudaMemcpyAsync(hdots.get(), dots, sizeof(double), cudaMemcpyDeviceToHost, st));
        P2_CUDA_TRY(cudaMemcpyAsync(hdots.get() + 1, scal + 4, sizeof(double), cudaMemcpyDeviceToHost, st));
        P2_CUDA_TRY(cudaStreamSynchronize(st));
        double rr = hdots.get()[0];
        rel = std::sqrt(rr) / bnorm;
        if (it == 0) info.rel_residual0 = rel;
        if (verbose) std::fprintf(stderr, "p2cuda: iteration %d rel residual %.3e\n", it, rel);
        if (hdots.get()[1] != 0.0 || !std::isfinite(rel)) { info.status = P2_ERR_NAN; break; }
        if (rel <= prm.tol) { info.status = P2_OK; break; }
        if (it >= prm.max_iter) { info.status = P2_ERR_NOT_CONVERGED; break; }
        Vec4<double> &z = Z[k], &q = Q[k];
        if (it >= lu_overlap_iters) lu_finish();
        coarse_mode = lu_pending ? 1 : 0;
        const int e0 = 2 * (int)vc_marks.size();
        if ((int)vc_ev.size() < e0 + 2) {
            const size_t old = vc_ev.size();
            vc_ev.resize(e0 + 2);
            for (size_t e = old; e < vc_ev.size(); e++) P2_CUDA_TRY(cudaEventCreate(&vc_ev[e]));
        }
        P2_CUDA_TRY(cudaEventRecord(vc_ev[e0], st));
        precondition();
        P2_CUDA_TRY(cudaEventRecord(vc_ev[e0 + 1], st));
        vc_marks.push_back({e0, e0 + 1});
        // q = A c for the correction c (x32 or x64 of level 0)
        if (prm.precision == 0) rows0(L0.x32, q, nullptr, 1);
        else rows0(L0.x64, q, nullptr, 1);
        // classical Gram-Schmidt against the stored directions: coefficients
        // on the device, then one pass that updates q and z and sums (q', q')
        // and (r, q'), then alpha on the device and the solution update
        if (k > 0) {
            J.nd = 0;
            for (int j = 0; j < k; j++) J.j[J.nd++] = job(q, Q[j]);
            P2_CUDA_TRY(launch_dots(st, J, L0.n, L0.pin, partial)); P2_COUNT_LAUNCH();
            k_dots_final<<<1, 1024, 0, st>>>(k, kRedBlocks, partial, dots); P2_COUNT_LAUNCH();
            k_gcr_coef<<<1, 32, 0, st>>>(k, dots, qq_dev, scal + 8); P2_COUNT_LAUNCH();
        }
        VecList X{}, Zl{};
        for (int j = 0; j < k; j++)
            for (int c = 0; c < 4; c++) { X.v[j][c] = Q[j].c[c]; Zl.v[j][c] = Z[j].c[c]; }
        X.nv = Zl.nv = k;
        if (prm.precision == 0)
            P2_CUDA_TRY(launch_cgs_update_dots<float>(st, k, (int)n, scal + 8, q, X, L0.x32, z, Zl, gr, L0.pin, partial));
        else
            P2_CUDA_TRY(launch_cgs_update_dots<double>(st, k, (int)n, scal + 8, q, X, L0.x64, z, Zl, gr, L0.pin, partial));
        P2_COUNT_LAUNCH();
        k_dots_final<<<1, 1024, 0, st>>>(2, kRedBlocks, partial, dots); P2_COUNT_LAUNCH();
        k_gcr_alpha<<<1, 32, 0, st>>>(dots, qq_dev + k, scal + 2, scal + 4); P2_COUNT_LAUNCH();
        k_axpy4<<<nblk(n), kThreads, 0, st>>>((int)n, scal + 2, 1.0, gx, z); P2_COUNT_LAUNCH();
        k = (k + 1) % m;
        it++;
    }
    for (const auto &mk : vc_marks) {
        float t = 0;
        P2_CUDA_TRY(cudaEventElapsedTime(&t, vc_ev[mk.first], vc_ev[mk.second]));
        vc_ms += t;
    }
    // the overlapped LU has to be finished (and its pivots checked) before
    // the solve returns; the graphs after it use the exact coarsest solve
    coarse_mode = 0;
    lu_finish();
    // pressure shift to the pinned value
    k_pressure_shift_value<<<1, 32, 0, st>>>(gx.c[0], L0.pin, L0.pinval, scal + 3); P2_COUNT_LAUNCH();
    k_pressure_shift<<<nblk(n), kThreads, 0, st>>>(L0.nx, L0.ny, L0.nz, gx.c[0], scal + 3); P2_COUNT_LAUNCH();
    P2_CUDA_TRY(cudaEventRecord(ev[4], st));
    P2_CUDA_TRY(cudaEventSynchronize(ev[4]));
    float tt = 0, ts = 0;
    P2_CUDA_TRY(cudaEventElapsedTime(&tt, ev[0], ev[4]));
    P2_CUDA_TRY(cudaEventElapsedTime(&ts, ev[0], ev[1]));
    solution_ready = true;
    info.iterations = it;
    info.rel_residual = rel;
    info.ms_total = tt;
    info.ms_setup = ts;
    info.ms_vcycles = vc_ms;
    info.kernels = g_launches - launches0;
    return info;
}

// Try each smoother configuration for trial_iters outer iterations; keep the
// one with the least estimated time to prm.tol.
p2_tune_info Solver::autotune(int trial_iters)
{
    if (!nodes_ready) throw Error(P2_ERR_STATE, "autotune before node fields were set");
    if (trial_iters < 2 || trial_iters > 1000) throw Error(P2_ERR_ARG, "trial_iters out of 2..1000");
    const p2_params saved = prm;
    const int nl = (int)L.size();
    const int base_pre = std::max(1, saved.npre[0]), base_post = std::max(1, saved.npost[0]);
    p2_tune_info best{};
    best.est_ms = INFINITY;
    best.trial_iters = trial_iters;
    double setup_ms = INFINITY;
    // candidates: smoother x (sweep growth per coarser level, most sweeps per
    // level) x (sweeps on level 0: the configured ones or half of them; the
    // coarser levels keep theirs)
    struct Cand { int smoother, growth, cap, half0; };
    const Cand cands[12] = {{1, 1, 64, 0}, {1, 2, 64, 0}, {1, 2, 16, 0}, {0, 1, 64, 0}, {0, 2, 64, 0}, {0, 2, 16, 0},
                            {1, 1, 64, 1}, {1, 2, 64, 1}, {1, 2, 16, 1}, {0, 1, 64, 1}, {0, 2, 64, 1}, {0, 2, 16, 1}};
    const int ncand = (base_pre >= 2 && base_post >= 2) ? 12 : 6;
    for (int ci = 0; ci < ncand; ci++) {
        const Cand &cd = cands[ci];
        {
            prm = saved;
            prm.smoother = cd.smoother;
            prm.max_iter = trial_iters;
            for (int l = 0; l < nl; l++) {
                long f = 1;
                for (int q = 0; q < l; q++) f *= cd.growth;
                prm.npre[l] = (int)std::min<long>(cd.cap, base_pre * f);
                prm.npost[l] = (int)std::min<long>(cd.cap, base_post * f);
            }
            if (cd.half0) {
                prm.npre[0] = base_pre / 2;
                prm.npost[0] = base_post / 2;
            }
            drop_graphs();
            set_initial(nullptr, nullptr, nullptr, nullptr);
            // the candidate's V-cycle graph is captured before its trial, so the
            // timed iterations hold no capture; the set-up (coarse viscosities,
            // factors, coarsest LU) is the same for every candidate and is left
            // out of the comparison (the first trial also captures the LU graph)
            if (prm.precision == 0) capture_vcycle_graph<float>();
            else capture_vcycle_graph<double>();
            p2_solve_info in = solve();
            double est = INFINITY, rate = 1.0;
            if (in.iterations > 0 && in.rel_residual > 0 && in.rel_residual0 > 0) {
                rate = std::pow(in.rel_residual / in.rel_residual0, 1.0 / in.iterations);
                double per_it = (in.ms_total - in.ms_setup) / in.iterations;
                if (in.status == P2_OK) est = in.ms_total - in.ms_setup;
                else if (rate < 1.0 && std::isfinite(rate))
                    est = per_it * (in.iterations + std::log(saved.tol / in.rel_residual) / std::log(rate));
            }
            setup_ms = std::min(setup_ms, (double)in.ms_setup);
            if (verbose)
                std::fprintf(stderr, "p2cuda: autotune smoother %d growth %d cap %d level-0 sweeps %d: %d its, rate %.3f, "
                             "est %.1f ms\n", prm.smoother, cd.growth, cd.cap, prm.npre[0], in.iterations, rate, est);
            best.candidates++;
            if (est < best.est_ms) {
                best.est_ms = est;
                best.smoother = prm.smoother;
                best.sweep_growth = cd.growth;
                best.sweep_max = cd.cap;
                best.sweeps0 = prm.npre[0];
                best.rate = rate;
            }
        }
    }
    prm = saved;
    if (std::isfinite(best.est_ms) && std::isfinite(setup_ms)) best.est_ms += setup_ms;
    if (!std::isfinite(best.est_ms)) {
        // nothing converged within the trials: keep the defaults
        best.smoother = saved.smoother;
        best.sweep_growth = 1;
        best.sweep_max = 64;
        best.sweeps0 = saved.npre[0];
    } else {
        prm.smoother = best.smoother;
        for (int l = 0; l < nl; l++) {
            long f = 1;
            for (int q = 0; q < l; q++) f *= best.sweep_growth;
            prm.npre[l] = (int)std::min<long>(best.sweep_max, base_pre * f);
            prm.npost[l] = (int)std::min<long>(best.sweep_max, base_post * f);
        }
        if (best.sweeps0 != base_pre) {
            prm.npre[0] = base_pre / 2;
            prm.npost[0] = base_post / 2;
        }
    }
    // GCR restart length: full solves of the chosen schedule with the
    // configured length and with 12 (the directions stay allocated for the
    // longer one); the trials above stop before a restart shows its effect
    best.restart = restart;
    if (std::isfinite(best.est_ms) && restart > 12) {
        const int configured = restart;
        double t_best = INFINITY;
        for (int m : {configured, 12}) {
            restart = m;
            drop_graphs();
            set_initial(nullptr, nullptr, nullptr, nullptr);
            if (prm.precision == 0) capture_vcycle_graph<float>();
            else capture_vcycle_graph<double>();
            p2_solve_info in = solve();
            const double t = in.status == P2_OK ? in.ms_total - in.ms_setup : INFINITY;
            if (verbose)
                std::fprintf(stderr, "p2cuda: autotune restart %d: %d its, %.1f ms\n", m, in.iterations, t);
            if (t < t_best) {
                t_best = t;
                best.restart = m;
            }
        }
        restart = best.restart;
    }
    drop_graphs();
    set_initial(nullptr, nullptr, nullptr, nullptr);
    return best;
}

// float -> double of one field (the initial guess of the host-array call)
__global__ void k_field_f32_to_f64(long n, const float *a, double *b)
{
    const long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n) b[u] = (double)a[u];
}

// the solution with the entries that are not unknowns (ghost positions) zero
__global__ void k_solution_masked(int nx, int ny, int nz, Vec4<double> x, Vec4<double> out)
{
    const long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= (long)nx * ny * nz) return;
    const int j = (int)(u % ny), i = (int)((u / ny) % nx), k = (int)(u / ((long)nx * ny));
#pragma unroll
    for (int c = 0; c < 4; c++)
        if (out.c[c]) out.c[c][u] = valid_pos(c, i, j, k, nx, ny, nz) ? x.c[c][u] : 0.0;
}

// Initial guess: float velocities and double pressure from the caller's
// arrays (copied as they are, converted on the device), or zero.
void Solver::set_initial(const float *vx, const float *vy, const float *vz, const double *pr)
{
    long n = L[0].n;
    for (int c = 0; c < 4; c++) P2_CUDA_TRY(cudaMemsetAsync(gx.c[c], 0, sizeof(double) * n, st));
    if (!vx && !vy && !vz && !pr) return;
    ensure_move_buffers(0);
    const float *fs[3] = {vx, vy, vz};
    for (int c = 1; c < 4; c++) {
        if (!fs[c - 1]) continue;
        P2_CUDA_TRY(cudaMemcpyAsync(mv_vel[c - 1], fs[c - 1], sizeof(float) * n, cudaMemcpyHostToDevice, st));
        k_field_f32_to_f64<<<nblk(n), kThreads, 0, st>>>(n, mv_vel[c - 1], gx.c[c]); P2_COUNT_LAUNCH();
    }
    if (pr) P2_CUDA_TRY(cudaMemcpyAsync(gx.c[0], pr, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    P2_CUDA_TRY(cudaStreamSynchronize(st));  // the caller's arrays may be reused after return
}

// FP64 solution into the caller's arrays (nullptr skips), ghost positions 0.
void Solver::get_solution(double *vx, double *vy, double *vz, double *pr)
{
    const Level &L0 = L[0];
    long n = L0.n;
    double *dst[4] = {pr, vx, vy, vz};
    Vec4<double> out = gr;  // the residual work vector is free after a solve
    for (int c = 0; c < 4; c++)
        if (!dst[c]) out.c[c] = nullptr;
    k_solution_masked<<<nblk(n), kThreads, 0, st>>>(L0.nx, L0.ny, L0.nz, gx, out); P2_COUNT_LAUNCH();
    for (int c = 0; c < 4; c++)
        if (dst[c]) P2_CUDA_TRY(cudaMemcpyAsync(dst[c], out.c[c], sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    P2_CUDA_TRY(cudaStreamSynchronize(st));
}

// The host-array form of the solution (vpiterate's write-back): float
// velocities (the FP64 solution rounded, ghost positions 0) and the double
// pressure, converted on the device and copied straight into the caller's
// arrays (nullptr skips).
void Solver::get_solution_f32(float *vx, float *vy, float *vz, double *pr)
{
    const Level &L0 = L[0];
    long n = L0.n;
    ensure_move_buffers(0);
    velocity_f32();
    if (pr) {
        Vec4<double> out{};
        out.c[0] = gr.c[0];
        k_solution_masked<<<nblk(n), kThreads, 0, st>>>(L0.nx, L0.ny, L0.nz, gx, out); P2_COUNT_LAUNCH();
        P2_CUDA_TRY(cudaMemcpyAsync(pr, gr.c[0], sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    }
    float *dst[3] = {vx, vy, vz};
    for (int c = 0; c < 3; c++)
        if (dst[c]) P2_CUDA_TRY(cudaMemcpyAsync(dst[c], mv_vel[c], sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    P2_CUDA_TRY(cudaStreamSynchronize(st));
}


// ---------------------------------------------------------------------------
// Test hooks (FP64, interleaved [P,Vx,Vy,Vz] per node as the reference's sol0).
static void to_vec4(cudaStream_t st, const double *h, int n, Vec4<double> &v)
{
    std::vector<double> tmp(n);
    for (int c = 0; c < 4; c++) {
        for (int u = 0; u < n; u++) tmp[u] = h[(size_t)u * 4 + c];
        P2_CUDA_TRY(cudaMemcpyAsync(v.c[c], tmp.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
        P2_CUDA_TRY(cudaStreamSynchronize(st));
    }
}
static void from_vec4(cudaStream_t st, const Vec4<double> &v, int n, double *h)
{
    std::vector<double> tmp(n);
    for (int c = 0; c < 4; c++) {
        P2_CUDA_TRY(cudaMemcpyAsync(tmp.data(), v.c[c], sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        P2_CUDA_TRY(cudaStreamSynchronize(st));
        for (int u = 0; u < n; u++) h[(size_t)u * 4 + c] = tmp[u];
    }
}
struct TmpVec {
    Vec4<double> v;
    double *base = nullptr;
    explicit TmpVec(int n)
    {
        P2_CUDA_TRY(cudaMalloc(&base, sizeof(double) * 4 * (size_t)n));
        P2_CUDA_TRY(cudaMemsetAsync(base, 0, sizeof(double) * 4 * (size_t)n, 0));
        P2_CUDA_TRY(cudaStreamSynchronize(0));  // ordered before copies on the non-blocking stream
        for (int c = 0; c < 4; c++) v.c[c] = base + (size_t)c * n;
        v.n = n;
    }
    ~TmpVec() { cudaFree(base); }
};

void Solver::debug_prepare()
{
    if (!nodes_ready) throw Error(P2_ERR_STATE, "node fields not set");
    set_nodes_device();
    P2_CUDA_TRY(cudaStreamSynchronize(st));
}

// y = A x on level l: operator rows, boundary rows x - koef x_t, identity elsewhere.
void Solver::debug_apply(int l, const double *x, double *y)
{
    if (l < 0 || l >= (int)L.size()) throw Error(P2_ERR_ARG, "level out of range");
    debug_prepare();
    Level &Lv = L[l];
    TmpVec X(Lv.n), Y(Lv.n), B(Lv.n);
    to_vec4(st, x, Lv.n, X.v);
    LevelView<double> V = view<double>(l, l == 0);
    Fields<double, double> f{X.v.c[0], X.v.c[1], X.v.c[2], X.v.c[3]};
    Vec4<float> none;
    launch_rows<double, double>(st, false, V, f, B.v, Y.v, none, 1, dbg_rows_variant);
    if (Lv.nbc)
        k_bc_rows<double, double><<<nblk(Lv.nbc), kThreads, 0, st>>>(Lv.nbc, Lv.bu, Lv.bt, Lv.bk, f, B.v, Y.v, none, 1); P2_COUNT_LAUNCH();
    P2_CUDA_TRY(cudaGetLastError());
    from_vec4(st, Y.v, Lv.n, y);
    // identity on positions that are not unknowns, the pinned row as a boundary row
    for (int u = 0; u < Lv.n; u++) {
        int j = u % Lv.ny, i = (u / Lv.ny) % Lv.nx, k = u / (Lv.nx * Lv.ny);
        for (int c = 0; c < 4; c++)
            if (!valid_pos(c, i, j, k, Lv.nx, Lv.ny, Lv.nz)) y[(size_t)u * 4 + c] = x[(size_t)u * 4 + c];
        if (u == Lv.pin) y[(size_t)u * 4] = x[(size_t)u * 4];
    }
}

// coarse rhs from a fine residual (vprestrict), optionally with the compatibility shift
void Solver::debug_restrict(int lc, const double *fine_res, double *coarse_rhs, int compat)
{
    if (lc < 1 || lc >= (int)L.size()) throw Error(P2_ERR_ARG, "level out of range");
    debug_prepare();
    Level &F = L[lc - 1], &Cl = L[lc];
    TmpVec R(F.n), Bc(Cl.n), Xc(Cl.n);
    to_vec4(st, fine_res, F.n, R.v);
    LevelView<double> VF = view<double>(lc - 1, false), VC = view<double>(lc, false);
    // the V-cycle's restriction kernel (with its fused compatibility sums)
    k_restrict_compat<double><<<nblk(4L * Cl.n), kThreads, 0, st>>>(VF, R.v, VC, Bc.v, Xc.v, F.tv, 1, Cl.compat_vol,
                                                                     rpartial, rticket, scal); P2_COUNT_LAUNCH();
    if (compat) {
        k_compat_apply<double><<<nblk(Cl.n), kThreads, 0, st>>>(VC, Bc.v.c[0], scal); P2_COUNT_LAUNCH();
    }
    P2_CUDA_TRY(cudaGetLastError());
    from_vec4(st, Bc.v, Cl.n, coarse_rhs);
}

void Solver::debug_prolong(int lc, const double *coarse_x, double *fine_x)
{
    if (lc < 1 || lc >= (int)L.size()) throw Error(P2_ERR_ARG, "level out of range");
    debug_prepare();
    Level &F = L[lc - 1], &Cl = L[lc];
    TmpVec Xf(F.n), Xc(Cl.n);
    to_vec4(st, fine_x, F.n, Xf.v);
    to_vec4(st, coarse_x, Cl.n, Xc.v);
    LevelView<double> VF = view<double>(lc - 1, false), VC = view<double>(lc, false);
    k_prolong<double><<<nblk(F.n), kThreads, 0, st>>>(VF, Xf.v, VC, Xc.v, F.tv, prm.p1koef, prm.v1koef); P2_COUNT_LAUNCH();
    P2_CUDA_TRY(cudaGetLastError());
    from_vec4(st, Xf.v, F.n, fine_x);
}

// `sweeps` sweeps of the configured smoother (as the V-cycle runs them, in its
// precision) on level l: state x (in/out) for the right-hand side b, both
// interleaved FP64 [P,Vx,Vy,Vz] per node of the level.
void Solver::debug_smooth(int l, int sweeps, const double *b, double *x)
{
    if (l < 0 || l >= (int)L.size() || sweeps < 0 || sweeps > 64) throw Error(P2_ERR_ARG, "bad level or sweep count");
    debug_prepare();
    factor_cells();
    Level &Lv = L[l];
    TmpVec X(Lv.n), B(Lv.n);
    to_vec4(st, x, Lv.n, X.v);
    to_vec4(st, b, Lv.n, B.v);
    if (prm.precision == 0) {
        for (int c = 0; c < 4; c++) {
            d2f(st, (size_t)Lv.n, X.v.c[c], Lv.x32.c[c]);
            d2f(st, (size_t)Lv.n, B.v.c[c], Lv.b32.c[c]);
        }
        smooth<float>(l, sweeps);
        k_f32_to_f64<<<nblk(Lv.n), kThreads, 0, st>>>(Lv.n, Lv.x32, X.v); P2_COUNT_LAUNCH();
    } else {
        for (int c = 0; c < 4; c++) {
            P2_CUDA_TRY(cudaMemcpyAsync(Lv.x64.c[c], X.v.c[c], sizeof(double) * Lv.n, cudaMemcpyDeviceToDevice, st));
            P2_CUDA_TRY(cudaMemcpyAsync(Lv.b64.c[c], B.v.c[c], sizeof(double) * Lv.n, cudaMemcpyDeviceToDevice, st));
        }
        smooth<double>(l, sweeps);
        for (int c = 0; c < 4; c++)
            P2_CUDA_TRY(cudaMemcpyAsync(X.v.c[c], Lv.x64.c[c], sizeof(double) * Lv.n, cudaMemcpyDeviceToDevice, st));
    }
    P2_CUDA_TRY(cudaGetLastError());
    from_vec4(st, X.v, Lv.n, x);
}

// One preconditioning V-cycle (in the solver's precision, with the exact
// coarsest solve) from x = 0 for the level-0 right-hand side b.
void Solver::debug_vcycle(const double *b, double *x)
{
    debug_prepare();
    factor_cells();
    coarse_setup();
    lu_finish();
    coarse_mode = 0;
    Level &L0 = L[0];
    TmpVec B(L0.n), X(L0.n);
    to_vec4(st, b, L0.n, B.v);
    if (prm.precision == 0) {
        for (int c = 0; c < 4; c++) {
            d2f(st, (size_t)L0.n, B.v.c[c], L0.b32.c[c]);
            P2_CUDA_TRY(cudaMemsetAsync(L0.x32.c[c], 0, sizeof(float) * L0.n, st));
        }
        run_vcycle_graph<float>();
        k_f32_to_f64<<<nblk(L0.n), kThreads, 0, st>>>(L0.n, L0.x32, X.v); P2_COUNT_LAUNCH();
    } else {
        for (int c = 0; c < 4; c++) {
            P2_CUDA_TRY(cudaMemcpyAsync(L0.b64.c[c], B.v.c[c], sizeof(double) * L0.n, cudaMemcpyDeviceToDevice, st));
            P2_CUDA_TRY(cudaMemsetAsync(L0.x64.c[c], 0, sizeof(double) * L0.n, st));
        }
        run_vcycle_graph<double>();
        for (int c = 0; c < 4; c++)
            P2_CUDA_TRY(cudaMemcpyAsync(X.v.c[c], L0.x64.c[c], sizeof(double) * L0.n, cudaMemcpyDeviceToDevice, st));
    }
    P2_CUDA_TRY(cudaGetLastError());
    from_vec4(st, X.v, L0.n, x);
}

// Average device time of one smoother sweep on level l as the V-cycle runs
// it (both colours and their boundary rows; fused where the level allows),
// on the state left by the last solve: `sweeps` sweeps timed together after
// a 256 MB write that evicts L2, repeated 10 times.
double Solver::debug_time_sweep(int l, int sweeps)
{
    if (l < 0 || l >= (int)L.size() || sweeps < 1 || sweeps > 64) throw Error(P2_ERR_ARG, "bad level or sweep count");
    if (!bc_ready) throw Error(P2_ERR_STATE, "no level data");
    factor_cells();
    const size_t flush_bytes = (size_t)256 << 20;
    void *flush = nullptr;
    P2_CUDA_TRY(cudaMalloc(&flush, flush_bytes));
    struct Free { void *p; ~Free() { if (p) cudaFree(p); } } hold{flush};
    double total = 0;
    const int reps = 10;
    for (int r = 0; r < reps; r++) {
        P2_CUDA_TRY(cudaMemsetAsync(flush, r & 0xff, flush_bytes, st));
        P2_CUDA_TRY(cudaEventRecord(ev[5], st));
        if (prm.precision == 0) smooth<float>(l, sweeps);
        else smooth<double>(l, sweeps);
        P2_CUDA_TRY(cudaEventRecord(ev[6], st));
        P2_CUDA_TRY(cudaEventSynchronize(ev[6]));
        float ms = 0;
        P2_CUDA_TRY(cudaEventElapsedTime(&ms, ev[5], ev[6]));
        total += ms;
    }
    P2_CUDA_TRY(cudaGetLastError());
    return total / reps / sweeps;
}

// Average device time of one stage of the solve on the state left by the
// last solve, each repetition timed alone after a 256 MB write that evicts
// L2: 0 the V-cycle residual of `level` (its rows kernel chosen by variant:
// 0 by grid size and precision, 1 k_rows, 2 k_rows_zm), 1 the level-0
// FP64 true residual with its float copy (same variants), 2 the restriction
// of `level` to level + 1, 3 the prolongation of level + 1 to `level`, 4 the
// level-0 FP64 operator q = A z (rows variants).
double Solver::debug_time_stage(int stage, int l, int variant, int reps)
{
    if (l < 0 || l >= (int)L.size() || reps < 1 || stage < 0 || stage > 4 || variant < 0 || variant > 2)
        throw Error(P2_ERR_ARG, "bad stage, level, variant or repetition count");
    if ((stage == 2 || stage == 3) && l + 1 >= (int)L.size()) throw Error(P2_ERR_ARG, "no coarser level");
    if (!nodes_ready) throw Error(P2_ERR_STATE, "no node fields");
    const size_t flush_bytes = (size_t)256 << 20;
    void *flush = nullptr;
    P2_CUDA_TRY(cudaMalloc(&flush, flush_bytes));
    struct Free { void *p; ~Free() { if (p) cudaFree(p); } } hold{flush};
    const int saved = dbg_rows_variant;
    dbg_rows_variant = variant;
    double total = 0;
    try {
        for (int r = 0; r < reps; r++) {
            P2_CUDA_TRY(cudaMemsetAsync(flush, r & 0xff, flush_bytes, st));
            P2_CUDA_TRY(cudaEventRecord(ev[5], st));
            const bool f32 = prm.precision == 0;
            if (stage == 0) {
                if (f32) level_residual<float>(l);
                else level_residual<double>(l);
            } else if (stage == 1) {
                rows0(gx, gr, f32 ? &L[0].r32 : nullptr, 0);
            } else if (stage == 4) {
                rows0(Z[0], Q[0], nullptr, 1);
            } else if (stage == 2) {
                Level &F = L[l], &Cl = L[l + 1];
                if (f32)
                    pdl_launch(st, nblk(4L * Cl.n), kThreads, k_restrict_compat<float>, view<float>(l, false), F.r32,
                               view<float>(l + 1, false), Cl.b32, Cl.x32, F.tv, 1, Cl.compat_vol, rpartial, rticket,
                               scal);
                else
                    pdl_launch(st, nblk(4L * Cl.n), kThreads, k_restrict_compat<double>, view<double>(l, false),
                               F.r64, view<double>(l + 1, false), Cl.b64, Cl.x64, F.tv, 1, Cl.compat_vol, rpartial,
                               rticket, scal);
            } else {
                Level &F = L[l], &Cl = L[l + 1];
                if (f32)
                    pdl_launch(st, nblk(F.n), kThreads, k_prolong<float>, view<float>(l, false), F.x32,
                               view<float>(l + 1, false), Cl.x32, F.tv, (float)prm.p1koef, (float)prm.v1koef);
                else
                    pdl_launch(st, nblk(F.n), kThreads, k_prolong<double>, view<double>(l, false), F.x64,
                               view<double>(l + 1, false), Cl.x64, F.tv, prm.p1koef, prm.v1koef);
            }
            P2_CUDA_TRY(cudaEventRecord(ev[6], st));
            P2_CUDA_TRY(cudaEventSynchronize(ev[6]));
            P2_CUDA_TRY(cudaGetLastError());
            float ms = 0;
            P2_CUDA_TRY(cudaEventElapsedTime(&ms, ev[5], ev[6]));
            total += ms;
        }
    } catch (...) {
        dbg_rows_variant = saved;
        throw;
    }
    dbg_rows_variant = saved;
    return total / reps;
}

// nu, ro of every level (after ronurestrict), concatenated like the reference's nu[] / ro[]
// Average time of one colour pass of the cell-block smoother on level l.
double Solver::debug_time_smoother(int l, int passes)
{
    if (l < 0 || l >= (int)L.size() || passes < 2) throw Error(P2_ERR_ARG, "bad level or pass count");
    if (!bc_ready) throw Error(P2_ERR_STATE, "no level data");
    Level &Lv = L[l];
    factor_cells();
    // Each pass is timed alone after a 256 MB write (twice the 126 MB L2), so
    // the level's fields come from HBM as they do in a V-cycle whose other
    // levels and Krylov vectors have evicted them.
    const size_t flush_bytes = (size_t)256 << 20;
    void *flush = nullptr;
    P2_CUDA_TRY(cudaMalloc(&flush, flush_bytes));
    struct Free { void *p; ~Free() { if (p) cudaFree(p); } } hold{flush};
    double total = 0;
    cudaError_t err = cudaSuccess;
    for (int p = 0; p < passes && err == cudaSuccess; p++) {
        err = cudaMemsetAsync(flush, p & 0xff, flush_bytes, st);
        if (err == cudaSuccess) err = cudaEventRecord(ev[5], st);
        if (err != cudaSuccess) break;
        if (prm.precision == 0) {
            LevelView<float> V = view<float>(l, false);
            Vec4<float> x = Lv.x32, y = Lv.y32;
            y.c[0] = x.c[0];
            smoother_pass<float>(l, V, x.c[0], (p & 1) ? y : x, (p & 1) ? x : y, Lv.b32, p & 1);
        } else {
            LevelView<double> V = view<double>(l, false);
            Vec4<double> x = Lv.x64, y = Lv.y64;
            y.c[0] = x.c[0];
            smoother_pass<double>(l, V, x.c[0], (p & 1) ? y : x, (p & 1) ? x : y, Lv.b64, p & 1);
        }
        err = cudaEventRecord(ev[6], st);
        if (err == cudaSuccess) err = cudaEventSynchronize(ev[6]);
        if (err == cudaSuccess) err = cudaGetLastError();
        float t = 0;
        if (err == cudaSuccess) err = cudaEventElapsedTime(&t, ev[5], ev[6]);
        total += t;
    }
    hold.p = nullptr;
    cudaError_t ferr = cudaFree(flush);
    P2_CUDA_TRY(err);
    P2_CUDA_TRY(ferr);
    return total / passes;
}

void Solver::debug_level_fields(float *nu, float *ro)
{
    debug_prepare();
    for (auto &Lv : L) {
        P2_CUDA_TRY(cudaMemcpy(nu + Lv.off, Lv.nu, sizeof(float) * Lv.n, cudaMemcpyDeviceToHost));
        P2_CUDA_TRY(cudaMemcpy(ro + Lv.off, Lv.ro, sizeof(float) * Lv.n, cudaMemcpyDeviceToHost));
    }
}

template LevelView<float> Solver::view<float>(int, bool) const;
template LevelView<double> Solver::view<double>(int, bool) const;

}  // namespace p2
