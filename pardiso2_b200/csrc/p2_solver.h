// Solver state of the p2cuda library (one per p2_ctx, one device, one stream).
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <memory>
#include <vector>

#include "p2_internal.cuh"

namespace p2 {

struct DeviceArena {
    std::vector<void *> ptrs;
    size_t guard = 0;  // zero-filled bytes appended to every allocation
    void *alloc(size_t bytes);
    void release();
};

struct HostAxis {
    std::vector<int> lo;
    std::vector<double> w0, w1;
    std::vector<int> ptr, idx;
    std::vector<double> w;
};

struct Level {
    int nx = 0, ny = 0, nz = 0, n = 0;
    long off = 0;                 // node offset of the level (mgp)
    std::vector<double> g[3];     // gridlines mggx/mggy/mggz
    int tabstride = 0;
    double *tabd = nullptr;       // 12 spacing tables (ih, ihc, ihe, ihv per axis), FP64
    float *tabf = nullptr;        // same in FP32
    TransferView tv{};            // this level -> next coarser level
    AxisMap ronu[3]{};            // ronurestrict weights
    float *nu = nullptr, *ro = nullptr;
    float *ec = nullptr, *exy = nullptr, *exz = nullptr, *eyz = nullptr;
    uint8_t *bcm = nullptr;
    std::vector<uint8_t> h_bcm;
    int pin = -1;
    double pinval = 0;
    double compat_vol = 0;        // total volume of the non-boundary pressure cells
    // stored cell factors of the full cell-block smoother: per colour
    // kBlkEntries x blk_stride values of the V-cycle's type, entry-major
    void *blk = nullptr;
    long blk_stride = 0;
    // fused sweeps (k_vanka_sweep): every boundary row's resolved target
    // within one node; the rows by node (first row per node, row order)
    bool fuse_ok = false;
    int *sw_first = nullptr, *sw_order = nullptr;
    // boundary rows sorted by copy-chain depth
    int nbc = 0;
    std::vector<int> bc_groups;
    int *bu = nullptr, *bt = nullptr, *bnext = nullptr;  // bnext: row owning the target, or -1
    float *bk = nullptr, *bconst = nullptr;
    std::vector<int> h_bu, h_rt;  // unknown, resolved (non-boundary) target
    std::vector<double> h_rk;     // resolved coefficient
    // vectors: x (and y, the second velocity buffer of the smoother), b, r
    Vec4<float> x32, y32, b32, r32;
    Vec4<double> x64, y64, b64, r64;
};

struct GraphSlot {
    cudaGraphExec_t exec = nullptr;
    long long kernels = 0;  // kernel nodes replayed per launch
};

struct RawFields {
    float *nu = nullptr, *ro = nullptr, *nxx = nullptr, *nxy = nullptr, *nxz = nullptr, *nyz = nullptr;
};

// heat equation state (p2_heat.cu)
struct HeatLevel {
    const double *g[3] = {nullptr, nullptr, nullptr};  // gridlines
    int *bci = nullptr;                   // per node: 0 heat row, q + 1 boundary row q
    int nbc = 0;
    int *bu = nullptr, *bt = nullptr;     // boundary row: unknown, resolved heat-row target (-1 none)
    double *bk = nullptr, *bconst = nullptr;
    unsigned char *bpass = nullptr;       // colour pass that sets the row (after its target's)
    float *kt = nullptr, *cp = nullptr, *ro = nullptr;  // coarse levels (level 0: HeatState)
    double *x = nullptr, *b = nullptr, *r = nullptr, *a = nullptr;  // b, a in colour order
    long nh = 0;                          // nodes per colour slot range
    AxisMap map[3]{};                     // this level -> next coarser level
};

struct HeatState {
    bool ready = false;
    std::vector<HeatLevel> lv;
    float *tk = nullptr, *tk0 = nullptr, *tk1 = nullptr, *tk2 = nullptr;
    float *kt = nullptr, *cp = nullptr, *ro = nullptr, *ht = nullptr, *et = nullptr;
    float *vel[3] = {nullptr, nullptr, nullptr};
    double *pr = nullptr;
    float *se[12] = {};
    int nblk = 0;
    double *partial = nullptr, *scal = nullptr, *S0 = nullptr, *S1 = nullptr;
    double *host = nullptr;
    std::shared_ptr<double> host_owner;
    long mcap = 0;
    float *mx = nullptr, *my = nullptr, *mz = nullptr, *mk = nullptr;
    signed char *mt = nullptr;
    cudaStream_t mst = nullptr;  // marker copies, overlapped with the sub-steps
    cudaEvent_t mev = nullptr;
    std::shared_ptr<CUstream_st> mst_owner;
    std::shared_ptr<CUevent_st> mev_owner;
    long long kernels = 0;
};

class Solver {
  public:
    explicit Solver(int device);
    ~Solver();

    void set_grid(long nx, long ny, long nz, const double *gx, const double *gy, const double *gz,
                  const p2_params &p);
    void set_bc(const int *bondm, long bondm_len, const float *bondv1, const int *bondn1, long bondnum);
    void upload_nodes(const float *nu, const float *ro, const float *nxx, const float *nxy, const float *nxz,
                      const float *nyz);
    void set_initial(const float *vx, const float *vy, const float *vz, const double *pr);
    p2_solve_info solve();
    void get_solution(double *vx, double *vy, double *vz, double *pr);
    void get_solution_f32(float *vx, float *vy, float *vz, double *pr);

    void upload_markers(long nmark, const float *mx, const float *my, const float *mz, const signed char *mt,
                        int nrock, const double *n0, const double *n1, const double *rho,
                        const double *marknu = nullptr, const double *markmm = nullptr, const double *val1 = nullptr);
    void ronurecalc_device();
    void movemark_host(double dt, int markmod, int outgrid, const float *vx, const float *vy, const float *vz, long nmark,
                       float *mx, float *my, float *mz, const signed char *mt);
    void movemark_device(double dt, int markmod, int outgrid);
    void movemark_strain_host(double dt, int markmod, int outgrid, const float *vx, const float *vy, const float *vz,
                              const float *const e[6], long nmark, float *mx, float *my, float *mz,
                              const signed char *mt, double *val1, float *marke);
    void get_markers(float *mx, float *my, float *mz);
    void stress_strain(float *const s[6], float *const e[6], double vrange[6]);
    void heat_set_bc(const int *bondm, long bondm_len, const float *bondv1, const int *bondn1, long bondnum);
    p2_heat_info titerate(const p2_heat_params &hp, double timestep, float *tk, const float *kt, const float *cp,
                          const float *ro, const float *ht, const float *et, const float *vx, const float *vy,
                          const float *vz, const double *pr, const float *const *se, long nmark, const float *mx,
                          const float *my, const float *mz, const signed char *mt, float *markk);
    void effbulk(const float *ro, const float *nxx, const float *nxy, const float *nxz, const float *nyz,
                 const float *const e[6], const float *const s[6], p2_effbulk *res);

    // test hooks (FP64, interleaved [P,Vx,Vy,Vz] per node)
    void debug_apply(int l, const double *x, double *y);
    void debug_restrict(int lc, const double *fine_res, double *coarse_rhs, int compat);
    void debug_prolong(int lc, const double *coarse_x, double *fine_x);
    void debug_level_fields(float *nu, float *ro);
    double debug_time_smoother(int level, int passes);
    double debug_time_sweep(int level, int sweeps);
    double debug_time_stage(int stage, int level, int variant, int reps);
    int dbg_rows_variant = 0;     // kernel of the operator rows (launch_rows), 0 = by grid size and precision
    void drop_graphs_public() { drop_graphs(); }
    void debug_smooth(int level, int sweeps, const double *b, double *x);
    void debug_vcycle(const double *b, double *x);
    p2_tune_info autotune(int trial_iters);
    bool verbose = false;

    int dev;
    cudaStream_t st = nullptr;
    cudaEvent_t ev[8];
    p2_params prm{};
    std::vector<Level> L;
    long total_nodes = 0;
    bool grid_ready = false, bc_ready = false, nodes_ready = false, markers_ready = false, solution_ready = false;
    RawFields f0;

    // markers
    long nmk = 0;
    float *mk_x = nullptr, *mk_y = nullptr, *mk_z = nullptr;
    signed char *mk_t = nullptr;
    unsigned *mk_key[2] = {nullptr, nullptr}, *mk_val[2] = {nullptr, nullptr}, *mk_hist = nullptr;
    unsigned *mk_scan = nullptr;  // per-block totals of the histogram scan
    int mk_cur = 0;
    float4 *mk_sorted = nullptr;
    int *cell_start = nullptr, *cell_end = nullptr;
    double *rock_f = nullptr, *rock_ro = nullptr;
    double *rock_pl = nullptr, *mk_val1 = nullptr;  // power-law table per type, val1 per marker
    double *d_g[3] = {nullptr, nullptr, nullptr};
    float *mk_nodes[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    // marker advection: float velocities and host-path marker buffers
    float *mv_vel[3] = {nullptr, nullptr, nullptr};
    float *mv_pos[3] = {nullptr, nullptr, nullptr};
    signed char *mv_type = nullptr;
    long mv_cap = 0;
    float *mv_e[6] = {};             // strain-rate fields for the strain-rate outputs of movemark
    double *mv_val1 = nullptr;       // per marker
    float *mv_marke = nullptr;
    // post-solve stress / strain-rate fields and velocity ranges
    float *post_out[12] = {};
    float *post_partial = nullptr;
    double *post_range = nullptr;
    float *bulk_in[17] = {};         // effbulk inputs
    double *bulk_partial = nullptr, *bulk_out = nullptr;

  private:
    template <typename T>
    LevelView<T> view(int l, bool raw_clamp) const;
    void drop_graphs();
    void allocate_work();
    void build_coarse_index();
    void coarse_setup();
    template <typename T>
    void coarse_solve(Vec4<T> &b, Vec4<T> &x);
    template <typename T>
    void bc_set(int l, Vec4<T> &x, Vec4<T> &b);
    template <typename T>
    void smooth(int l, int sweeps);
    template <typename T>
    void smoother_pass(int l, const LevelView<T> &V, T *P, Vec4<T> &vin, Vec4<T> &vout, Vec4<T> &b, int col);
    bool use_fused(int l) const;
    template <typename T>
    void sweep_fused(int l, const LevelView<T> &V, Vec4<T> &xin, Vec4<T> &xout, Vec4<T> &b);
    template <typename T>
    void factor_smoother();
    void factor_cells();
    template <typename T>
    void level_residual(int l);

    template <typename T>
    void vcycle();
    template <typename T>
    void run_vcycle_graph();
    template <typename T>
    void capture_vcycle_graph();
    void set_nodes_device();
    void dots_sync(const DotJobs &jobs);
    template <typename S>
    void rows0(const Vec4<S> &x, Vec4<double> &out, Vec4<float> *r32, int mode);
    void precondition();
    std::vector<cudaEvent_t> vc_ev;  // V-cycle timing events of a solve (reused)
    double *qq_dev = nullptr;        // (Q_j, Q_j) of the stored directions
    void debug_prepare();
    Grid3 grid3() const;
    void ensure_move_buffers(long nmark);
    void velocity_f32();

    void heat_smooth(int l, int sweeps, double t0koef);
    void heat_batch(const p2_heat_params &hp);

    DeviceArena arena, grid_arena, marker_arena, move_arena, post_arena, heat_arena, heat_mk_arena;
    HeatState heat;
    std::array<GraphSlot, 2> graphs;
    // Coarsest LU + inverse on a second stream, overlapped with the first
    // lu_overlap_iters outer iterations, whose V-cycles smooth the coarsest level.
    std::array<GraphSlot, 2> graphs_apx;
    cudaStream_t st_lu = nullptr;
    cudaEvent_t ev_lu = nullptr;
    bool lu_pending = false;
    int coarse_mode = 0;  // 0: exact coarsest solve (inverse), 1: smoothing sweeps
    int lu_overlap_iters = 0;
    void lu_finish();
    template <typename T>
    void coarse_approx(Vec4<T> &b, Vec4<T> &x);
    LuGraph lu_graph;  // coarsest LU + inverse launch sequence
    int restart = 8;
    Vec4<double> gx, gb, gr;
    std::vector<Vec4<double>> Z, Q;
    double *partial = nullptr, *dots = nullptr, *scal = nullptr;
    double *rpartial = nullptr;   // per-block partial sums of the fused restriction
    unsigned *rticket = nullptr;  // its last-block ticket (returns to zero)
    double *hdots_raw = nullptr;
    std::shared_ptr<double> hdots;
    // coarsest level
    int nF = 0;
    std::vector<int> coarse_col;
    int *d_free = nullptr, *d_colmap = nullptr, *d_crt = nullptr;
    float *d_crk = nullptr;
    double *A_c = nullptr, *Ainv64 = nullptr;
    float *Ainv32 = nullptr;
    int *d_ipiv = nullptr, *d_info = nullptr;
    double *probes = nullptr;
    int *d_bw = nullptr, *h_bw = nullptr;  // band of the coarsest operator (kl, ku)
    std::shared_ptr<int> h_bw_keep;
    double *cb64 = nullptr, *cx64 = nullptr;
    float *cb32 = nullptr, *cx32 = nullptr;
};

}  // namespace p2
