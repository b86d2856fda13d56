/*
 * p2cuda — B200 (sm_100a) Stokes multigrid behind the Pardiso2 entry points.
 *
 * Plain C ABI: host pointers, sizes and a status code; no CUDA or torch
 * types cross this boundary.  Every array uses the reference's own layout:
 * node index n = m3*ynumy*xnumx + m1*ynumy + m2 (y fastest, then x, then z),
 * velocities vx/vy/vz as float, pressure pr as double, node fields
 * nu/ro/nxx/nxy/nxz/nyz as float, boundary tables bondm/bondv1/bondn1 as in
 * the reference's head3mg.c.
 *
 * Which reference interface each entry point replaces (paths relative to the
 * reference project):
 *   p2_set_grid        gridcheck() level tables, pardiso/load3mg.c:2011-2195
 *   p2_set_bc          bondm/bondv1/bondn1 tables, pardiso/head3mg.c:110-112
 *                      (filled by pardiso/in3mg.c:304-388)
 *   p2_set_nodes       the node fields vpiterate() reads, head3mg.c:95-96
 *   p2_stokes_solve    void vpiterate(int m0, int f0), pardiso/move3mgNew.c:1791
 *                      (prototype pardiso/head3mg.c:362); the coarsest
 *                      pardisomat() PARDISO solve, pardiso/gaus3mg_SerieMG.c:64
 *   p2_ronurecalc      void ronurecalc(void), pardiso/mark3mg.c:630
 *                      (prototype pardiso/head3mg.c:417); with power-law
 *                      rocks p2_ronurecalc_powerlaw
 *   p2_movemark        void movemark(void), pardiso/mark3mg.c:174
 *                      (prototype pardiso/head3mg.c:416)
 *   p2_effbulk_visc    void effbulkvisccalc(int), pardiso/mark3mg.c:2
 *                      (prototype pardiso/head3mg.c:435), mode 1
 *   p2_titerate        void titerate(int m0), pardiso/heat3mg.c:292
 *                      (called from pardiso/i3mg.c:148 when tempmod is set)
 * A C shim with the reference's own signatures on top of these calls is in
 * pardiso2_b200/csrc/move3mg_cuda.c.
 */
#ifndef P2CUDA_H
#define P2CUDA_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct p2_ctx p2_ctx;

typedef enum {
    P2_OK = 0,
    P2_ERR_ARG = 1,            /* bad argument or inconsistent sizes */
    P2_ERR_CUDA = 2,           /* a CUDA runtime call failed */
    P2_ERR_NOMEM = 3,          /* device allocation failed */
    P2_ERR_NOT_CONVERGED = 4,  /* iteration cap reached above the tolerance */
    P2_ERR_NAN = 5,            /* NaN/Inf in the residual */
    P2_ERR_SINGULAR = 6,       /* zero pivot in the coarsest LU */
    P2_ERR_STATE = 7,          /* call out of order (e.g. solve before set_grid) */
    P2_ERR_UNSUPPORTED = 8     /* periodic boundaries, p2koef != 0, open boundary rows */
} p2_status;

#define P2_MAX_LEVELS 12

/* The mode.t3c knobs vpiterate() reads (pardiso/mode.t3c:77-97) plus the
 * solver controls of this library. */
typedef struct {
    double p0koef, p1koef, p2koef, v0koef, v1koef; /* smoother / transfer scaling */
    double nubeg, nuend;                           /* viscosity clamp */
    double nukoef;                                 /* marker weight threshold (ronurecalc) */
    double gxkoef, gykoef, gzkoef;                 /* gravity components */
    double pinit;                                  /* pressure value in the pinned cell */
    int pxinit, pyinit, pzinit;                    /* pinned pressure cell */
    int viscmod;                                   /* 0 arithmetic, 1 geometric, 2 harmonic */
    int multinum;                                  /* coarse levels (levels = multinum + 1) */
    int npre[P2_MAX_LEVELS];                       /* multinnn[0][level] */
    int npost[P2_MAX_LEVELS];                      /* multinnn[1][level] */
    /* library controls */
    double tol;          /* relative residual target ||b-Ax||/||b|| (default 1e-8) */
    int max_iter;        /* outer iteration cap (default 200) */
    int precision;       /* 0: FP32 V-cycle in an FP64 outer loop; 1: FP64 V-cycle */
    int restart;         /* GCR restart length (default 16, at most 18) */
    double omega;        /* cell-block smoother damping (default 0.7) */
    int use_graphs;      /* capture the V-cycle in a CUDA graph (default 1) */
    int smoother;        /* cell-block smoother: 1 = exact 7x7 cell solve with the cell
                            factors computed once per solve and stored (default; one
                            launch per colour), 5 = the same with both colours of a sweep
                            in one launch on large levels (z-marching tiles in shared
                            memory; slower on B200 as measured, kept for comparison),
                            3 = the same solve factored on every sweep (no stored factors),
                            0 = diagonal velocity block (cheaper, weak at stiff inclusions),
                            2 = the exact cell solve evaluated row by row (slower; a cross-check) */
} p2_params;

typedef struct {
    int iterations;          /* outer (GCR) iterations */
    double rel_residual;     /* final ||b-Ax||/||b|| of the level-0 system, FP64 */
    double rel_residual0;    /* initial */
    double ms_total;         /* device time of the whole solve (CUDA events) */
    double ms_setup;         /* coarse viscosity, coarsest LU and inverse */
    double ms_vcycles;       /* preconditioner V-cycles */
    int status;
    long long kernels;       /* kernels this library launched during the solve */
} p2_solve_info;

/* Choice made by p2_autotune. */
typedef struct {
    int smoother;        /* chosen p2_params.smoother */
    int sweep_growth;    /* sweep growth per coarser level (pre and post), see sweep_max */
    double est_ms;       /* estimated device time of one solve to tol with the choice */
    double rate;         /* measured residual reduction per outer iteration */
    int candidates;      /* configurations tried */
    int trial_iters;     /* outer iterations per trial */
    int sweep_max;       /* most sweeps on any level: sweeps on level l >= 1 =
                            min(sweep_max, npre[0] * sweep_growth^l) with the configured npre[0] */
    int restart;         /* chosen GCR restart length (12 or the configured one, whichever
                            full solve of the chosen schedule was faster) */
    int sweeps0;         /* pre- (and post-) sweeps on level 0: npre[0], or half of it */
} p2_tune_info;

/* Fill p with the reference's defaults (mode.t3c) and this library's. */
void p2_default_params(p2_params *p);

p2_status p2_create(p2_ctx **ctx, int device);
void p2_destroy(p2_ctx *ctx);
/* Human-readable text of the last error on this context (never NULL). */
const char *p2_last_error(const p2_ctx *ctx);

/* Grid: node counts and gridlines; builds the multigrid levels exactly as
 * gridcheck() does.  Periodic flags must be 0 (P2_ERR_UNSUPPORTED otherwise). */
p2_status p2_set_grid(p2_ctx *ctx, long xnumx, long ynumy, long znumz, const double *gx, const double *gy,
                      const double *gz, int xperiodic, int yperiodic, int zperiodic, const p2_params *prm);

/* Boundary tables in the reference layout: bondm has 4*(sum of level nodes)
 * entries, bondv1 has 2*(bondnum+1) (const, koef), bondn1 has bondnum+1
 * (1 + coupled unknown index, 0 = none). */
p2_status p2_set_bc(p2_ctx *ctx, const int *bondm, long bondm_len, const float *bondv1, const int *bondn1,
                    long bondnum);

/* Level-0 node fields (host arrays of xnumx*ynumy*znumz floats). */
p2_status p2_set_nodes(p2_ctx *ctx, const float *nu, const float *ro, const float *nxx, const float *nxy,
                       const float *nxz, const float *nyz);

/* vpiterate(): solve the Stokes system; vx,vy,vz (float) and pr (double)
 * are the initial guess on entry (NULL = zero) and the solution on return,
 * with the pressure shifted so that cell (pxinit,pyinit,pzinit) holds pinit. */
p2_status p2_stokes_solve(p2_ctx *ctx, float *vx, float *vy, float *vz, double *pr, p2_solve_info *info);

/* Same solve on the resident node fields with the solution kept on the
 * device (no host transfers); read it back with p2_get_solution. */
p2_status p2_stokes_solve_resident(p2_ctx *ctx, p2_solve_info *info);

/* Batched solves (no counterpart in the reference, which solves one model per
 * process): p2_stokes_solve_resident on each of count contexts at once.
 * Every context must hold its grid, boundary tables and node fields; each
 * has its own stream and graphs, so the device overlaps the instances'
 * kernels.  host_threads workers (0: one per context, at most the hardware
 * threads) take the contexts largest first.  infos[i] (may be null) gets
 * context i's result; *ms (may be null) the device time from the first
 * launch to the last result, measured with events on device 0 of the batch.
 * Returns the first failing status in context order, else P2_OK. */
p2_status p2_stokes_solve_batch(p2_ctx *const *ctxs, int count, int host_threads, p2_solve_info *infos, double *ms);
p2_status p2_get_solution(p2_ctx *ctx, double *vx, double *vy, double *vz, double *pr);

/* Smoother autotuner (no counterpart in the reference, whose sweep counts
 * come from mode.t3c multinnn): on the resident node fields, runs
 * trial_iters outer iterations from a zero guess with each candidate (full
 * or diagonal cell block, constant or doubling sweeps per coarser level, the
 * configured or half the sweeps on level 0), estimates each candidate's time
 * to p2_params.tol from its measured rate and time per iteration, keeps the
 * cheapest in this context's parameters, then picks the GCR restart length
 * (12 or the configured one) by two full solves.  Call it once per model
 * before the time loop. */
p2_status p2_autotune(p2_ctx *ctx, int trial_iters, p2_tune_info *info);

/* ronurecalc(): marker -> node viscosity/density interpolation.  Rock
 * viscosity is the per-type constant markn0 (pardiso/mark3mg.c:1479-1482;
 * types 0..20 with markn0 != markn1 are power-law rocks and need
 * p2_ronurecalc_powerlaw), density markro (densimod 0).
 * nu..nyz are in/out: nodes that receive no marker keep their input value,
 * then every viscosity is clamped to [nubeg, nuend], as in the reference.
 * The fields also become this context's resident node fields. */
p2_status p2_ronurecalc(p2_ctx *ctx, long nmark, const float *markx, const float *marky, const float *markz,
                        const signed char *markt, int nrock, const double *markn0, const double *markn1,
                        const double *markro, float *nu, float *ro, float *nxx, float *nxy, float *nxz,
                        float *nyz);

/* ronurecalc() with power-law rocks (viscalc, pardiso/mark3mg.c:1463-1498):
 * for a rock type t <= 20 with markn0[t] != markn1[t] a marker's viscosity is
 * marknu[t] * val1^((1 - markmm[t]) / markmm[t]) clamped to
 * [markn0[t], markn1[t]], val1 being the marker's strain-rate invariant (what
 * movemark / p2_movemark_strain leaves per marker); other types as in
 * p2_ronurecalc.  The power is the device's pow, whose last-place rounding
 * can differ from the host C library's, so node fields of power-law markers
 * agree with the reference's to a few units in the last place of a float.
 * The reference also sets marke to 1e-20 where it is 0 for the markers it
 * interpolates; that array is the caller's and is not touched here. */
p2_status p2_ronurecalc_powerlaw(p2_ctx *ctx, long nmark, const float *markx, const float *marky,
                                 const float *markz, const signed char *markt, int nrock, const double *markn0,
                                 const double *markn1, const double *markro, const double *marknu,
                                 const double *markmm, const double *val1, float *nu, float *ro, float *nxx,
                                 float *nxy, float *nxz, float *nyz);

/* Same interpolation on markers already resident on the device (see
 * p2_upload_markers), writing the resident node fields only. */
p2_status p2_upload_markers(p2_ctx *ctx, long nmark, const float *markx, const float *marky, const float *markz,
                            const signed char *markt, int nrock, const double *markn0, const double *markn1,
                            const double *markro);
p2_status p2_ronurecalc_resident(p2_ctx *ctx, double *ms);
p2_status p2_get_nodes(p2_ctx *ctx, float *nu, float *ro, float *nxx, float *nxy, float *nxz, float *nyz);

/* movemark(): marker advection over one time step, pardiso/mark3mg.c:174
 * (prototype pardiso/head3mg.c:416): markmod 2 is the fourth-order
 * Runge-Kutta branch, markmod 1 the single-velocity one, with the velocity at
 * a point interpolated from the staggered
 * vx, vy, vz nodes as vxyzcalc1 (mark3mg.c:2963) does; non-periodic boxes.
 * Markers are moved when inside the box or, unless outgrid is 1, when their
 * type is below 50 or at least 100; outgrid 2 keeps the motion of markers
 * outside the box orthogonal to the wall.  Positions come out bit-identical
 * to the reference's.  Not reproduced: the strain-rate side outputs (val1,
 * marke: p2_movemark_strain below), the temperature reset (markk = 0) of
 * markers that leave the box, and the water/melt moves that the reference
 * has switched off.
 *   p2_movemark: vx, vy, vz host arrays (float, node layout) and markers in/out;
 *   p2_movemark_resident: the resident markers (p2_upload_markers) with the
 *   solution of the last resident solve; read them with p2_get_markers. */
p2_status p2_movemark(p2_ctx *ctx, double timestep, int markmod, int outgrid, const float *vx, const float *vy, const float *vz,
                      long nmark, float *markx, float *marky, float *markz, const signed char *markt);
p2_status p2_movemark_resident(p2_ctx *ctx, double timestep, int markmod, int outgrid, double *ms);
/* p2_movemark with movemark's strain-rate outputs (mark3mg.c:218-220, 358-410,
 * 488): val1[m] (double) = the second invariant
 * sqrt(0.5 (exx^2 + eyy^2 + ezz^2) + exy^2 + exz^2 + eyz^2) of the strain
 * rate at marker m before the move, interpolated from the node fields
 * exx..eyz as epscalc1 (mark3mg.c:3244) does, written for the markers that
 * move; for markers with marke > 0 the brittle strain marke (float, in/out)
 * grows by timestep times the Runge-Kutta average of the invariant over the
 * four stage points (markers of type < 100).  The invariant is taken with a
 * correctly rounded square root where the reference calls pow(x, 0.5): the
 * two agree to within one unit in the last place.  In the single-velocity
 * branch (markmod 1) the reference adds an average left from an earlier
 * marker; here the marker's own invariant is used. */
p2_status p2_movemark_strain(p2_ctx *ctx, double timestep, int markmod, int outgrid, const float *vx,
                             const float *vy, const float *vz, const float *exx, const float *eyy, const float *ezz,
                             const float *exy, const float *exz, const float *eyz, long nmark, float *markx,
                             float *marky, float *markz, const signed char *markt, double *val1, float *marke);
p2_status p2_get_markers(p2_ctx *ctx, float *markx, float *marky, float *markz);

/* The post-solve fields of vpiterate (pardiso/move3mgNew.c:2908-3038):
 * deviatoric stresses sxx..syz and strain rates exx..eyz on level 0 from the
 * last solution's velocities rounded to float (what p2_stokes_solve returns)
 * and the resident node viscosities clamped to [nubeg, nuend], bit-identical
 * to the reference's value-mode stencils (sxxcalc .. syzcalc, ynval = 0).
 * Arrays are in/out host arrays in the node layout: positions the reference
 * does not write keep their values; a null pointer skips that field.
 * vrange (may be null) receives {min vx, max vx, min vy, max vy, min vz,
 * max vz} over the valid velocity positions, from which vpiterate limits the
 * marker time step (move3mgNew.c:3293-3316). */
p2_status p2_stress_strain(p2_ctx *ctx, float *sxx, float *syy, float *szz, float *sxy, float *sxz, float *syz,
                           float *exx, float *eyy, float *ezz, float *exy, float *exz, float *eyz, double vrange[6]);

/* Effective bulk viscosity diagnostics of a solution: effbulkvisccalc(1)
 * (pardiso/mark3mg.c:2-150; prototype pardiso/head3mg.c:435).  Over the
 * level-0 nodes with ro > 1500 and every index > 0: the averages of the
 * strain-rate and stress second invariants of the cell behind the node
 * (eiin, siin; shear terms averaged over the cell's four edges of each
 * orientation), of the visco-plastic strain-rate invariant from the stresses
 * (eiivp), of the dissipation (hsn) and of nxx * eiin (tau2), the harmonic
 * mean of nxx (nubulkn), nubulk1..4 formed from them, and the averages of the
 * twelve tensor components (exx eyy ezz exy exz eyz sxx syy szz sxy sxz syz)
 * over inclusion nodes (ro > 3850) and matrix nodes.  Inputs are host arrays
 * in the node layout, as vpiterate / p2_stress_strain leave them.  Per-node
 * values follow the reference's float/double operations; the sums run in a
 * different (fixed) order, so results agree to about 1e-12 relative. */
typedef struct {
    double eiin, siin, eiivp, tau2, hsn, nubulkn;
    double nubulk1, nubulk2, nubulk3, nubulk4;
    double matrix[12], incl[12];
    long numtot, nummat, numinc;
} p2_effbulk;
p2_status p2_effbulk_visc(p2_ctx *ctx, const float *ro, const float *nxx, const float *nxy, const float *nxz,
                          const float *nyz, const float *exx, const float *eyy, const float *ezz, const float *exy,
                          const float *exz, const float *eyz, const float *sxx, const float *syy, const float *szz,
                          const float *sxy, const float *sxz, const float *syz, p2_effbulk *out);

/* titerate() (pardiso/heat3mg.c:292; prototype pardiso/head3mg.c:386): one
 * thermal step of `timestep` seconds on the level-0 temperature tk.
 *   T boundary rows first go in through p2_heat_set_bc: bondm in the
 *   reference layout, whose rows for the temperature start at 8 * nodenum
 *   (bondm[8*nodenum + u] for the node u of every level, in3mg.c:367-383),
 *   bondm_len >= 8 * nodenum + (sum of level nodes).  Every node on a wall of
 *   every level needs a T boundary row; chains of copy rows are followed.
 *   The step: heat sources ht (+ adiabatic heating with adiabyn 1 or 2 from
 *   vx, vy, vz, gravity of p2_params, and pr; + shear heating with frictyn 1
 *   from the twelve float fields sxx syy szz sxy sxz syz exx eyy ezz exy exz
 *   eyz) give the right-hand side and the sub-step limit maxtkstep / max
 *   |dT/dt|; each sub-step solves the implicit conduction rows with V-cycles
 *   on levels 0..multinumt (multittt[0][l] pre-sweeps, multittt[1][l] sweeps
 *   on the way up, multicyct cycles between error checks) until the RMS error
 *   of the rows times the sub-step is at most heatmin (at most max_cycles
 *   checks per sub-step; 0 = 10000; P2_OK with converged = 0 when reached).
 *   Then the markers (optional, nmark 0 skips them): types 50..99 take the
 *   node temperature, types below 50 the numerical-diffusion update of
 *   markk (heatdif, tdeep, zdeep), as heat3mg.c:641-829 does.
 *   tk and markk are updated in place; kt, cp, ro, ht, et are level-0 float
 *   fields (ro of the node layout, as ronurecalc writes it).
 *   The smoother is Gauss-Seidel in two colours (the reference sweeps the
 *   rows in order), so the iterates differ and the temperatures agree with
 *   the reference's to the tolerance heatmin sets. */
typedef struct {
    double maxtkstep;      /* K per sub-step */
    double heatmin;        /* HEATMIN, K */
    double t0koef, t1koef; /* smoother damping, prolongation factor */
    double heatdif;        /* numerical diffusion of marker temperatures */
    double tdeep, zdeep;   /* temperature of markers arriving below zdeep */
    int multinumt, multicyct;
    int multittt[2][P2_MAX_LEVELS];
    int frictyn, adiabyn;
    int max_cycles;
} p2_heat_params;
typedef struct {
    double tktimestep;     /* sub-step limit (1e30 when no node heats) */
    double maxtkrate;      /* max |dT/dt| of the right-hand side, K/s */
    int substeps;          /* thermal sub-steps taken */
    int cycles;            /* error checks, all sub-steps */
    int converged;         /* 1 when every sub-step reached heatmin */
    double heatsum;        /* RMS error after the last check, K */
    double mintk, maxtk;   /* temperature range after the step */
    double ms_total;       /* device time of the call, transfers included */
    long long kernels;     /* kernel launches */
} p2_heat_info;
void p2_default_heat_params(p2_heat_params *hp);
p2_status p2_heat_set_bc(p2_ctx *ctx, const int *bondm, long bondm_len, const float *bondv1, const int *bondn1,
                         long bondnum);
p2_status p2_titerate(p2_ctx *ctx, const p2_heat_params *hp, double timestep, float *tk, const float *kt,
                      const float *cp, const float *ro, const float *ht, const float *et, const float *vx,
                      const float *vy, const float *vz, const double *pr, const float *const *stress_strain,
                      long marknum, const float *markx, const float *marky, const float *markz,
                      const signed char *markt, float *markk, p2_heat_info *info);

/* The reference's binary model file (.prn), the branch of loader() and
 * saver() that needs no HDF5: pardiso/load3mg.c:745-905 (read) and
 * 1298-1443 (write).  Host code only (no device, no context).  The file holds
 * the writer's sizeof(int/long/float/double) in its first four bytes; a file
 * written with other sizes is refused, as the reference refuses it.  Arrays
 * keep the file's layout; p2_prn_read_header gives the sizes to allocate. */
typedef struct {
    long xnumx, ynumy, znumz;   /* nodes per axis */
    long mnumx, mnumy, mnumz;   /* markers per cell (the generator's counts) */
    double xsize, ysize, zsize;
    long pxinit, pyinit, pzinit;
    double pinit, gxkoef, gykoef, gzkoef;
    int rocknum;
    long bondnum, marknum;
    int cycle;                  /* the saver's cycle number n0 */
    double timesum_years;       /* timesum / 3.15576e7 as stored; the reference multiplies it back */
    double gridcur, gridtot;
} p2_prn_header;
typedef struct {
    double *rocks;         /* 24 * rocknum: markn0 markn1 marks0 marks1 marknu markdh markdv markss
                              markmm markll marka0 marka1 markb0 markb1 marke0 marke1 markro markbb
                              markaa markcp markkt markkf markkp markht, one table after another */
    float *nodes;          /* 11 per node (node order of the grid): pr vx vy vz ro nu tk cp et kt ht */
    float *gx, *gy, *gz;   /* gridlines (float in the file) */
    long *bond_index;      /* bondnum: the bondm index of the row (4 * node + unknown, or
                              8 * nodenum + node for a temperature row) */
    long *bond_row;        /* bondnum: the row number (the value of bondm there) */
    float *bond_value;     /* 2 * bondnum: bondv1 const, koef */
    long *bond_target;     /* bondnum: bondn1 of the row (1 + coupled unknown, 0 none) */
    float *markers;        /* 7 per marker: x y z markk markw markd marke */
    signed char *markt;    /* marknum types */
} p2_prn_data;
p2_status p2_prn_read_header(const char *path, p2_prn_header *h, char *err, long errlen);
p2_status p2_prn_read(const char *path, const p2_prn_header *h, const p2_prn_data *d, char *err, long errlen);
p2_status p2_prn_write(const char *path, const p2_prn_header *h, const p2_prn_data *d, char *err, long errlen);

/* The p2_ronurecalc interpolation for callers that cannot allocate device
 * memory: a host code whose device memory is all handed out by its own pool
 * at start-up, or one that cannot take the device-wide synchronisation that
 * cudaMalloc/cudaFree imply inside its time loop.  This entry point has no
 * counterpart in the reference.  It needs no p2_ctx and allocates nothing:
 * its scratch is one fixed 9.1 MiB device array inside this library, which
 * every GPU that loads the library holds until the process exits.
 *   Limits: at most 262144 markers, 131072 cells and 1024 gridlines per axis;
 *   larger sizes return P2_ERR_ARG and a message naming the limit.
 *   Arrays: gridlines, params (viscmod, nukoef, nubeg, nuend are read) and the
 *   rock tables are host arrays; markx..markt and nu..nyz are device arrays
 *   on the current device (nu..nyz of nx*ny*nz floats, in/out as in
 *   p2_ronurecalc).  Work runs on `stream` (a cudaStream_t; NULL = default).
 *   The call waits once for the stream (a check of the marker types) and
 *   returns with the node pass queued on it.
 *   Rock types 0..20 with markn0 != markn1 (power law) return
 *   P2_ERR_UNSUPPORTED; types above 20 take markn0, as p2_ronurecalc does.
 *   The first call on a device (and the first after a cudaDeviceReset, which
 *   unloads the array) looks up the scratch array's device address with that
 *   device current; make that first call before any stream capture begins.
 *   All calls share the one array: calls whose work overlaps on the GPU
 *   (different streams or host threads without ordering) race, so serialise
 *   them (one stream, or ordering by the caller).
 *   On an error, a message is written to err (errlen bytes; may be NULL). */
p2_status p2_ronurecalc_noalloc(int nx, int ny, int nz, const double *gx, const double *gy, const double *gz,
                                const p2_params *prm, int nrock, const double *markn0, const double *markn1,
                                const double *markro, long nmark, const float *markx, const float *marky,
                                const float *markz, const signed char *markt, float *nu, float *ro, float *nxx,
                                float *nxy, float *nxz, float *nyz, void *stream, char *err, long errlen);

/* Test hooks (no counterpart in the reference; they expose single stages so
 * parity tests can compare them with the reference's own functions).  Vectors
 * are FP64, interleaved [P,Vx,Vy,Vz] per node of the given level (the layout
 * of the reference's sol0/fre0/fre1 slices); the node fields must be set. */
/* y = A x with the level operator (move3mgNew.c:796-1576 rows, boundary rows
 * x - koef x_t, identity on non-unknown positions and on the pinned cell). */
p2_status p2_debug_apply(p2_ctx *ctx, int level, const double *x, double *y);
/* vprestrict (move3mgNew.c:3965) of a fine residual onto coarse_level;
 * compat != 0 adds the continuity compatibility shift of the V-cycle. */
p2_status p2_debug_restrict(p2_ctx *ctx, int coarse_level, const double *fine_res, double *coarse_rhs, int compat);
/* vpprolong (move3mgNew.c:3534): fine_x += P coarse_x. */
p2_status p2_debug_prolong(p2_ctx *ctx, int coarse_level, const double *coarse_x, double *fine_x);
/* nu, ro of all levels after ronurestrict (move3mgNew.c:3386), concatenated
 * with the level offsets mgp (float[sum of level nodes] each). */
p2_status p2_debug_level_fields(p2_ctx *ctx, float *nu, float *ro);
/* Average device time (CUDA events on the library's stream) of one colour
 * pass of the cell-block smoother on `level` (FP32 when precision is 0),
 * over `passes` passes on the state left by the last solve, each timed alone
 * after a 256 MB write that evicts the level from L2 (allocated and freed by
 * this call). */
p2_status p2_debug_time_smoother(p2_ctx *ctx, int level, int passes, double *ms_per_pass);
/* `sweeps` sweeps of the configured smoother on `level` as the V-cycle runs
 * them (in its precision; fused sweeps where the level allows), applied to the
 * state x (in/out) for the right-hand side b, both interleaved as above. */
p2_status p2_debug_smooth(p2_ctx *ctx, int level, int sweeps, const double *b, double *x);
/* Average device time of one smoother sweep on `level` as the V-cycle runs it
 * (both colours with their boundary rows), `sweeps` sweeps timed together
 * after a 256 MB write that evicts L2, mean of 10 repetitions. */
p2_status p2_debug_time_sweep(p2_ctx *ctx, int level, int sweeps, double *ms_per_sweep);
/* Average device time of one stage of the solve on the state left by the
 * last solve, each of `reps` repetitions timed alone after a 256 MB write
 * that evicts L2: stage 0 the V-cycle residual of `level`, 1 the level-0
 * FP64 true residual, 2 the restriction of `level` to level + 1, 3 the
 * prolongation of level + 1 to `level`, 4 the level-0 FP64 operator.
 * `variant` selects the kernel of the operator rows (0 by the level's grid
 * size and the precision, 1 one thread per node from global memory, 2
 * z-marching planes in shared memory). */
p2_status p2_debug_time_stage(p2_ctx *ctx, int stage, int level, int variant, int reps, double *ms);
/* Kernel of the operator rows for the following calls of this context
 * (variant as for p2_debug_time_stage; 0, the default, chooses by the
 * level's grid size and the precision).  Captured V-cycle graphs are dropped
 * so that solves use it too. */
p2_status p2_debug_rows_kernel(p2_ctx *ctx, int variant);
/* x = one preconditioning V-cycle (the solver's precision, exact coarsest
 * solve) applied from zero to the level-0 right-hand side b, both
 * interleaved [P, Vx, Vy, Vz] per node of level 0. */
p2_status p2_debug_vcycle(p2_ctx *ctx, const double *b, double *x);

#ifdef __cplusplus
}
#endif
#endif
