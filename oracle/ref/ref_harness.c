/*
 * Reference harness (TEST INFRASTRUCTURE ONLY — never linked by the product).
 *
 * Compiles the reference's own active unity build sources where they lie
 * (pardiso/i3mg.c:12-19 includes head3mg.c, load3mg.c, move3mgNew.c,
 * mark3mg.c, gaus3mg_SerieMG.c, heat3mg.c) and drives them through a small
 * C API so that Python tests can:
 *   - run the reference's marker->node interpolation ronurecalc()
 *     (pardiso/mark3mg.c:630-1133) on given markers,
 *   - run the reference's Stokes solve vpiterate() (pardiso/move3mgNew.c:1791)
 *     for its first (assembly + direct coarsest solve) iteration, then keep
 *     iterating with the reference's own gausmat4/vprestrict/vpprolong
 *     (move3mgNew.c:3854, 3965, 3534) exactly as the m2prn>0 branch of
 *     vpiterate does (move3mgNew.c:2709-2791), stopping on the true FP64
 *     relative residual ||fre1 - A sol0|| / ||fre1|| of the level-0 row store
 *     instead of the reference's RMS criterion (move3mgNew.c:3281).
 *
 * Two stand-ins are needed to compile: a type-only hdf5.h (stubs/hdf5.h;
 * the harness never calls loader()/saver()) and the PARDISO entry point
 * (pardiso/gaus3mg_SerieMG.c:170,185,198,216), implemented below on top of
 * the oracle's banded pivoted LU (../banded_lu.h).
 */
#define _GNU_SOURCE
#include <stdio.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>
#include <time.h>
#include <unistd.h>
#include <fcntl.h>
#include "hdf5.h"
#include "../banded_lu.h"

void PARDISO(void **pt, int *maxfct, int *mnum, int *mtype, int *phase, int *n,
             double *a, int *ia, int *ja, int *perm, int *nrhs, int *iparm,
             int *msglvl, double *b, double *x, int *error);

#include "head3mg.c"
#include "load3mg.c"
#ifdef P2REF_SHIM
/* drop-in variant: vpiterate()/ronurecalc()/movemark() come from move3mg_cuda.c (GPU) */
#define vpiterate vpiterate_cpu
#define ronurecalc ronurecalc_cpu
#define movemark movemark_cpu
#define effbulkvisccalc effbulkvisccalc_cpu
#endif
#include "move3mgNew.c"
#include "mark3mg.c"
#ifdef P2REF_SHIM
#undef vpiterate
#undef ronurecalc
#undef movemark
#undef effbulkvisccalc
#endif
#include "gaus3mg_SerieMG.c"
#ifdef P2REF_SHIM
#define titerate titerate_cpu
#endif
#include "heat3mg.c"
#ifdef P2REF_SHIM
#undef titerate
#include "move3mg_cuda.c"
#endif

/* ---------------------------------------------------------------------- */
/* PARDISO-ABI shim.  A factorisation is cached across calls with the same
 * matrix (the reference re-runs phases 11/22 on every pardisomat(0) call). */
static p2_csr_lu g_lu;
static int g_lu_valid = 0;
static long g_lu_n = 0;
static double *g_lu_a = NULL;
static int *g_lu_ia = NULL, *g_lu_ja = NULL;
static long g_lu_nnz = 0;
int p2ref_lu_factorizations = 0;

static int same_matrix(long n, const int *ia, const int *ja, const double *a)
{
    long nnz = ia[n] - 1;
    if (!g_lu_valid || n != g_lu_n || nnz != g_lu_nnz) return 0;
    if (memcmp(ia, g_lu_ia, sizeof(int) * (size_t)(n + 1))) return 0;
    if (memcmp(ja, g_lu_ja, sizeof(int) * (size_t)nnz)) return 0;
    if (memcmp(a, g_lu_a, sizeof(double) * (size_t)nnz)) return 0;
    return 1;
}

void PARDISO(void **pt, int *maxfct, int *mnum, int *mtype, int *phase, int *n,
             double *a, int *ia, int *ja, int *perm, int *nrhs, int *iparm,
             int *msglvl, double *b, double *x, int *error)
{
    long nn = *n;
    (void)pt; (void)maxfct; (void)mnum; (void)mtype; (void)perm; (void)nrhs; (void)msglvl;
    *error = 0;
    if (*phase == 11) return;
    if (*phase == 22) {
        if (same_matrix(nn, ia, ja, a)) return;
        if (g_lu_valid) p2_band_free(&g_lu.lu);
        free(g_lu_a); free(g_lu_ia); free(g_lu_ja);
        g_lu_nnz = ia[nn] - 1;
        g_lu_a = (double *)malloc(sizeof(double) * (size_t)g_lu_nnz);
        g_lu_ia = (int *)malloc(sizeof(int) * (size_t)(nn + 1));
        g_lu_ja = (int *)malloc(sizeof(int) * (size_t)g_lu_nnz);
        memcpy(g_lu_a, a, sizeof(double) * (size_t)g_lu_nnz);
        memcpy(g_lu_ia, ia, sizeof(int) * (size_t)(nn + 1));
        memcpy(g_lu_ja, ja, sizeof(int) * (size_t)g_lu_nnz);
        g_lu_n = nn;
        if (p2_csr_lu_factor(&g_lu, nn, g_lu_ia, g_lu_ja, g_lu_a)) *error = -4;
        g_lu_valid = 1;
        p2ref_lu_factorizations++;
        return;
    }
    if (*phase == 33) {
        p2_csr_lu_solve(&g_lu, b, x, iparm[7] > 0 ? iparm[7] : 0);
        return;
    }
    /* phase -1: keep the cached factorisation for reuse. */
}

/* ---------------------------------------------------------------------- */
static int g_quiet = 1;
static int saved_out = -1, saved_err = -1;

static void mute(void)
{
    int devnull;
    if (!g_quiet) return;
    fflush(stdout); fflush(stderr);
    devnull = open("/dev/null", O_WRONLY);
    saved_out = dup(1); saved_err = dup(2);
    dup2(devnull, 1); dup2(devnull, 2);
    close(devnull);
}

static void unmute(void)
{
    if (!g_quiet) return;
    fflush(stdout); fflush(stderr);
    dup2(saved_out, 1); dup2(saved_err, 2);
    close(saved_out); close(saved_err);
}

static char g_scratch[512];

void p2ref_set_quiet(int q) { g_quiet = q; }

/*
 * Set up grid, levels and storage.  gx/gy/gz are the fine gridlines.
 * Mirrors what in3mg.c:62-103 + loadconf do before a solve: sizes,
 * dynmemall(0), gridcheck() (load3mg.c:2011-2195), dynmemall(1,2).
 */
int p2ref_init(long nx, long ny, long nz, const double *ggx, const double *ggy,
               const double *ggz, int nlev, long nmark)
{
    long i;
    const char *base = getenv("TMPDIR");
    snprintf(g_scratch, sizeof(g_scratch), "%s/p2ref_XXXXXX", base ? base : "/tmp");
    if (!mkdtemp(g_scratch) || chdir(g_scratch)) return -1;

    xnumx = nx; ynumy = ny; znumz = nz;
    xsize = ggx[nx - 1] - ggx[0];
    ysize = ggy[ny - 1] - ggy[0];
    zsize = ggz[nz - 1] - ggz[0];
    multinum = nlev;
    marknum = nmark;
    nodenum = xnumx * ynumy * znumz;
    printmod = 0;
    mute();
    dynmemall(0);
    for (i = 0; i < nx; i++) gx[i] = ggx[i];
    for (i = 0; i < ny; i++) gy[i] = ggy[i];
    for (i = 0; i < nz; i++) gz[i] = ggz[i];
    gridcheck();
    dynmemall(1);
    dynmemall(2);
    unmute();
    /* markk (temperature), markd, markw are read and written by movemark()
     * (mark3mg.c:249, 494, 525-527) but dynmemall() never allocates them
     * (load3mg.c:2323-2334; only the visualiser's load3viz.c:2141 does), so
     * the stock program dereferences null pointers once a marker of type
     * < 100 leaves the box or a marker of type >= 100 exists.  The harness
     * gives them storage so that those branches can be exercised. */
    if (!markk) markk = (float *)calloc((size_t)marknum0, sizeof(float));
    if (!markd) markd = (float *)calloc((size_t)marknum0, sizeof(float));
    if (!markw) markw = (float *)calloc((size_t)marknum0, sizeof(float));
    {
        long mcmax = mgp[multinum] + mgn[multinum];
        memset(bondm, 0, sizeof(int) * (size_t)(mcmax + nodenum8));
        memset(sol0, 0, sizeof(double) * (size_t)(mcmax * 4));
        memset(sol1, 0, sizeof(double) * (size_t)(mcmax * 4));
        memset(fre0, 0, sizeof(double) * (size_t)(mcmax * 4));
        memset(fre1, 0, sizeof(double) * (size_t)(mcmax * 4));
        memset(num0, 0, sizeof(int) * (size_t)(mcmax * 4));
        memset(nu, 0, sizeof(float) * (size_t)nodenum * 2);
        memset(ro, 0, sizeof(float) * (size_t)nodenum * 2);
        memset(nd, 0, sizeof(float) * (size_t)nodenum * 2);
        memset(nxx, 0, sizeof(float) * (size_t)nodenum * 2);
        memset(nxy, 0, sizeof(float) * (size_t)nodenum * 2);
        memset(nxz, 0, sizeof(float) * (size_t)nodenum * 2);
        memset(nyz, 0, sizeof(float) * (size_t)nodenum * 2);
        memset(pr, 0, sizeof(double) * (size_t)nodenum);
        memset(vx, 0, sizeof(float) * (size_t)nodenum);
        memset(vy, 0, sizeof(float) * (size_t)nodenum);
        memset(vz, 0, sizeof(float) * (size_t)nodenum);
        if (marknum > 0) memset(marke, 0, sizeof(float) * (size_t)marknum);
        /* pardisomat() (gaus3mg_SerieMG.c:264-296) reads curs[]/bufvs[] that
         * dynmemall() mallocs without initialising: the reference relies on
         * fresh zero pages; a process that reuses heap memory must clear them. */
        {
            long nc = (long)mgn[multinum] * 4;
            int t, nt = 1;
#pragma omp parallel
            {
#pragma omp master
                nt = omp_get_num_threads();
            }
            memset(bufvs, 0, sizeof(double) * (size_t)nc);
            memset(curs, 0, sizeof(int) * (size_t)nc);
            memset(bufv0, 0, sizeof(double) * (size_t)nc);
            memset(cur0, 0, sizeof(int) * (size_t)nc);
            memset(ia, 0, sizeof(int) * (size_t)(nc + 1));
            memset(x, 0, sizeof(double) * (size_t)nc);
            memset(b, 0, sizeof(double) * (size_t)nc);
            memset(ja, 0, sizeof(int) * (size_t)mgn[multinum] * 57);
            memset(a, 0, sizeof(double) * (size_t)mgn[multinum] * 57);
            memset(bufv, 0, sizeof(double) * (size_t)(mcmax * 4));
            memset(lin0, 0, sizeof(int) * (size_t)(mcmax * 57));
            memset(pos0, 0, sizeof(int) * (size_t)(mcmax * 4));
            memset(val1, 0, sizeof(double) * (size_t)(mcmax * 57));
            for (t = 0; t < nt; t++) {
                memset(Sol0[t], 0, sizeof(double) * (size_t)(mcmax * 4));
                memset(Sol1[t], 0, sizeof(double) * (size_t)(mcmax * 4));
                memset(Nu[t], 0, sizeof(float) * (size_t)(mcmax * 4));
                memset(Ro[t], 0, sizeof(float) * (size_t)(mcmax * 4));
                memset(Nxx[t], 0, sizeof(float) * (size_t)nodenum * 2);
                memset(Nxy[t], 0, sizeof(float) * (size_t)nodenum * 2);
                memset(Nxz[t], 0, sizeof(float) * (size_t)nodenum * 2);
                memset(Nyz[t], 0, sizeof(float) * (size_t)nodenum * 2);
            }
        }
    }
    /* Fixed knobs of this harness (mode.t3c:77-97 equivalents set by caller). */
    xperiodic = yperiodic = zperiodic = 0;
    spheryn = 0;
    densimod = 0;
    timesum = 0; timebeg = 0; timeend = 1e30; velocitykf = 1.0;
    maxxystep = 1e30; timestep = 1e30;
    fl0cyc[0][2] = 1 << 30;   /* never switch multinum (move3mgNew.c:3271) */
    fl0cyc[0][3] = multinum;
    DIVVMAX = 0;
    numult = 1.0;
    return multinum;
}

void p2ref_levels(int *ox, int *oy, int *oz, int *op, int *on)
{
    int l;
    for (l = 0; l <= multinum; l++) {
        ox[l] = mgx[l]; oy[l] = mgy[l]; oz[l] = mgz[l]; op[l] = mgp[l]; on[l] = mgn[l];
    }
}

void p2ref_level_coords(int l, double *cx, double *cy, double *cz)
{
    int i;
    for (i = 0; i < mgx[l]; i++) cx[i] = mggx[l][i];
    for (i = 0; i < mgy[l]; i++) cy[i] = mggy[l][i];
    for (i = 0; i < mgz[l]; i++) cz[i] = mggz[l][i];
}

/*
 * dpar: p0koef p1koef p2koef v0koef v1koef nubeg nuend nukoef GX GY GZ pinit
 * ipar: viscmod pxinit pyinit pzinit multicyc
 * npre/npost: sweeps per level (multinnn[0][*], multinnn[1][*]).
 */
void p2ref_set_params(const double *dpar, const int *ipar, const int *npre, const int *npost)
{
    int l;
    p0koef = dpar[0]; p1koef = dpar[1]; p2koef = dpar[2]; v0koef = dpar[3]; v1koef = dpar[4];
    nubeg = dpar[5]; nuend = dpar[6]; nukoef = dpar[7];
    GXKOEF = dpar[8]; GYKOEF = dpar[9]; GZKOEF = dpar[10]; pinit = dpar[11];
    viscmod = ipar[0]; pxinit = ipar[1]; pyinit = ipar[2]; pzinit = ipar[3]; multicyc = ipar[4];
    for (l = 0; l <= multinum; l++) { multinnn[0][l] = npre[l]; multinnn[1][l] = npost[l]; }
}

/* BC tables in the reference layout (head3mg.c:110-112, in3mg.c:331-349). */
int p2ref_set_bc(const int *bm, long nb, const float *bv, const int *bn)
{
    long mcmax = mgp[multinum] + mgn[multinum], i;
    if (nb + 1 > MAXBON) return -1;
    for (i = 0; i < mcmax * 4; i++) bondm[i] = bm[i];
    for (i = 0; i <= nb; i++) { bondv1[i][0] = bv[2 * i]; bondv1[i][1] = bv[2 * i + 1]; bondn1[i] = bn[i]; }
    bondnum = nb;
    return 0;
}

void p2ref_set_rocks(int nrock, const double *n0, const double *n1, const double *rho)
{
    int i;
    rocknum = nrock;
    for (i = 0; i < nrock; i++) { markn0[i] = n0[i]; markn1[i] = n1[i]; markro[i] = rho[i]; marknu[i] = n0[i]; markmm[i] = 1.0; }
}

/* Power-law rheology parameters per rock type and the markers' val1. */
void p2ref_set_rheology(int nrock, const double *nu, const double *mm, const double *v1)
{
    long i;
    for (i = 0; i < nrock; i++) { marknu[i] = nu[i]; markmm[i] = mm[i]; }
    for (i = 0; i < marknum; i++) val1[i] = v1[i];
}

void p2ref_set_markers(const float *mx, const float *my, const float *mz, const signed char *mt)
{
    long i;
    for (i = 0; i < marknum; i++) { markx[i] = mx[i]; marky[i] = my[i]; markz[i] = mz[i]; markt[i] = (char)mt[i]; }
}

/* Level-0 node fields in/out (float, node layout m3*xynumxy+m1*ynumy+m2). */
void p2ref_set_nodes(const float *inu, const float *iro, const float *ixx, const float *ixy,
                     const float *ixz, const float *iyz)
{
    memcpy(nu, inu, sizeof(float) * (size_t)nodenum);
    memcpy(ro, iro, sizeof(float) * (size_t)nodenum);
    memcpy(nxx, ixx, sizeof(float) * (size_t)nodenum);
    memcpy(nxy, ixy, sizeof(float) * (size_t)nodenum);
    memcpy(nxz, ixz, sizeof(float) * (size_t)nodenum);
    memcpy(nyz, iyz, sizeof(float) * (size_t)nodenum);
}

void p2ref_get_nodes(float *onu, float *oro, float *oxx, float *oxy, float *oxz, float *oyz)
{
    memcpy(onu, nu, sizeof(float) * (size_t)nodenum);
    memcpy(oro, ro, sizeof(float) * (size_t)nodenum);
    memcpy(oxx, nxx, sizeof(float) * (size_t)nodenum);
    memcpy(oxy, nxy, sizeof(float) * (size_t)nodenum);
    memcpy(oxz, nxz, sizeof(float) * (size_t)nodenum);
    memcpy(oyz, nyz, sizeof(float) * (size_t)nodenum);
}

/* Float velocities in node layout, as vpiterate leaves them for movemark. */
void p2ref_set_velocity(const float *ivx, const float *ivy, const float *ivz)
{
    memcpy(vx, ivx, sizeof(float) * (size_t)nodenum);
    memcpy(vy, ivy, sizeof(float) * (size_t)nodenum);
    memcpy(vz, ivz, sizeof(float) * (size_t)nodenum);
}

/* movemark() (mark3mg.c:174) over one step; returns its wall time in seconds. */
double p2ref_movemark(double dt, int mmod, int og)
{
    double t0;
    timestep = dt;
    markmod = mmod;
    outgrid = og;
    mute();
    t0 = omp_get_wtime();
    movemark();
    t0 = omp_get_wtime() - t0;
    unmute();
    return t0;
}

/* The post-solve stress / strain-rate pass of vpiterate (move3mgNew.c:
 * 2908-3038, non-periodic branches) on the current vx, vy, vz and nxx..nyz,
 * through the reference's own value-mode stencils (sxxcalc .. syzcalc with
 * ynval = 0).  out: 12 float[nodenum] arrays sxx syy szz sxy sxz syz exx eyy
 * ezz exy exz eyz; positions the reference does not write are left alone. */
void p2ref_stress_strain(float **out)
{
    long m1, m2, m3, u;
    double e1[100], ui[100];
    long un[100];
    int g = 0;
    for (m3 = 0; m3 < mgz[g]; m3++)
        for (m1 = 0; m1 < mgx[g]; m1++)
            for (m2 = 0; m2 < mgy[g]; m2++) {
                u = m3 * mgxy[g] + m1 * mgy[g] + m2;
                un[0] = 0;
                if (m1 > 0 && m2 > 0 && m3 > 0) {
                    out[0][u] = (float)sxxcalc(m1, m2, m3, 0, g, e1, un, ui); out[6][u] = (float)e1[0];
                    out[1][u] = (float)syycalc(m1, m2, m3, 0, g, e1, un, ui); out[7][u] = (float)e1[0];
                    out[2][u] = (float)szzcalc(m1, m2, m3, 0, g, e1, un, ui); out[8][u] = (float)e1[0];
                }
                if (m1 > 0 && m1 < mgx[g] - 1 && m2 > 0 && m2 < mgy[g] - 1 && m3 < mgz[g] - 1) {
                    out[3][u] = (float)sxycalc(m1, m2, m3, 0, g, e1, un, ui); out[9][u] = (float)e1[0];
                }
                if (m1 > 0 && m1 < mgx[g] - 1 && m3 > 0 && m3 < mgz[g] - 1 && m2 < mgy[g] - 1) {
                    out[4][u] = (float)sxzcalc(m1, m2, m3, 0, g, e1, un, ui); out[10][u] = (float)e1[0];
                }
                if (m2 > 0 && m2 < mgy[g] - 1 && m3 > 0 && m3 < mgz[g] - 1 && m1 < mgx[g] - 1) {
                    out[5][u] = (float)syzcalc(m1, m2, m3, 0, g, e1, un, ui); out[11][u] = (float)e1[0];
                }
            }
}

/* vpiterate's own stress / strain-rate globals: fill, read; step limits. */
static float **stress_globals(float **g)
{
    g[0] = sxx; g[1] = syy; g[2] = szz; g[3] = sxy; g[4] = sxz; g[5] = syz;
    g[6] = exx; g[7] = eyy; g[8] = ezz; g[9] = exy; g[10] = exz; g[11] = eyz;
    return g;
}

void p2ref_fill_stress(float v)
{
    float *g[12];
    long q, i;
    stress_globals(g);
    for (q = 0; q < 12; q++)
        for (i = 0; i < nodenum; i++) g[q][i] = v;
}

void p2ref_get_stress(float **out)
{
    float *g[12];
    long q;
    stress_globals(g);
    for (q = 0; q < 12; q++) memcpy(out[q], g[q], sizeof(float) * (size_t)nodenum);
}

void p2ref_set_stress(float **in)
{
    float *g[12];
    long q;
    stress_globals(g);
    for (q = 0; q < 12; q++) memcpy(g[q], in[q], sizeof(float) * (size_t)nodenum);
}

void p2ref_set_step(double max_step, double ts)
{
    maxxystep = max_step;
    timestep = ts;
}

double p2ref_get_timestep(void) { return timestep; }

/* The stress / strain-rate pass run into vpiterate's own globals (what a
 * vpiterate call leaves for movemark's strain-rate outputs). */
void p2ref_update_stress(void)
{
    float *g[12];
    p2ref_stress_strain(stress_globals(g));
}

void p2ref_set_marke(const float *v)
{
    long i;
    for (i = 0; i < marknum; i++) marke[i] = v[i];
}

void p2ref_fill_val1(double v)
{
    long i;
    for (i = 0; i < marknum; i++) val1[i] = v;
}

void p2ref_get_val1_marke(double *ov, float *oe)
{
    long i;
    for (i = 0; i < marknum; i++) { ov[i] = val1[i]; oe[i] = marke[i]; }
}

/* effbulkvisccalc(1) (mark3mg.c:2-150) on vpiterate's globals; it appends a
 * line to effbulkvisc.txt in the current directory and prints. */
void p2ref_effbulk(const float *iro)
{
    memcpy(ro, iro, sizeof(float) * (size_t)nodenum);
    mute();
    effbulkvisccalc(1);
    unmute();
}

void p2ref_fill_markk(float v)
{
    long i;
    for (i = 0; i < marknum; i++) markk[i] = v;
}

void p2ref_get_markers(float *mx, float *my, float *mz, float *mk)
{
    long i;
    for (i = 0; i < marknum; i++) { mx[i] = markx[i]; my[i] = marky[i]; mz[i] = markz[i]; if (mk) mk[i] = markk[i]; }
}

/* Coarse-level nu/ro/nd after ronurestrict (all levels, concatenated). */
void p2ref_get_level_fields(float *onu, float *oro, float *ond)
{
    long mcmax = mgp[multinum] + mgn[multinum];
    memcpy(onu, nu, sizeof(float) * (size_t)mcmax);
    memcpy(oro, ro, sizeof(float) * (size_t)mcmax);
    memcpy(ond, nd, sizeof(float) * (size_t)mcmax);
}

double p2ref_ronurecalc(void)
{
    double t0;
    mute();
    t0 = omp_get_wtime();
    ronurecalc();
    t0 = omp_get_wtime() - t0;
    unmute();
    return t0;
}

/* True relative residual of the level-0 rows: ||fre1 - A sol0|| / ||fre1||. */
double p2ref_true_residual(double *rnorm_out, double *bnorm_out)
{
    long m, k, n = (long)mgn[0] * 4;
    double rr = 0, bb = 0;
#pragma omp parallel for reduction(+:rr,bb) private(k) schedule(static)
    for (m = 0; m < n; m++) {
        if (num0[m]) {
            double r = fre1[m];
            for (k = 0; k < num0[m]; k++) r -= val1[pos0[m] + k] * sol0[lin0[pos0[m] + k]];
            rr += r * r;
            bb += fre1[m] * fre1[m];
        }
    }
    if (rnorm_out) *rnorm_out = sqrt(rr);
    if (bnorm_out) *bnorm_out = sqrt(bb);
    return bb > 0 ? sqrt(rr / bb) : sqrt(rr);
}

/*
 * First vpiterate() call: assembly of every level (move3mgNew.c:2329-2662),
 * the direct coarsest solve and the nested down-sweep (2741-2791), write-back
 * (2818-2903).  The stop test (3281) is made to pass after this iteration.
 */
double p2ref_vpiterate_first(void)
{
    double t0;
    DIVVMIN = 1e300; STOKSMIN = 1e300; STOKSMAX = 1.0;
    mute();
    t0 = omp_get_wtime();
    vpiterate(0, 0);
    t0 = omp_get_wtime() - t0;
    unmute();
    return t0;
}

/*
 * One further outer iteration exactly as the m2prn>0 branch of vpiterate
 * (move3mgNew.c:2716-2791): pre-smooth + restrict on levels 0..multinum-1,
 * then post-smooth + prolong from multinum-1 down to 0.  With coarse=1 the
 * coarsest level also receives a direct correction (b := restricted rhs,
 * PARDISO, vpprolong(multinum)), the classic V-cycle of the reference's
 * mg/move3mgold.c:2496-2581 variant.
 */
void p2ref_vcycle(int coarse)
{
    int n2, mgi;
    mute();
    for (n2 = 0; n2 < multinum; n2++) {
        mgi = n2;
        if (multinnn[0][mgi] > 0) gausmat4(multinnn[0][mgi], (mgp[mgi] + mgn[mgi]) * 4 - 1, mgp[mgi] * 4, mgi);
        vprestrict(mgi + 1);
    }
    if (coarse) {
        long m1, mc = 0;
        for (m1 = (long)mgp[multinum] * 4; m1 < (long)(mgp[multinum] + mgn[multinum]) * 4; m1++) b[mc++] = fre1[m1];
        pardisomat(0, mgn[multinum] * 4, 0, 0, 0, NULL, NULL);
        vpprolong(multinum, 0);
    }
    for (n2 = multinum - 1; n2 > 0; n2--) {
        mgi = n2;
        if (multinnn[1][mgi] > 0) gausmat4(multinnn[1][mgi], (mgp[mgi] + mgn[mgi]) * 4 - 1, mgp[mgi] * 4, mgi);
        vpprolong(mgi, 0);
    }
    mgi = 0;
    if (multinnn[1][mgi] > 0) gausmat4(multinnn[1][mgi], (mgp[mgi] + mgn[mgi]) * 4 - 1, mgp[mgi] * 4, mgi);
    unmute();
}

/*
 * Level-0 solution in FP64 from sol0, with the reference's pressure reset
 * to pinit in cell (pxinit,pyinit,pzinit) (move3mgNew.c:2834-2855).
 * Fields use the node layout; entries that are not unknowns are 0.
 */
void p2ref_get_solution(double *opr, double *ovx, double *ovy, double *ovz)
{
    long m1, m2, m3, i, n;
    long pin = (pzinit * mgxy[0] + pxinit * mgy[0] + pyinit) * 4;
    double shift = pinit - sol0[pin];
    for (m3 = 0; m3 < mgz[0]; m3++)
        for (m1 = 0; m1 < mgx[0]; m1++)
            for (m2 = 0; m2 < mgy[0]; m2++) {
                i = m3 * mgxy[0] + m1 * mgy[0] + m2;
                n = i * 4;
                opr[i] = (m1 && m2 && m3) ? sol0[n] + shift : 0.0;
                ovx[i] = (m2 < mgy[0] - 1 && m3 < mgz[0] - 1) ? sol0[n + 1] : 0.0;
                ovy[i] = (m1 < mgx[0] - 1 && m3 < mgz[0] - 1) ? sol0[n + 2] : 0.0;
                ovz[i] = (m1 < mgx[0] - 1 && m2 < mgy[0] - 1) ? sol0[n + 3] : 0.0;
            }
}

/* The float/double host arrays vpiterate itself wrote back (vx,vy,vz float; pr double). */
void p2ref_get_written(double *opr, float *ovx, float *ovy, float *ovz)
{
    memcpy(opr, pr, sizeof(double) * (size_t)nodenum);
    memcpy(ovx, vx, sizeof(float) * (size_t)nodenum);
    memcpy(ovy, vy, sizeof(float) * (size_t)nodenum);
    memcpy(ovz, vz, sizeof(float) * (size_t)nodenum);
}

/* Raw FP64 solver vectors of every level (interleaved [P,Vx,Vy,Vz] per node). */
void p2ref_get_vectors(double *osol0, double *ofre1, double *ofre0)
{
    long n = (long)(mgp[multinum] + mgn[multinum]) * 4;
    if (osol0) memcpy(osol0, sol0, sizeof(double) * (size_t)n);
    if (ofre1) memcpy(ofre1, fre1, sizeof(double) * (size_t)n);
    if (ofre0) memcpy(ofre0, fre0, sizeof(double) * (size_t)n);
}

void p2ref_set_sol0(const double *isol0)
{
    long n = (long)(mgp[multinum] + mgn[multinum]) * 4;
    memcpy(sol0, isol0, sizeof(double) * (size_t)n);
}

/* Number of stored coefficients of the level-0 rows (for export sizing). */
long p2ref_rows_nnz(int lev)
{
    long m, nnz = 0;
    for (m = (long)mgp[lev] * 4; m < (long)(mgp[lev] + mgn[lev]) * 4; m++) nnz += num0[m];
    return nnz;
}

/* Export the row store of a level as COO relative to that level. */
void p2ref_get_rows(int lev, int *row, int *col, double *val, double *rhs)
{
    long m, k, c = 0, off = (long)mgp[lev] * 4;
    for (m = off; m < (long)(mgp[lev] + mgn[lev]) * 4; m++) {
        rhs[m - off] = fre1[m];
        for (k = 0; k < num0[m]; k++) {
            row[c] = (int)(m - off);
            col[c] = lin0[pos0[m] + k] - (int)off;
            val[c] = val1[pos0[m] + k];
            c++;
        }
    }
}

/* Apply the reference's level operator (row store) to sol0, returning A x - b
 * per row (the gausmat4 residual with the opposite sign convention). */
void p2ref_rows_apply(int lev, const double *xin, double *yout)
{
    long m, k, off = (long)mgp[lev] * 4, n = (long)mgn[lev] * 4;
    for (m = 0; m < n; m++) {
        double acc = 0;
        for (k = 0; k < num0[m + off]; k++) acc += val1[pos0[m + off] + k] * xin[lin0[pos0[m + off] + k] - off];
        yout[m] = acc;
    }
}

/* Run the reference's restriction / prolongation on given vectors. */
void p2ref_restrict(int lev_coarse, const double *fine_res, double *coarse_rhs)
{
    long nf = (long)mgn[lev_coarse - 1] * 4, nc = (long)mgn[lev_coarse] * 4;
    memcpy(fre0 + (long)mgp[lev_coarse - 1] * 4, fine_res, sizeof(double) * (size_t)nf);
    mute();
    vprestrict(lev_coarse);
    unmute();
    memcpy(coarse_rhs, fre1 + (long)mgp[lev_coarse] * 4, sizeof(double) * (size_t)nc);
}

void p2ref_prolong(int lev_coarse, const double *coarse_x, double *fine_x)
{
    long nf = (long)mgn[lev_coarse - 1] * 4, nc = (long)mgn[lev_coarse] * 4;
    memcpy(sol0 + (long)mgp[lev_coarse] * 4, coarse_x, sizeof(double) * (size_t)nc);
    memcpy(sol0 + (long)mgp[lev_coarse - 1] * 4, fine_x, sizeof(double) * (size_t)nf);
    mute();
    vpprolong(lev_coarse, 0);
    unmute();
    memcpy(fine_x, sol0 + (long)mgp[lev_coarse - 1] * 4, sizeof(double) * (size_t)nf);
}

/* ronurestrict for all coarse levels (move3mgNew.c:3386-3527). */
void p2ref_ronurestrict_all(void)
{
    int l;
    mute();
    for (l = 1; l <= multinum; l++) ronurestrict(l);
    unmute();
}

int p2ref_lu_count(void) { return p2ref_lu_factorizations; }
int p2ref_num_threads(void) { int n = 1;
#pragma omp parallel
    {
#pragma omp master
        n = omp_get_num_threads();
    }
    return n; }

/* am sweeps of the reference smoother gausmat4 on one level (then its residual pass). */
void p2ref_smooth(int mgi, int am)
{
    mute();
    gausmat4(am, (mgp[mgi] + mgn[mgi]) * 4 - 1, mgp[mgi] * 4, mgi);
    unmute();
}

/* ---------------------------------------------------------------------- */
/* titerate() (heat3mg.c:292) on the harness globals.  The active build's  */
/* dynmemall() never allocates tk, tk0, tk1, tk2, cp, kt, ht and et        */
/* (load3mg.c:2239-2334; mode.t3c sets tempmod 0), so the harness gives    */
/* them storage for every level (rocprestrict writes the coarse levels).   */
static void heat_arrays(void)
{
    size_t n = (size_t)nodenum * 2;
    if (!tk) {
        tk = calloc(n, sizeof(float)); tk0 = calloc(n, sizeof(float)); tk1 = calloc(n, sizeof(float));
        tk2 = calloc(n, sizeof(float)); cp = calloc(n, sizeof(float)); kt = calloc(n, sizeof(float));
        ht = calloc(n, sizeof(float)); et = calloc(n, sizeof(float));
    }
}

/* saver() (load3mg.c:1275-1443) in its binary branch (fl1otp 1) to `path`
 * (shorter than fl1out's 60 characters): the harness's node fields, with tk,
 * cp, et, kt, ht (level 0) and the markers' markk, markw, markd, marke set
 * from the arguments first, the gridlines, the boundary rows, the rock table
 * and the markers.  Returns -1 when the path is too long. */
int p2ref_save(const char *path, int cycle, const float *itk, const float *icp, const float *iet, const float *ikt,
               const float *iht, const float *imk, const float *imw, const float *imd, const float *ime)
{
    if (strlen(path) >= sizeof(fl1out)) return -1;
    heat_arrays();
    /* saver() scans bondm[0 .. 10 * nodenum) (load3mg.c:1399-1400) while
     * dynmemall() allocates mcmax + 8 * nodenum entries (load3mg.c:2250):
     * the stock program reads past the array.  The harness extends it with
     * zeros so that the scan stays in bounds (every row index is below
     * 8 * nodenum + mcmax, so the extension adds no row). */
    {
        long mcmax = mgp[multinum] + mgn[multinum], have = mcmax + nodenum8, need = nodenum * 10;
        if (need > have) {
            int *nb = (int *)realloc(bondm, sizeof(int) * (size_t)need);
            if (!nb) return -2;
            memset(nb + have, 0, sizeof(int) * (size_t)(need - have));
            bondm = nb;
        }
    }
    memcpy(tk, itk, sizeof(float) * (size_t)nodenum);
    memcpy(cp, icp, sizeof(float) * (size_t)nodenum);
    memcpy(et, iet, sizeof(float) * (size_t)nodenum);
    memcpy(kt, ikt, sizeof(float) * (size_t)nodenum);
    memcpy(ht, iht, sizeof(float) * (size_t)nodenum);
    memcpy(markk, imk, sizeof(float) * (size_t)marknum);
    memcpy(markw, imw, sizeof(float) * (size_t)marknum);
    memcpy(markd, imd, sizeof(float) * (size_t)marknum);
    memcpy(marke, ime, sizeof(float) * (size_t)marknum);
    strcpy(fl1out, path);
    fl1otp = 1;
    /* saver() ends by reading stop.yn from the working directory
     * (load3mg.c:1744-1761), which loadconf() creates in the stock program */
    {
        FILE *sf = fopen("stop.yn", "wt");
        if (!sf) return -3;
        fprintf(sf, "n\n");
        fclose(sf);
    }
    mute();
    saver(0, cycle);
    unmute();
    return 0;
}

/* T boundary rows: bondm[nodenum8 + u] for the nodes u of every level
 * (in3mg.c:367-383); the rows themselves come with p2ref_set_bc. */
void p2ref_set_tbc(const int *bt)
{
    long mcmax = mgp[multinum] + mgn[multinum], i;
    for (i = 0; i < mcmax; i++) bondm[nodenum8 + i] = bt[i];
}

/* dpar: timestep, maxtkstep, HEATMIN, t0koef, t1koef, heatdif, tdeep, zdeep
 * ipar: multinumt, multicyct, frictyn, adiabyn, multittt[0][0..15], multittt[1][0..15]
 * Node fields are level 0; tk and markk are updated in place; out[0] is the
 * step limit tktimestep the first loop found, out[1] the timestep after. */
void p2ref_titerate(const double *dpar, const int *ipar, float *itk, const float *ikt, const float *icp,
                    const float *iht, const float *iet, const double *ipr, float *imarkk, double *out)
{
    long i, keep;
    int l;
    heat_arrays();
    memcpy(tk, itk, sizeof(float) * (size_t)nodenum);
    memcpy(kt, ikt, sizeof(float) * (size_t)nodenum);
    memcpy(cp, icp, sizeof(float) * (size_t)nodenum);
    memcpy(ht, iht, sizeof(float) * (size_t)nodenum);
    memcpy(et, iet, sizeof(float) * (size_t)nodenum);
    if (ipr) memcpy(pr, ipr, sizeof(double) * (size_t)nodenum);
    /* The marker loops run to marknum inclusive (heat3mg.c:660, 796) and
     * marknum0 == marknum (MRKNEW 1.0), so it reads one slot past the
     * arrays: the harness's last marker is that slot, kept outside the box,
     * and titerate sees marknum - 1 markers. */
    keep = marknum;
    if (keep < 1) return;
    marknum = keep - 1;
    markx[marknum] = -1.0f;
    for (i = 0; i < marknum; i++) markk[i] = imarkk[i];
    timestep = dpar[0]; maxtkstep = dpar[1]; HEATMIN = dpar[2]; t0koef = dpar[3]; t1koef = dpar[4];
    heatdif = dpar[5]; tdeep = dpar[6]; zdeep = dpar[7];
    multinumt = ipar[0]; multicyct = ipar[1]; frictyn = ipar[2]; adiabyn = ipar[3];
    for (l = 0; l < 16; l++) { multittt[0][l] = ipar[4 + l]; multittt[1][l] = ipar[20 + l]; }
    mute();
    titerate(0);
    unmute();
    memcpy(itk, tk, sizeof(float) * (size_t)nodenum);
    for (i = 0; i < marknum; i++) imarkk[i] = markk[i];
    marknum = keep;
    out[0] = 0;
    out[1] = timestep;
}
