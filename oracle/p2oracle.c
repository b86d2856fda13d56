/*
 * CPU oracle: a plain-C restatement of the reference's Stokes multigrid path
 * (TEST INFRASTRUCTURE ONLY — tests, smoke() and bench.py's CPU-baseline leg
 * use it as the checker; the product never links it).
 *
 * What is restated, with the reference lines each part follows
 * (paths relative to the reference project):
 *   level tables / coarse gridlines ...... pardiso/load3mg.c:2056-2194
 *   viscosity per stencil (nxx/nxy/nxz/nyz on level 0, 8- or 2-node averages
 *     of nu on coarse levels, clamp [nubeg,nuend]) ...
 *                                          pardiso/move3mgNew.c:36-49, 431-444,
 *                                          563-577, 701-714, 1506-1523
 *   deviatoric stresses sxx..syz ......... pardiso/move3mgNew.c:3-130, 132-257,
 *                                          259-386, 388-518, 520-657, 659-794
 *   x/y/z-Stokes rows, right-hand sides ... pardiso/move3mgNew.c:796-1008,
 *                                          1011-1228, 1231-1450
 *   continuity row ....................... pardiso/move3mgNew.c:1455-1576
 *   boundary rows x_i = c + k x_j ........ pardiso/move3mgNew.c:1682-1729
 *   damped Gauss-Seidel / Uzawa smoother . pardiso/move3mgNew.c:3854-3959
 *   residual restriction ................. pardiso/move3mgNew.c:3965-4353
 *   correction prolongation .............. pardiso/move3mgNew.c:3534-3849
 *   nu/ro restriction .................... pardiso/move3mgNew.c:3386-3527
 *   pressure reset to pinit .............. pardiso/move3mgNew.c:2834-2855
 *   marker -> node interpolation ......... pardiso/mark3mg.c:630-1133
 *     (power-law rock viscosity, viscalc 1463-1498)
 *   stresses / strain rates after a solve  pardiso/move3mgNew.c:2908-3038
 *   effective bulk viscosity diagnostics . pardiso/mark3mg.c:2-150
 *   marker advection (RK4 / simple) ...... pardiso/mark3mg.c:174-629, with
 *     the staggered velocity interpolation vxyzcalc1 2963-3243
 *     (cell search m1serch..m3serch 1138-1204, constant rock viscosity
 *      viscalc 1481-1482, constant density dencalc1 1429)
 *   coarsest direct solve (MKL PARDISO) .. banded pivoted LU (banded_lu.h)
 *
 * Two deliberate solver-level differences from vpiterate() (the discrete
 * problem is unchanged, so the converged solution is the reference's):
 *   - a classic V-cycle with a direct coarsest correction on every cycle
 *     (the reference solves the coarsest level only on its first outer
 *     iteration, move3mgNew.c:2741-2768);
 *   - the pressure cell pinned by a pure constant boundary row is smoothed
 *     as a continuity row and the pressure is shifted afterwards so that
 *     the pinned value holds; restricted continuity right-hand sides on
 *     coarse levels get a volume-weighted compatibility shift.  With sealed
 *     edges the pinned cell's continuity row is implied by the others, so
 *     the pinned system and this formulation have the same solution.
 * Periodic boundaries (x/y/zperiodic) and the grad-div term (p2koef != 0)
 * are not restated: the oracle rejects them.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "banded_lu.h"

#define MAXLEV 12

typedef struct {
    int nx, ny, nz;
    long n;           /* nodes */
    long off;         /* node offset of the level in the reference layout (mgp) */
    double *gx, *gy, *gz;
    /* inverse spacings, see p2o_spacings() */
    double *ihx, *ihy, *ihz;       /* 1/(g[i]-g[i-1])      (i>=1) */
    double *ihxc, *ihyc, *ihzc;    /* 2/(g[i+1]-g[i-1])    (1<=i<=n-2) */
    double *ihxe, *ihye, *ihze;    /* 1/(g[i+1]-g[i-1])    (1<=i<=n-2) */
    double *ihxv, *ihyv, *ihzv;    /* 1/(g[i+1]-g[i])      (i<=n-2) */
    float *nu, *ro;
    double *ec, *exy, *exz, *eyz;  /* clamped viscosities per stencil */
    double *x[4], *b[4], *r[4];
    unsigned char *bcmask;         /* bit c set: unknown (node,c) is a boundary row */
    int pin;                       /* node index of the pinned pressure cell, -1 none */
    double pinval;
} p2o_level;

typedef struct {
    int nlev;                      /* levels 0..nlev-1 (multinum = nlev-1) */
    p2o_level L[MAXLEV];
    /* boundary tables, reference layout */
    const int *bondm;
    const float *bondv1;
    const int *bondn1;
    /* parameters */
    double p0koef, p1koef, v0koef, v1koef, nubeg, nuend;
    double GX, GY, GZ;
    int viscmod;
    int npre[MAXLEV], npost[MAXLEV];
    /* coarsest factorisation */
    p2_band_lu lu;
    int lu_ready;
} p2o_ctx;

#define IDX(l, i, j, k) ((long)(k) * (l)->nx * (l)->ny + (long)(i) * (l)->ny + (j))

static double clampd(const p2o_ctx *c, double v)
{
    if (v > c->nuend) v = c->nuend;
    if (v < c->nubeg) v = c->nubeg;
    return v;
}

static double vavg(int viscmod, const double *v, int n)
{
    double s = 0;
    int i;
    if (viscmod == 0) { for (i = 0; i < n; i++) s += v[i]; return s / n; }
    if (viscmod == 1) { for (i = 0; i < n; i++) s += log(v[i]); return exp(s / n); }
    for (i = 0; i < n; i++) s += 1.0 / v[i];
    return 1.0 / (s / n);
}

static void spacings(double *g, int n, double **ih, double **ihc, double **ihe, double **ihv)
{
    int i;
    *ih = calloc(n, sizeof(double));
    *ihc = calloc(n, sizeof(double));
    *ihe = calloc(n, sizeof(double));
    *ihv = calloc(n, sizeof(double));
    for (i = 1; i < n; i++) (*ih)[i] = 1.0 / (g[i] - g[i - 1]);
    for (i = 1; i < n - 1; i++) {
        (*ihc)[i] = 2.0 / (g[i + 1] - g[i - 1]);
        (*ihe)[i] = 1.0 / (g[i + 1] - g[i - 1]);
    }
    for (i = 0; i < n - 1; i++) (*ihv)[i] = 1.0 / (g[i + 1] - g[i]);
}

/* ---------------------------------------------------------------------- */
/* Stencil building blocks (level-generic).                               */
#define VX(i, j, k) (l->x[1][IDX(l, i, j, k)])
#define VY(i, j, k) (l->x[2][IDX(l, i, j, k)])
#define VZ(i, j, k) (l->x[3][IDX(l, i, j, k)])
#define PR(i, j, k) (l->x[0][IDX(l, i, j, k)])

/* normal strain-rate parts in cell (a,b,c) */
static void cell_rates(const p2o_level *l, int a, int b, int c, double *dxx, double *dyy, double *dzz)
{
    *dxx = (VX(a, b - 1, c - 1) - VX(a - 1, b - 1, c - 1)) * l->ihx[a];
    *dyy = (VY(a - 1, b, c - 1) - VY(a - 1, b - 1, c - 1)) * l->ihy[b];
    *dzz = (VZ(a - 1, b - 1, c) - VZ(a - 1, b - 1, c - 1)) * l->ihz[c];
}
static double sxx(const p2o_level *l, int a, int b, int c)
{
    double dxx, dyy, dzz;
    cell_rates(l, a, b, c, &dxx, &dyy, &dzz);
    return 2.0 * l->ec[IDX(l, a, b, c)] * (dxx - (dxx + dyy + dzz) / 3.0);
}
static double syy(const p2o_level *l, int a, int b, int c)
{
    double dxx, dyy, dzz;
    cell_rates(l, a, b, c, &dxx, &dyy, &dzz);
    return 2.0 * l->ec[IDX(l, a, b, c)] * (dyy - (dxx + dyy + dzz) / 3.0);
}
static double szz(const p2o_level *l, int a, int b, int c)
{
    double dxx, dyy, dzz;
    cell_rates(l, a, b, c, &dxx, &dyy, &dzz);
    return 2.0 * l->ec[IDX(l, a, b, c)] * (dzz - (dxx + dyy + dzz) / 3.0);
}
static double sxy(const p2o_level *l, int a, int b, int c)
{
    return 2.0 * l->exy[IDX(l, a, b, c)] *
           ((VX(a, b, c) - VX(a, b - 1, c)) * l->ihye[b] + (VY(a, b, c) - VY(a - 1, b, c)) * l->ihxe[a]);
}
static double sxz(const p2o_level *l, int a, int b, int c)
{
    return 2.0 * l->exz[IDX(l, a, b, c)] *
           ((VX(a, b, c) - VX(a, b, c - 1)) * l->ihze[c] + (VZ(a, b, c) - VZ(a - 1, b, c)) * l->ihxe[a]);
}
static double syz(const p2o_level *l, int a, int b, int c)
{
    return 2.0 * l->eyz[IDX(l, a, b, c)] *
           ((VY(a, b, c) - VY(a, b, c - 1)) * l->ihze[c] + (VZ(a, b, c) - VZ(a, b - 1, c)) * l->ihye[b]);
}

/* Rows: (A x) and the diagonal coefficient. */
static double row_vx(const p2o_level *l, int i, int j, int k, double *diag)
{
    double v = (sxx(l, i + 1, j + 1, k + 1) - sxx(l, i, j + 1, k + 1)) * l->ihxc[i] +
               (sxy(l, i, j + 1, k) - sxy(l, i, j, k)) * l->ihyv[j] +
               (sxz(l, i, j, k + 1) - sxz(l, i, j, k)) * l->ihzv[k] -
               (PR(i + 1, j + 1, k + 1) - PR(i, j + 1, k + 1)) * l->ihxc[i];
    if (diag)
        *diag = -(l->ihxc[i] * (4.0 / 3.0) *
                      (l->ec[IDX(l, i + 1, j + 1, k + 1)] * l->ihx[i + 1] + l->ec[IDX(l, i, j + 1, k + 1)] * l->ihx[i]) +
                  l->ihyv[j] * 2.0 * (l->exy[IDX(l, i, j + 1, k)] * l->ihye[j + 1] + l->exy[IDX(l, i, j, k)] * l->ihye[j]) +
                  l->ihzv[k] * 2.0 * (l->exz[IDX(l, i, j, k + 1)] * l->ihze[k + 1] + l->exz[IDX(l, i, j, k)] * l->ihze[k]));
    return v;
}
static double row_vy(const p2o_level *l, int i, int j, int k, double *diag)
{
    double v = (syy(l, i + 1, j + 1, k + 1) - syy(l, i + 1, j, k + 1)) * l->ihyc[j] +
               (sxy(l, i + 1, j, k) - sxy(l, i, j, k)) * l->ihxv[i] +
               (syz(l, i, j, k + 1) - syz(l, i, j, k)) * l->ihzv[k] -
               (PR(i + 1, j + 1, k + 1) - PR(i + 1, j, k + 1)) * l->ihyc[j];
    if (diag)
        *diag = -(l->ihyc[j] * (4.0 / 3.0) *
                      (l->ec[IDX(l, i + 1, j + 1, k + 1)] * l->ihy[j + 1] + l->ec[IDX(l, i + 1, j, k + 1)] * l->ihy[j]) +
                  l->ihxv[i] * 2.0 * (l->exy[IDX(l, i + 1, j, k)] * l->ihxe[i + 1] + l->exy[IDX(l, i, j, k)] * l->ihxe[i]) +
                  l->ihzv[k] * 2.0 * (l->eyz[IDX(l, i, j, k + 1)] * l->ihze[k + 1] + l->eyz[IDX(l, i, j, k)] * l->ihze[k]));
    return v;
}
static double row_vz(const p2o_level *l, int i, int j, int k, double *diag)
{
    double v = (szz(l, i + 1, j + 1, k + 1) - szz(l, i + 1, j + 1, k)) * l->ihzc[k] +
               (sxz(l, i + 1, j, k) - sxz(l, i, j, k)) * l->ihxv[i] +
               (syz(l, i, j + 1, k) - syz(l, i, j, k)) * l->ihyv[j] -
               (PR(i + 1, j + 1, k + 1) - PR(i + 1, j + 1, k)) * l->ihzc[k];
    if (diag)
        *diag = -(l->ihzc[k] * (4.0 / 3.0) *
                      (l->ec[IDX(l, i + 1, j + 1, k + 1)] * l->ihz[k + 1] + l->ec[IDX(l, i + 1, j + 1, k)] * l->ihz[k]) +
                  l->ihxv[i] * 2.0 * (l->exz[IDX(l, i + 1, j, k)] * l->ihxe[i + 1] + l->exz[IDX(l, i, j, k)] * l->ihxe[i]) +
                  l->ihyv[j] * 2.0 * (l->eyz[IDX(l, i, j + 1, k)] * l->ihye[j + 1] + l->eyz[IDX(l, i, j, k)] * l->ihye[j]));
    return v;
}
static double row_p(const p2o_level *l, int i, int j, int k)
{
    return (VX(i, j - 1, k - 1) - VX(i - 1, j - 1, k - 1)) * l->ihx[i] +
           (VY(i - 1, j, k - 1) - VY(i - 1, j - 1, k - 1)) * l->ihy[j] +
           (VZ(i - 1, j - 1, k) - VZ(i - 1, j - 1, k - 1)) * l->ihz[k];
}

static int valid(const p2o_level *l, int c, int i, int j, int k)
{
    if (c == 0) return i > 0 && j > 0 && k > 0;
    if (c == 1) return j < l->ny - 1 && k < l->nz - 1;
    if (c == 2) return i < l->nx - 1 && k < l->nz - 1;
    return i < l->nx - 1 && j < l->ny - 1;
}

/* Boundary row of unknown (node u, comp c) on level li: x = cst + koef * x[target]. */
static void bc_of(const p2o_ctx *C, int li, long u, int c, double *cst, double *koef, long *tnode, int *tcomp)
{
    const p2o_level *l = &C->L[li];
    long g = (l->off + u) * 4 + c;
    int bi = C->bondm[g];
    long t = C->bondn1[bi];
    *cst = C->bondv1[2 * bi];
    *koef = 0;
    *tnode = -1;
    *tcomp = 0;
    if (t) {
        t -= 1;
        *koef = C->bondv1[2 * bi + 1];
        *tnode = t / 4 - l->off;
        *tcomp = (int)(t % 4);
    }
}

/* Is unknown (u,c) a boundary row that is NOT the pressure pin? */
static int is_bc(const p2o_level *l, long u, int c)
{
    if (!(l->bcmask[u] & (1 << c))) return 0;
    if (c == 0 && u == l->pin) return 0;
    return 1;
}

/* r = b - A x on all rows of level li (BC rows: r = cst*(li==0) + koef*x_t - x). */
static void residual(p2o_ctx *C, int li)
{
    p2o_level *l = &C->L[li];
    int i, j, k, c;
#pragma omp parallel for private(i, j, c) schedule(static)
    for (k = 0; k < l->nz; k++)
        for (i = 0; i < l->nx; i++)
            for (j = 0; j < l->ny; j++) {
                long u = IDX(l, i, j, k);
                for (c = 0; c < 4; c++) {
                    double ax;
                    if (!valid(l, c, i, j, k)) { l->r[c][u] = 0; continue; }
                    if (is_bc(l, u, c)) {
                        double cst, koef; long tn; int tc;
                        bc_of(C, li, u, c, &cst, &koef, &tn, &tc);
                        l->r[c][u] = l->b[c][u] + (tn >= 0 ? koef * l->x[tc][tn] : 0.0) - l->x[c][u];
                        continue;
                    }
                    if (c == 0) ax = row_p(l, i, j, k);
                    else if (c == 1) ax = row_vx(l, i, j, k, NULL);
                    else if (c == 2) ax = row_vy(l, i, j, k, NULL);
                    else ax = row_vz(l, i, j, k, NULL);
                    l->r[c][u] = l->b[c][u] - ax;
                }
            }
}

/* Level-0 relative residual of the pinned system: every row except the pinned
 * cell's continuity row (whose pin row is exact after the pressure shift). */
static double rel_residual(p2o_ctx *C, double *rnorm, double *bnorm)
{
    p2o_level *l = &C->L[0];
    long u;
    int c;
    double rr = 0, bb = 0;
    residual(C, 0);
    for (c = 0; c < 4; c++)
        for (u = 0; u < l->n; u++) {
            double bv;
            if (c == 0 && u == l->pin) continue;
            rr += l->r[c][u] * l->r[c][u];
            bv = l->b[c][u];
            bb += bv * bv;
        }
    /* the pin row itself: b = pinval */
    if (l->pin >= 0) bb += l->pinval * l->pinval;
    if (rnorm) *rnorm = sqrt(rr);
    if (bnorm) *bnorm = sqrt(bb);
    return bb > 0 ? sqrt(rr / bb) : sqrt(rr);
}

/* Lexicographic damped Gauss-Seidel with Uzawa pressure update, per node
 * P, Vx, Vy, Vz as gausmat4 does (move3mgNew.c:3880-3924). */
static void smooth(p2o_ctx *C, int li, int sweeps)
{
    p2o_level *l = &C->L[li];
    int s, i, j, k, c;
    for (s = 0; s < sweeps; s++)
        for (k = 0; k < l->nz; k++)
            for (i = 0; i < l->nx; i++)
                for (j = 0; j < l->ny; j++) {
                    long u = IDX(l, i, j, k);
                    for (c = 0; c < 4; c++) {
                        double ax, dg;
                        if (!valid(l, c, i, j, k)) continue;
                        if (is_bc(l, u, c)) {
                            double cst, koef; long tn; int tc;
                            bc_of(C, li, u, c, &cst, &koef, &tn, &tc);
                            l->x[c][u] = l->b[c][u] + (tn >= 0 ? koef * l->x[tc][tn] : 0.0);
                            continue;
                        }
                        if (c == 0) {
                            ax = row_p(l, i, j, k);
                            l->x[0][u] -= (ax - l->b[0][u]) * l->ec[u] * C->p0koef;
                            continue;
                        }
                        if (c == 1) ax = row_vx(l, i, j, k, &dg);
                        else if (c == 2) ax = row_vy(l, i, j, k, &dg);
                        else ax = row_vz(l, i, j, k, &dg);
                        l->x[c][u] -= (ax - l->b[c][u]) / dg * C->v0koef;
                    }
                }
}

/* Coloured cell-block smoother (diagonal Vanka / SCGS): for every cell of one
 * colour (parity of i+j+k) the six face velocities and the cell pressure are
 * corrected together, with the velocity block replaced by its diagonal:
 *   d_v dv_v + g_v dp = r_v,  sum_v c_v dv_v = r_p.
 * All cells of a colour read the state from before that colour's pass
 * (Jacobi within a colour, Gauss-Seidel between colours), which is what a
 * parallel GPU pass does.  Boundary-row faces are excluded from the block and
 * re-applied after each colour. */
static double row_any(const p2o_level *l, int c, int i, int j, int k, double *dg)
{
    if (c == 1) return row_vx(l, i, j, k, dg);
    if (c == 2) return row_vy(l, i, j, k, dg);
    return row_vz(l, i, j, k, dg);
}

static void apply_bc_rows(p2o_ctx *C, int li)
{
    p2o_level *l = &C->L[li];
    int i, j, k, c, pass;
    for (pass = 0; pass < 2; pass++) /* two passes resolve copy chains of length 2 */
        for (k = 0; k < l->nz; k++)
            for (i = 0; i < l->nx; i++)
                for (j = 0; j < l->ny; j++) {
                    long u = IDX(l, i, j, k);
                    for (c = 0; c < 4; c++) {
                        double cst, koef; long tn; int tc;
                        if (!valid(l, c, i, j, k) || !is_bc(l, u, c)) continue;
                        bc_of(C, li, u, c, &cst, &koef, &tn, &tc);
                        l->x[c][u] = l->b[c][u] + (tn >= 0 ? koef * l->x[tc][tn] : 0.0);
                    }
                }
}

double p2o_vanka_omega = 0.7;

/* Off-diagonal couplings between the 6 face velocities of cell (i,j,k) in
 * their own momentum rows (faces: vx left/right, vy front/back, vz
 * bottom/top).  Derived from the stencils above: through the normal stresses
 * of the cell (sxxcalc..szzcalc, move3mgNew.c:3-387) and through the shear
 * stresses on the edges the faces share (sxycalc..syzcalc, 388-795). */
static void face_block(const p2o_level *l, int i, int j, int k, double M[6][6])
{
    const double Ec = l->ec[IDX(l, i, j, k)], hx = l->ihx[i], hy = l->ihy[j], hz = l->ihz[k];
    double dn[3][6];
    int a, b;
#define EXY(a_, b_, c_) l->exy[IDX(l, a_, b_, c_)]
#define EXZ(a_, b_, c_) l->exz[IDX(l, a_, b_, c_)]
#define EYZ(a_, b_, c_) l->eyz[IDX(l, a_, b_, c_)]
    for (a = 0; a < 6; a++)
        for (b = 0; b < 6; b++) M[a][b] = 0.0;
    /* d snn_d(cell) / d face */
    dn[0][0] = -4.0 / 3 * hx; dn[0][1] = 4.0 / 3 * hx; dn[0][2] = 2.0 / 3 * hy; dn[0][3] = -2.0 / 3 * hy;
    dn[0][4] = 2.0 / 3 * hz;  dn[0][5] = -2.0 / 3 * hz;
    dn[1][0] = 2.0 / 3 * hx;  dn[1][1] = -2.0 / 3 * hx; dn[1][2] = -4.0 / 3 * hy; dn[1][3] = 4.0 / 3 * hy;
    dn[1][4] = 2.0 / 3 * hz;  dn[1][5] = -2.0 / 3 * hz;
    dn[2][0] = 2.0 / 3 * hx;  dn[2][1] = -2.0 / 3 * hx; dn[2][2] = 2.0 / 3 * hy; dn[2][3] = -2.0 / 3 * hy;
    dn[2][4] = -4.0 / 3 * hz; dn[2][5] = 4.0 / 3 * hz;
    for (b = 0; b < 6; b++) {
        M[0][b] += Ec * dn[0][b] * l->ihxc[i - 1];
        M[1][b] -= Ec * dn[0][b] * l->ihxc[i];
        M[2][b] += Ec * dn[1][b] * l->ihyc[j - 1];
        M[3][b] -= Ec * dn[1][b] * l->ihyc[j];
        M[4][b] += Ec * dn[2][b] * l->ihzc[k - 1];
        M[5][b] -= Ec * dn[2][b] * l->ihzc[k];
    }
    M[0][3] += 2 * EXY(i - 1, j, k - 1) * l->ihxe[i - 1] * l->ihyv[j - 1];
    M[0][2] -= 2 * EXY(i - 1, j - 1, k - 1) * l->ihxe[i - 1] * l->ihyv[j - 1];
    M[0][5] += 2 * EXZ(i - 1, j - 1, k) * l->ihxe[i - 1] * l->ihzv[k - 1];
    M[0][4] -= 2 * EXZ(i - 1, j - 1, k - 1) * l->ihxe[i - 1] * l->ihzv[k - 1];
    M[1][3] -= 2 * EXY(i, j, k - 1) * l->ihxe[i] * l->ihyv[j - 1];
    M[1][2] += 2 * EXY(i, j - 1, k - 1) * l->ihxe[i] * l->ihyv[j - 1];
    M[1][5] -= 2 * EXZ(i, j - 1, k) * l->ihxe[i] * l->ihzv[k - 1];
    M[1][4] += 2 * EXZ(i, j - 1, k - 1) * l->ihxe[i] * l->ihzv[k - 1];
    M[2][1] += 2 * EXY(i, j - 1, k - 1) * l->ihye[j - 1] * l->ihxv[i - 1];
    M[2][0] -= 2 * EXY(i - 1, j - 1, k - 1) * l->ihye[j - 1] * l->ihxv[i - 1];
    M[2][5] += 2 * EYZ(i - 1, j - 1, k) * l->ihye[j - 1] * l->ihzv[k - 1];
    M[2][4] -= 2 * EYZ(i - 1, j - 1, k - 1) * l->ihye[j - 1] * l->ihzv[k - 1];
    M[3][1] -= 2 * EXY(i, j, k - 1) * l->ihye[j] * l->ihxv[i - 1];
    M[3][0] += 2 * EXY(i - 1, j, k - 1) * l->ihye[j] * l->ihxv[i - 1];
    M[3][5] -= 2 * EYZ(i - 1, j, k) * l->ihye[j] * l->ihzv[k - 1];
    M[3][4] += 2 * EYZ(i - 1, j, k - 1) * l->ihye[j] * l->ihzv[k - 1];
    M[4][1] += 2 * EXZ(i, j - 1, k - 1) * l->ihze[k - 1] * l->ihxv[i - 1];
    M[4][0] -= 2 * EXZ(i - 1, j - 1, k - 1) * l->ihze[k - 1] * l->ihxv[i - 1];
    M[4][3] += 2 * EYZ(i - 1, j, k - 1) * l->ihze[k - 1] * l->ihyv[j - 1];
    M[4][2] -= 2 * EYZ(i - 1, j - 1, k - 1) * l->ihze[k - 1] * l->ihyv[j - 1];
    M[5][1] -= 2 * EXZ(i, j - 1, k) * l->ihze[k] * l->ihxv[i - 1];
    M[5][0] += 2 * EXZ(i - 1, j - 1, k) * l->ihze[k] * l->ihxv[i - 1];
    M[5][3] -= 2 * EYZ(i - 1, j, k) * l->ihze[k] * l->ihyv[j - 1];
    M[5][2] += 2 * EYZ(i - 1, j - 1, k) * l->ihze[k] * l->ihyv[j - 1];
#undef EXY
#undef EXZ
#undef EYZ
}

/* Solve the cell system [M g; cc^T 0] [dv; dp] = [r; rp] by its Schur
 * complement, with M the 6x6 face block (diagonal d), inactive faces held
 * (identity rows), and dp = 0 when the cell pressure is not updated.
 * Gaussian elimination without pivoting: -M is diagonally dominant. */
static void cell_solve(double M[6][6], const int act[6], const double g[6], const double cc[6], const double r[6],
                       double rp, int pact, double dv[6], double *dp)
{
    double A[6][8];
    int a, b, c;
    for (a = 0; a < 6; a++) {
        for (b = 0; b < 6; b++) A[a][b] = (act[a] && act[b]) ? M[a][b] : (a == b ? 1.0 : 0.0);
        A[a][6] = act[a] ? r[a] : 0.0;
        A[a][7] = act[a] ? g[a] : 0.0;
    }
    for (c = 0; c < 6; c++)
        for (a = c + 1; a < 6; a++) {
            double f = A[a][c] / A[c][c];
            if (f == 0.0) continue;
            for (b = c; b < 8; b++) A[a][b] -= f * A[c][b];
        }
    for (c = 5; c >= 0; c--) {
        for (b = c + 1; b < 6; b++) {
            A[c][6] -= A[c][b] * A[b][6];
            A[c][7] -= A[c][b] * A[b][7];
        }
        A[c][6] /= A[c][c];
        A[c][7] /= A[c][c];
    }
    *dp = 0.0;
    if (pact) {
        double num = -rp, den = 0.0;
        for (a = 0; a < 6; a++) {
            num += cc[a] * A[a][6];
            den += cc[a] * A[a][7];
        }
        if (den != 0.0) *dp = num / den;
    }
    for (a = 0; a < 6; a++) dv[a] = act[a] ? A[a][6] - *dp * A[a][7] : 0.0;
}

int p2o_smoother = 2; /* 0: lexicographic GS + Uzawa (reference scheme), 1: diagonal cell-block Vanka,
                         2: full cell-block Vanka (the default), 3: full where smooth_cell, else diagonal */
double p2o_hybrid_ratio = 10.0;

/* Cell whose viscosity is within p2o_hybrid_ratio of its six neighbour cells. */
static int smooth_cell(const p2o_level *l, int i, int j, int k)
{
    const double e = l->ec[IDX(l, i, j, k)];
    const int nb[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    int q;
    for (q = 0; q < 6; q++) {
        int a = i + nb[q][0], b = j + nb[q][1], c = k + nb[q][2];
        double o;
        if (a < 1 || b < 1 || c < 1 || a > l->nx - 1 || b > l->ny - 1 || c > l->nz - 1) continue;
        o = l->ec[IDX(l, a, b, c)];
        if (o > e * p2o_hybrid_ratio || e > o * p2o_hybrid_ratio) return 0;
    }
    return 1;
}

static void smooth_vanka(p2o_ctx *C, int li, int sweeps)
{
    p2o_level *l = &C->L[li];
    double *dx[4];
    int s, col, i, j, k, c;
    for (c = 0; c < 4; c++) dx[c] = calloc(l->n, sizeof(double));
    apply_bc_rows(C, li);
    for (s = 0; s < sweeps; s++)
        for (col = 0; col < 2; col++) {
            for (c = 0; c < 4; c++) memset(dx[c], 0, sizeof(double) * l->n);
#pragma omp parallel for private(i, j) schedule(static)
            for (k = 1; k < l->nz; k++)
                for (i = 1; i < l->nx; i++)
                    for (j = 1; j < l->ny; j++) {
                        long u = IDX(l, i, j, k), vn[6];
                        int vc[6], vi[6], vj[6], vk[6], q, pbc;
                        double r[6], d[6], g[6], cc[6], rp, num = 0, den = 0, dp = 0;
                        if (((i + j + k) & 1) != col) continue;
                        /* faces: vx left/right, vy front/back, vz bottom/top */
                        vc[0] = 1; vi[0] = i - 1; vj[0] = j - 1; vk[0] = k - 1; g[0] = -l->ihxc[i - 1]; cc[0] = -l->ihx[i];
                        vc[1] = 1; vi[1] = i;     vj[1] = j - 1; vk[1] = k - 1; g[1] = +l->ihxc[i];     cc[1] = +l->ihx[i];
                        vc[2] = 2; vi[2] = i - 1; vj[2] = j - 1; vk[2] = k - 1; g[2] = -l->ihyc[j - 1]; cc[2] = -l->ihy[j];
                        vc[3] = 2; vi[3] = i - 1; vj[3] = j;     vk[3] = k - 1; g[3] = +l->ihyc[j];     cc[3] = +l->ihy[j];
                        vc[4] = 3; vi[4] = i - 1; vj[4] = j - 1; vk[4] = k - 1; g[4] = -l->ihzc[k - 1]; cc[4] = -l->ihz[k];
                        vc[5] = 3; vi[5] = i - 1; vj[5] = j - 1; vk[5] = k;     g[5] = +l->ihzc[k];     cc[5] = +l->ihz[k];
                        pbc = is_bc(l, u, 0);
                        for (q = 0; q < 6; q++) {
                            vn[q] = IDX(l, vi[q], vj[q], vk[q]);
                            if (is_bc(l, vn[q], vc[q])) { d[q] = 0; r[q] = 0; continue; }
                            r[q] = l->b[vc[q]][vn[q]] - row_any(l, vc[q], vi[q], vj[q], vk[q], &d[q]);
                            if (!pbc) { num += cc[q] * r[q] / d[q]; den += cc[q] * g[q] / d[q]; }
                        }
                        if (p2o_smoother == 3 && !smooth_cell(l, i, j, k)) {
                            /* interface cell: fall through to the diagonal block */
                        } else if (p2o_smoother >= 2) {
                            double M[6][6], dv[6];
                            int act[6];
                            face_block(l, i, j, k, M);
                            for (q = 0; q < 6; q++) {
                                act[q] = d[q] != 0.0;
                                M[q][q] = d[q];
                            }
                            rp = pbc ? 0.0 : l->b[0][u] - row_p(l, i, j, k);
                            cell_solve(M, act, g, cc, r, rp, !pbc, dv, &dp);
                            if (!pbc) dx[0][u] = dp;
                            for (q = 0; q < 6; q++)
                                if (act[q]) dx[vc[q]][vn[q]] = dv[q];
                            continue;
                        }
                        if (!pbc && den != 0.0) {
                            rp = l->b[0][u] - row_p(l, i, j, k);
                            dp = (num - rp) / den;
                            dx[0][u] = dp;
                        }
                        for (q = 0; q < 6; q++)
                            if (d[q] != 0.0) dx[vc[q]][vn[q]] = (r[q] - (pbc ? 0.0 : g[q] * dp)) / d[q];
                    }
            for (c = 0; c < 4; c++) {
                long u;
#pragma omp parallel for schedule(static)
                for (u = 0; u < l->n; u++) l->x[c][u] += p2o_vanka_omega * dx[c][u];
            }
            apply_bc_rows(C, li);
        }
    for (c = 0; c < 4; c++) free(dx[c]);
}


/* ---------------------------------------------------------------------- */
/* Transfer weights along one axis (vprestrict/vpprolong index rules).     */
typedef struct { int lo; double w0, w1; } axw;

static int cmin_common(int m, int nf, int nc)
{
    int r = (m - 2) / 2 + 2;
    if (m < 3) r = m;
    if (m > nf - 4) r = nc - (nf - m);
    return r;
}

/* node-located component along its own axis */
static axw axis_node(const double *gf, int nf, const double *gc, int nc, int m)
{
    axw a;
    double d;
    int lo = cmin_common(m, nf, nc);
    if (lo > nc - 2) lo = nc - 2;
    d = gc[lo + 1] - gc[lo];
    a.lo = lo;
    a.w0 = 1.0 + (gc[lo] - gf[m]) / d;
    a.w1 = 1.0 - (gc[lo + 1] - gf[m]) / d;
    return a;
}
/* mid-located (between lines m and m+1) */
static axw axis_mid(const double *gf, int nf, const double *gc, int nc, int m)
{
    axw a;
    double d, xf;
    int lo = cmin_common(m, nf, nc);
    if (lo > nc - 3) lo = nc - 3;
    if ((gf[m] + gf[m + 1]) / 2.0 < (gc[lo] + gc[lo + 1]) / 2.0 && lo > 0) lo -= 1;
    d = (gc[lo + 2] - gc[lo]) / 2.0;
    xf = gf[m] + gf[m + 1];
    a.lo = lo;
    a.w0 = 1.0 + (gc[lo] + gc[lo + 1] - xf) / 2.0 / d;
    a.w1 = 1.0 - (gc[lo + 1] + gc[lo + 2] - xf) / 2.0 / d;
    return a;
}
/* pressure cell centre (between lines m-1 and m) */
static axw axis_cell(const double *gf, int nf, const double *gc, int nc, int m)
{
    axw a;
    double d, xf;
    int lo = cmin_common(m, nf, nc);
    if (lo > nc - 2) lo = nc - 2;
    if ((gf[m] + gf[m - 1]) / 2.0 < (gc[lo] + gc[lo - 1]) / 2.0 && lo > 1) lo -= 1;
    d = (gc[lo + 1] - gc[lo - 1]) / 2.0;
    xf = gf[m] + gf[m - 1];
    a.lo = lo;
    a.w0 = 1.0 + (gc[lo] + gc[lo - 1] - xf) / 2.0 / d;
    a.w1 = 1.0 - (gc[lo + 1] + gc[lo] - xf) / 2.0 / d;
    return a;
}

static void axes_for(const p2o_level *f, const p2o_level *cl, int c, int i, int j, int k, axw *ax, axw *ay, axw *az)
{
    if (c == 0) {
        *ax = axis_cell(f->gx, f->nx, cl->gx, cl->nx, i);
        *ay = axis_cell(f->gy, f->ny, cl->gy, cl->ny, j);
        *az = axis_cell(f->gz, f->nz, cl->gz, cl->nz, k);
    } else if (c == 1) {
        *ax = axis_node(f->gx, f->nx, cl->gx, cl->nx, i);
        *ay = axis_mid(f->gy, f->ny, cl->gy, cl->ny, j);
        *az = axis_mid(f->gz, f->nz, cl->gz, cl->nz, k);
    } else if (c == 2) {
        *ax = axis_mid(f->gx, f->nx, cl->gx, cl->nx, i);
        *ay = axis_node(f->gy, f->ny, cl->gy, cl->ny, j);
        *az = axis_mid(f->gz, f->nz, cl->gz, cl->nz, k);
    } else {
        *ax = axis_mid(f->gx, f->nx, cl->gx, cl->nx, i);
        *ay = axis_mid(f->gy, f->ny, cl->gy, cl->ny, j);
        *az = axis_node(f->gz, f->nz, cl->gz, cl->nz, k);
    }
}

static double cell_volume(const p2o_level *l, int i, int j, int k)
{
    return 1.0 / (l->ihx[i] * l->ihy[j] * l->ihz[k]);
}

/* Coarse right-hand side from the fine residual (vprestrict), then the
 * compatibility shift of the continuity rows. */
int p2o_eta_scale = 1;
static int p2o_compat = 1;
static void restrict_level(p2o_ctx *C, int lc)
{
    p2o_level *f = &C->L[lc - 1], *cl = &C->L[lc];
    double *acc[4], *wsum[4];
    int c, i, j, k, a, b2, d;
    for (c = 0; c < 4; c++) {
        acc[c] = calloc(cl->n, sizeof(double));
        wsum[c] = calloc(cl->n, sizeof(double));
    }
    for (k = 0; k < f->nz; k++)
        for (i = 0; i < f->nx; i++)
            for (j = 0; j < f->ny; j++) {
                long u = IDX(f, i, j, k);
                for (c = 0; c < 4; c++) {
                    axw ax, ay, az;
                    if (!valid(f, c, i, j, k) || is_bc(f, u, c)) continue;
                    axes_for(f, cl, c, i, j, k, &ax, &ay, &az);
                    for (d = 0; d < 2; d++)
                        for (a = 0; a < 2; a++)
                            for (b2 = 0; b2 < 2; b2++) {
                                long v = IDX(cl, ax.lo + a, ay.lo + b2, az.lo + d);
                                double w = (a ? ax.w1 : ax.w0) * (b2 ? ay.w1 : ay.w0) * (d ? az.w1 : az.w0);
                                double val = f->r[c][u];
                                if (is_bc(cl, v, c)) continue;
                                if (c == 0 && p2o_eta_scale) val *= f->ec[u] / cl->ec[v];
                                acc[c][v] += val * w;
                                wsum[c][v] += w;
                            }
                }
            }
    for (c = 0; c < 4; c++) {
        long v;
        for (v = 0; v < cl->n; v++) {
            cl->b[c][v] = wsum[c][v] != 0 ? acc[c][v] / wsum[c][v] : 0.0;
            cl->x[c][v] = 0;
        }
        free(acc[c]);
        free(wsum[c]);
    }
    /* compatibility: sum over continuity rows of volume * rhs must vanish */
    if (p2o_compat) {
        double sv = 0, s = 0;
        for (k = 1; k < cl->nz; k++)
            for (i = 1; i < cl->nx; i++)
                for (j = 1; j < cl->ny; j++) {
                    long v = IDX(cl, i, j, k);
                    if (is_bc(cl, v, 0)) continue;
                    s += cell_volume(cl, i, j, k) * cl->b[0][v];
                    sv += cell_volume(cl, i, j, k);
                }
        if (sv > 0) {
            double sh = s / sv;
            for (k = 1; k < cl->nz; k++)
                for (i = 1; i < cl->nx; i++)
                    for (j = 1; j < cl->ny; j++) {
                        long v = IDX(cl, i, j, k);
                        if (!is_bc(cl, v, 0)) cl->b[0][v] -= sh;
                    }
        }
    }
}

static void prolong_level(p2o_ctx *C, int lc)
{
    p2o_level *f = &C->L[lc - 1], *cl = &C->L[lc];
    int c, i, j, k, a, b2, d;
#pragma omp parallel for private(i, j, c, a, b2, d) schedule(static)
    for (k = 0; k < f->nz; k++)
        for (i = 0; i < f->nx; i++)
            for (j = 0; j < f->ny; j++) {
                long u = IDX(f, i, j, k);
                for (c = 0; c < 4; c++) {
                    axw ax, ay, az;
                    double s = 0;
                    if (!valid(f, c, i, j, k)) continue;
                    axes_for(f, cl, c, i, j, k, &ax, &ay, &az);
                    for (d = 0; d < 2; d++)
                        for (a = 0; a < 2; a++)
                            for (b2 = 0; b2 < 2; b2++) {
                                long v = IDX(cl, ax.lo + a, ay.lo + b2, az.lo + d);
                                double w = (a ? ax.w1 : ax.w0) * (b2 ? ay.w1 : ay.w0) * (d ? az.w1 : az.w0);
                                s += cl->x[c][v] * w;
                            }
                    f->x[c][u] += s * (c == 0 ? C->p1koef : C->v1koef);
                }
            }
}

/* Coarse-level viscosity scheme (a preconditioner choice; the level-0
 * problem does not depend on it):
 *   -1     the model's viscmod (the reference's ronurestrict,
 *          move3mgNew.c:3386-3527, then 8-/2-node stencil means 45-47, 442-444);
 *   0/1/2  the same chain with linear / log / inverse means;
 *   3/4/5  stencil-consistent: each coarse stencil viscosity is the log /
 *          linear / inverse mean of the finer level's viscosity of the same
 *          kind (cells for ec; z-, y-, x-edges for exy, exz, eyz) over the
 *          coarse position's control volume, weighted by overlap. */
int p2o_coarse_avg = -1;

static int coarse_mode(const p2o_ctx *C)
{
    return p2o_coarse_avg >= 0 && p2o_coarse_avg <= 2 ? p2o_coarse_avg : C->viscmod;
}

/* kind 0: cell m = [g[m-1], g[m]]; 1: segment [g[m], g[m+1]]; 2: dual of node m */
static void span(const double *g, int n, int kind, int m, double *a, double *b)
{
    if (kind == 0) { *a = g[m - 1]; *b = g[m]; return; }
    if (kind == 1) { *a = g[m]; *b = g[m + 1]; return; }
    *a = m > 0 ? 0.5 * (g[m - 1] + g[m]) : g[0];
    *b = m < n - 1 ? 0.5 * (g[m] + g[m + 1]) : g[n - 1];
}

static double overlap(double a0, double b0, double a1, double b1)
{
    double lo = a0 > a1 ? a0 : a1, hi = b0 < b1 ? b0 : b1;
    return hi > lo ? hi - lo : 0.0;
}

static void consistent_viscosity(p2o_ctx *C, int li)
{
    p2o_level *l = &C->L[li], *f = &C->L[li - 1];
    const int mode = p2o_coarse_avg;
    /* position kind per field and axis (x, y, z) */
    static const int kinds[4][3] = {{0, 0, 0}, {2, 2, 1}, {2, 1, 2}, {1, 2, 2}};
    double *dst[4];
    const double *src[4];
    int nc[3], nf[3], q, k;
    const double *gc[3], *gf[3];
    dst[0] = l->ec; dst[1] = l->exy; dst[2] = l->exz; dst[3] = l->eyz;
    src[0] = f->ec; src[1] = f->exy; src[2] = f->exz; src[3] = f->eyz;
    nc[0] = l->nx; nc[1] = l->ny; nc[2] = l->nz;
    nf[0] = f->nx; nf[1] = f->ny; nf[2] = f->nz;
    gc[0] = l->gx; gc[1] = l->gy; gc[2] = l->gz;
    gf[0] = f->gx; gf[1] = f->gy; gf[2] = f->gz;
    for (q = 0; q < 4; q++)
#pragma omp parallel for schedule(static)
        for (k = 0; k < l->nz; k++) {
            int i, j;
            for (i = 0; i < l->nx; i++)
                for (j = 0; j < l->ny; j++) {
                    int I[3], ax, ok = 1, lo[3], hi[3], a, b2, d;
                    double A[3], B[3], s = 0.0, ws = 0.0, m;
                    long u = IDX(l, i, j, k);
                    I[0] = i; I[1] = j; I[2] = k;
                    for (ax = 0; ax < 3; ax++) {
                        int kd = kinds[q][ax];
                        if ((kd == 0 && I[ax] < 1) || (kd == 1 && I[ax] > nc[ax] - 2)) ok = 0;
                    }
                    if (!ok) continue;  /* keeps the value of the node-viscosity chain */
                    for (ax = 0; ax < 3; ax++) {
                        int c0 = 2 * I[ax] - 2;
                        span(gc[ax], nc[ax], kinds[q][ax], I[ax], &A[ax], &B[ax]);
                        lo[ax] = c0 - 4 < 0 ? 0 : c0 - 4;
                        hi[ax] = c0 + 4 > nf[ax] - 1 ? nf[ax] - 1 : c0 + 4;
                    }
                    if (mode == 6 && q > 0) {
                        /* shear viscosity: harmonic (in series) over the two gradient
                         * directions, arithmetic (in parallel) along the edge */
                        const int par = q == 1 ? 2 : (q == 2 ? 1 : 0);
                        int t;
                        for (t = lo[par]; t <= hi[par]; t++) {
                            double wp, fa, fb, sh = 0.0, wh = 0.0;
                            int kd = kinds[q][par];
                            if ((kd == 0 && t < 1) || (kd == 1 && t > nf[par] - 2)) continue;
                            span(gf[par], nf[par], kd, t, &fa, &fb);
                            wp = overlap(A[par], B[par], fa, fb);
                            if (wp <= 0.0) continue;
                            for (d = lo[2]; d <= hi[2]; d++)
                                for (a = lo[0]; a <= hi[0]; a++)
                                    for (b2 = lo[1]; b2 <= hi[1]; b2++) {
                                        int J[3];
                                        double w = 1.0;
                                        J[0] = a; J[1] = b2; J[2] = d;
                                        if (J[par] != t) continue;
                                        for (ax = 0; ax < 3; ax++) {
                                            int kk2 = kinds[q][ax];
                                            if (ax == par) continue;
                                            if ((kk2 == 0 && J[ax] < 1) || (kk2 == 1 && J[ax] > nf[ax] - 2)) { w = 0.0; break; }
                                            span(gf[ax], nf[ax], kk2, J[ax], &fa, &fb);
                                            w *= overlap(A[ax], B[ax], fa, fb);
                                            if (w <= 0.0) break;
                                        }
                                        if (w <= 0.0) continue;
                                        sh += w / src[q][IDX(f, a, b2, d)];
                                        wh += w;
                                    }
                            if (wh <= 0.0) continue;
                            s += wp * (wh / sh);
                            ws += wp;
                        }
                        if (ws <= 0.0) continue;
                        dst[q][u] = clampd(C, s / ws);
                        continue;
                    }
                    for (d = lo[2]; d <= hi[2]; d++)
                        for (a = lo[0]; a <= hi[0]; a++)
                            for (b2 = lo[1]; b2 <= hi[1]; b2++) {
                                int J[3];
                                double w = 1.0, fa, fb, v;
                                J[0] = a; J[1] = b2; J[2] = d;
                                for (ax = 0; ax < 3; ax++) {
                                    int kd = kinds[q][ax];
                                    if ((kd == 0 && J[ax] < 1) || (kd == 1 && J[ax] > nf[ax] - 2)) { w = 0.0; break; }
                                    span(gf[ax], nf[ax], kd, J[ax], &fa, &fb);
                                    w *= overlap(A[ax], B[ax], fa, fb);
                                    if (w <= 0.0) break;
                                }
                                if (w <= 0.0) continue;
                                v = src[q][IDX(f, a, b2, d)];
                                s += w * ((mode == 3 || mode == 6) ? log(v) : mode == 4 ? v : 1.0 / v);
                                ws += w;
                            }
                    if (ws <= 0.0) continue;
                    m = s / ws;
                    m = (mode == 3 || mode == 6) ? exp(m) : mode == 4 ? m : 1.0 / m;
                    dst[q][u] = clampd(C, m);
                }
        }
}

/* nu, ro of level lc from level lc-1 (ronurestrict). */
static void ronurestrict_level(p2o_ctx *C, int lc)
{
    p2o_level *f = &C->L[lc - 1], *cl = &C->L[lc];
    const int vm = coarse_mode(C);
    double *sn = calloc(cl->n, sizeof(double)), *sr = calloc(cl->n, sizeof(double)), *sw = calloc(cl->n, sizeof(double));
    int i, j, k, a, b2, d;
    long v;
    for (k = 0; k < f->nz; k++)
        for (i = 0; i < f->nx; i++)
            for (j = 0; j < f->ny; j++) {
                long u = IDX(f, i, j, k);
                int lo[3], m[3], n[3], nf[3], q;
                const double *gf[3], *gc[3];
                m[0] = i; m[1] = j; m[2] = k;
                nf[0] = f->nx; nf[1] = f->ny; nf[2] = f->nz;
                n[0] = cl->nx; n[1] = cl->ny; n[2] = cl->nz;
                gf[0] = f->gx; gf[1] = f->gy; gf[2] = f->gz;
                gc[0] = cl->gx; gc[1] = cl->gy; gc[2] = cl->gz;
                for (q = 0; q < 3; q++) {
                    lo[q] = cmin_common(m[q], nf[q], n[q]);
                    if (lo[q] > n[q] - 2) lo[q] = n[q] - 2;
                }
                for (d = 0; d < 2; d++)
                    for (a = 0; a < 2; a++)
                        for (b2 = 0; b2 < 2; b2++) {
                            double wz = 1.0 - fabs((gc[2][lo[2] + d] - gf[2][k]) / (gc[2][lo[2] + 1] - gc[2][lo[2]]));
                            double wx = 1.0 - fabs((gc[0][lo[0] + a] - gf[0][i]) / (gc[0][lo[0] + 1] - gc[0][lo[0]]));
                            double wy = 1.0 - fabs((gc[1][lo[1] + b2] - gf[1][j]) / (gc[1][lo[1] + 1] - gc[1][lo[1]]));
                            double w = wx * wy * wz, fv;
                            long t = IDX(cl, lo[0] + a, lo[1] + b2, lo[2] + d);
                            if (vm == 0) fv = f->nu[u];
                            else if (vm == 1) fv = log(f->nu[u]);
                            else fv = 1.0 / f->nu[u];
                            sn[t] += fv * w;
                            sr[t] += f->ro[u] * w;
                            sw[t] += w;
                        }
            }
    for (v = 0; v < cl->n; v++) {
        double nv = sn[v] / sw[v];
        if (vm == 1) nv = exp(nv);
        if (vm == 2) nv = 1.0 / nv;
        cl->nu[v] = (float)nv;
        cl->ro[v] = (float)(sr[v] / sw[v]);
    }
    free(sn); free(sr); free(sw);
}

/* Viscosity per stencil on a level (level 0 from nxx..nyz, coarse from nu). */
static void level_viscosity(p2o_ctx *C, int li, const float *nxx, const float *nxy, const float *nxz, const float *nyz)
{
    p2o_level *l = &C->L[li];
    int i, j, k;
    for (k = 0; k < l->nz; k++)
        for (i = 0; i < l->nx; i++)
            for (j = 0; j < l->ny; j++) {
                long u = IDX(l, i, j, k);
                if (li == 0) {
                    l->ec[u] = clampd(C, nxx[u]);
                    l->exy[u] = clampd(C, nxy[u]);
                    l->exz[u] = clampd(C, nxz[u]);
                    l->eyz[u] = clampd(C, nyz[u]);
                    continue;
                }
                if (i > 0 && j > 0 && k > 0) {
                    double v[8];
                    v[0] = l->nu[IDX(l, i - 1, j - 1, k - 1)]; v[1] = l->nu[IDX(l, i - 1, j, k - 1)];
                    v[2] = l->nu[IDX(l, i, j - 1, k - 1)];     v[3] = l->nu[IDX(l, i, j, k - 1)];
                    v[4] = l->nu[IDX(l, i - 1, j - 1, k)];     v[5] = l->nu[IDX(l, i - 1, j, k)];
                    v[6] = l->nu[IDX(l, i, j - 1, k)];         v[7] = l->nu[IDX(l, i, j, k)];
                    l->ec[u] = clampd(C, vavg(coarse_mode(C), v, 8));
                } else {
                    l->ec[u] = C->nubeg;
                }
                {
                    double v[2];
                    v[0] = l->nu[u];
                    v[1] = k + 1 < l->nz ? l->nu[IDX(l, i, j, k + 1)] : l->nu[u];
                    l->exy[u] = clampd(C, vavg(coarse_mode(C), v, 2));
                    v[1] = j + 1 < l->ny ? l->nu[IDX(l, i, j + 1, k)] : l->nu[u];
                    l->exz[u] = clampd(C, vavg(coarse_mode(C), v, 2));
                    v[1] = i + 1 < l->nx ? l->nu[IDX(l, i + 1, j, k)] : l->nu[u];
                    l->eyz[u] = clampd(C, vavg(coarse_mode(C), v, 2));
                }
            }
}

/* ---------------------------------------------------------------------- */
/* Coarsest operator: probe the matrix-free rows (pinned system: the pin row
 * is x = 0, ghost rows are the identity) and factor as a band. */
static int coarse_factor(p2o_ctx *C)
{
    int li = C->nlev - 1;
    p2o_level *l = &C->L[li];
    long N = l->n * 4, kl = 4 * ((long)l->nx * l->ny + l->ny + 1) + 8;
    int cx, cy, cz, cc, i, j, k, c;
    double *save[4];
    if (C->lu_ready) { p2_band_free(&C->lu); C->lu_ready = 0; }
    if (p2_band_alloc(&C->lu, N, kl, kl)) return -1;
    for (c = 0; c < 4; c++) { save[c] = l->x[c]; l->x[c] = calloc(l->n, sizeof(double)); }
    for (cz = 0; cz < 5; cz++)
        for (cx = 0; cx < 5; cx++)
            for (cy = 0; cy < 5; cy++)
                for (cc = 0; cc < 4; cc++) {
                    for (c = 0; c < 4; c++) memset(l->x[c], 0, sizeof(double) * l->n);
                    for (k = cz; k < l->nz; k += 5)
                        for (i = cx; i < l->nx; i += 5)
                            for (j = cy; j < l->ny; j += 5) l->x[cc][IDX(l, i, j, k)] = 1.0;
                    for (k = 0; k < l->nz; k++)
                        for (i = 0; i < l->nx; i++)
                            for (j = 0; j < l->ny; j++) {
                                long u = IDX(l, i, j, k);
                                int ci = i + ((cx - i) % 5 + 5) % 5, cj = j + ((cy - j) % 5 + 5) % 5, ck = k + ((cz - k) % 5 + 5) % 5;
                                long col;
                                if (ci > i + 2) ci -= 5;
                                if (cj > j + 2) cj -= 5;
                                if (ck > k + 2) ck -= 5;
                                if (ci < 0 || cj < 0 || ck < 0 || ci >= l->nx || cj >= l->ny || ck >= l->nz) continue;
                                col = IDX(l, ci, cj, ck) * 4 + cc;
                                for (c = 0; c < 4; c++) {
                                    long row = u * 4 + c;
                                    double a;
                                    if (!valid(l, c, i, j, k)) {
                                        a = (row == col) ? 1.0 : 0.0;
                                    } else if ((l->bcmask[u] & (1 << c))) {
                                        double cst, koef; long tn; int tc;
                                        bc_of(C, li, u, c, &cst, &koef, &tn, &tc);
                                        a = (row == col) ? 1.0 : 0.0;
                                        if (tn >= 0 && tn * 4 + tc == col) a -= koef;
                                    } else if (c == 0) {
                                        a = row_p(l, i, j, k);
                                    } else if (c == 1) {
                                        a = row_vx(l, i, j, k, NULL);
                                    } else if (c == 2) {
                                        a = row_vy(l, i, j, k, NULL);
                                    } else {
                                        a = row_vz(l, i, j, k, NULL);
                                    }
                                    if (a != 0.0) {
                                        if (labs(row - col) > kl) { fprintf(stderr, "coarse band overflow\n"); return -2; }
                                        *p2_band_at(&C->lu, row, col) = a;
                                    }
                                }
                            }
                }
    for (c = 0; c < 4; c++) { free(l->x[c]); l->x[c] = save[c]; }
    C->lu_ready = 1;
    return p2_band_factor(&C->lu);
}

static void coarse_solve(p2o_ctx *C)
{
    int li = C->nlev - 1;
    p2o_level *l = &C->L[li];
    long N = l->n * 4, u;
    int c;
    double *rhs = calloc(N, sizeof(double));
    for (u = 0; u < l->n; u++)
        for (c = 0; c < 4; c++) {
            int ii = (int)((u / l->ny) % l->nx), jj = (int)(u % l->ny), kk = (int)(u / ((long)l->nx * l->ny));
            if (!valid(l, c, ii, jj, kk) || (l->bcmask[u] & (1 << c))) rhs[u * 4 + c] = 0;
            else rhs[u * 4 + c] = l->b[c][u];
        }
    p2_band_solve(&C->lu, rhs);
    for (u = 0; u < l->n; u++)
        for (c = 0; c < 4; c++) l->x[c][u] = rhs[u * 4 + c];
    free(rhs);
}

/* Shift the pressure so that the pinned cell holds its value. */
static void normalize_pressure(p2o_ctx *C, int li)
{
    p2o_level *l = &C->L[li];
    long u;
    double sh;
    if (l->pin < 0) return;
    sh = (li == 0 ? l->pinval : 0.0) - l->x[0][l->pin];
    for (u = 0; u < l->n; u++) {
        int i = (int)((u / l->ny) % l->nx), j = (int)(u % l->ny), k = (int)(u / ((long)l->nx * l->ny));
        if (i > 0 && j > 0 && k > 0) l->x[0][u] += sh;
    }
}

static void vcycle(p2o_ctx *C)
{
    int li;
    for (li = 0; li < C->nlev - 1; li++) {
        if (p2o_smoother) smooth_vanka(C, li, C->npre[li]); else smooth(C, li, C->npre[li]);
        residual(C, li);
        restrict_level(C, li + 1);
    }
    coarse_solve(C);
    for (li = C->nlev - 2; li >= 0; li--) {
        prolong_level(C, li + 1);
        if (p2o_smoother) smooth_vanka(C, li, C->npost[li]); else smooth(C, li, C->npost[li]);
    }
}

/* ---------------------------------------------------------------------- */
/* Public API (ctypes).                                                    */

void *p2o_create(int nx, int ny, int nz, const double *gx, const double *gy, const double *gz, int multinum,
                 const int *bondm, const float *bondv1, const int *bondn1)
{
    p2o_ctx *C = calloc(1, sizeof(p2o_ctx));
    int li;
    long off = 0;
    if (multinum + 1 > MAXLEV) { free(C); return NULL; }
    C->nlev = multinum + 1;
    C->bondm = bondm; C->bondv1 = bondv1; C->bondn1 = bondn1;
    for (li = 0; li <= multinum; li++) {
        p2o_level *l = &C->L[li];
        int q, c, s = 1 << li;
        if (li == 0) { l->nx = nx; l->ny = ny; l->nz = nz; }
        else {
            l->nx = (C->L[li - 1].nx - 5) / 2 + 5;
            l->ny = (C->L[li - 1].ny - 5) / 2 + 5;
            l->nz = (C->L[li - 1].nz - 5) / 2 + 5;
        }
        l->n = (long)l->nx * l->ny * l->nz;
        l->off = off;
        off += l->n;
        l->gx = malloc(sizeof(double) * l->nx);
        l->gy = malloc(sizeof(double) * l->ny);
        l->gz = malloc(sizeof(double) * l->nz);
        /* load3mg.c:2079-2194: outer three lines copied, interior (n2-2)*s+2 */
        for (q = 0; q < 3; q++) {
            int n = q == 0 ? l->nx : q == 1 ? l->ny : l->nz, nf = q == 0 ? nx : q == 1 ? ny : nz, n2;
            const double *g = q == 0 ? gx : q == 1 ? gy : gz;
            double *o = q == 0 ? l->gx : q == 1 ? l->gy : l->gz;
            o[0] = g[0]; o[1] = g[1]; o[2] = g[2];
            o[n - 1] = g[nf - 1]; o[n - 2] = g[nf - 2]; o[n - 3] = g[nf - 3];
            for (n2 = 3; n2 < n - 3; n2++) o[n2] = g[(n2 - 2) * s + 2];
        }
        spacings(l->gx, l->nx, &l->ihx, &l->ihxc, &l->ihxe, &l->ihxv);
        spacings(l->gy, l->ny, &l->ihy, &l->ihyc, &l->ihye, &l->ihyv);
        spacings(l->gz, l->nz, &l->ihz, &l->ihzc, &l->ihze, &l->ihzv);
        l->nu = calloc(l->n, sizeof(float));
        l->ro = calloc(l->n, sizeof(float));
        l->ec = calloc(l->n, sizeof(double));
        l->exy = calloc(l->n, sizeof(double));
        l->exz = calloc(l->n, sizeof(double));
        l->eyz = calloc(l->n, sizeof(double));
        for (c = 0; c < 4; c++) {
            l->x[c] = calloc(l->n, sizeof(double));
            l->b[c] = calloc(l->n, sizeof(double));
            l->r[c] = calloc(l->n, sizeof(double));
        }
        l->bcmask = calloc(l->n, 1);
        l->pin = -1;
        {
            long u;
            int npin = 0;
            for (u = 0; u < l->n; u++)
                for (c = 0; c < 4; c++)
                    if (bondm[(l->off + u) * 4 + c]) {
                        l->bcmask[u] |= (unsigned char)(1 << c);
                        if (c == 0 && bondn1[bondm[(l->off + u) * 4]] == 0) {
                            npin++;
                            l->pin = u;
                            l->pinval = bondv1[2 * bondm[(l->off + u) * 4]];
                        }
                    }
            if (npin != 1) l->pin = -1; /* several pure pins: all stay boundary rows */
        }
    }
    return C;
}

void p2o_destroy(void *h)
{
    p2o_ctx *C = h;
    int li, c;
    if (!C) return;
    for (li = 0; li < C->nlev; li++) {
        p2o_level *l = &C->L[li];
        free(l->gx); free(l->gy); free(l->gz);
        free(l->ihx); free(l->ihxc); free(l->ihxe); free(l->ihxv);
        free(l->ihy); free(l->ihyc); free(l->ihye); free(l->ihyv);
        free(l->ihz); free(l->ihzc); free(l->ihze); free(l->ihzv);
        free(l->nu); free(l->ro); free(l->ec); free(l->exy); free(l->exz); free(l->eyz);
        for (c = 0; c < 4; c++) { free(l->x[c]); free(l->b[c]); free(l->r[c]); }
        free(l->bcmask);
    }
    if (C->lu_ready) p2_band_free(&C->lu);
    free(C);
}

/* dpar: p0koef p1koef v0koef v1koef nubeg nuend GX GY GZ ; viscmod */
void p2o_set_params(void *h, const double *dpar, int viscmod, const int *npre, const int *npost)
{
    p2o_ctx *C = h;
    int li;
    C->p0koef = dpar[0]; C->p1koef = dpar[1]; C->v0koef = dpar[2]; C->v1koef = dpar[3];
    C->nubeg = dpar[4]; C->nuend = dpar[5]; C->GX = dpar[6]; C->GY = dpar[7]; C->GZ = dpar[8];
    C->viscmod = viscmod;
    for (li = 0; li < C->nlev; li++) { C->npre[li] = npre[li]; C->npost[li] = npost[li]; }
}

/* Node fields (level 0) -> coarse nu/ro, stencil viscosities, level-0 rhs,
 * coarsest factorisation.  Returns 0 or the LU status. */
int p2o_set_fields(void *h, const float *nu, const float *ro, const float *nxx, const float *nxy,
                   const float *nxz, const float *nyz)
{
    p2o_ctx *C = h;
    p2o_level *l = &C->L[0];
    int li, i, j, k;
    memcpy(l->nu, nu, sizeof(float) * l->n);
    memcpy(l->ro, ro, sizeof(float) * l->n);
    for (li = 1; li < C->nlev; li++) ronurestrict_level(C, li);
    level_viscosity(C, 0, nxx, nxy, nxz, nyz);
    for (li = 1; li < C->nlev; li++) {
        level_viscosity(C, li, NULL, NULL, NULL, NULL);
        if (p2o_coarse_avg >= 3) consistent_viscosity(C, li);
    }
    /* level-0 right-hand sides (xstokserr:845, ystokserr:1060, zstokserr:1279) */
    for (k = 0; k < l->nz; k++)
        for (i = 0; i < l->nx; i++)
            for (j = 0; j < l->ny; j++) {
                long u = IDX(l, i, j, k);
                l->b[0][u] = 0;
                l->b[1][u] = l->b[2][u] = l->b[3][u] = 0;
                /* the four float densities are summed in float, as the reference does */
                if (valid(l, 1, i, j, k)) {
                    float s = ro[u] + ro[IDX(l, i, j + 1, k)] + ro[IDX(l, i, j, k + 1)] + ro[IDX(l, i, j + 1, k + 1)];
                    l->b[1][u] = -C->GX * s / 4.0;
                }
                if (valid(l, 2, i, j, k)) {
                    float s = ro[u] + ro[IDX(l, i + 1, j, k)] + ro[IDX(l, i, j, k + 1)] + ro[IDX(l, i + 1, j, k + 1)];
                    l->b[2][u] = -C->GY * s / 4.0;
                }
                if (valid(l, 3, i, j, k)) {
                    float s = ro[u] + ro[IDX(l, i, j + 1, k)] + ro[IDX(l, i + 1, j, k)] + ro[IDX(l, i + 1, j + 1, k)];
                    l->b[3][u] = -C->GZ * s / 4.0;
                }
            }
    for (k = 0; k < l->nz; k++)
        for (i = 0; i < l->nx; i++)
            for (j = 0; j < l->ny; j++) {
                long u = IDX(l, i, j, k);
                int c;
                for (c = 0; c < 4; c++)
                    if (is_bc(l, u, c)) l->b[c][u] = C->bondv1[2 * C->bondm[u * 4 + c]];
            }
    return coarse_factor(C);
}

/* Solve from the current x (zero after create) to rel residual tol.
 * restart == 0: plain defect correction x += V(b - A x);
 * restart >= 1: GCR(restart) with the V-cycle as preconditioner.
 * Returns iterations used; hist[0..it] receives relative residuals. */
static void vec_zero(double **v, long n) { int c; for (c = 0; c < 4; c++) memset(v[c], 0, sizeof(double) * n); }
static double vec_dot(double **a, double **b, long n)
{
    double s = 0; long u; int c;
    for (c = 0; c < 4; c++) {
#pragma omp parallel for reduction(+ : s) schedule(static)
        for (u = 0; u < n; u++) s += a[c][u] * b[c][u];
    }
    return s;
}
static void vec_axpy(double **y, double a, double **x, long n)
{
    long u; int c;
    for (c = 0; c < 4; c++) {
#pragma omp parallel for schedule(static)
        for (u = 0; u < n; u++) y[c][u] += a * x[c][u];
    }
}
static void vec_copy(double **y, double **x, long n) { int c; for (c = 0; c < 4; c++) memcpy(y[c], x[c], sizeof(double) * n); }
static void zero_pin_row(p2o_level *l, double **v) { if (l->pin >= 0) v[0][l->pin] = 0; }

/* z = V(r): one V-cycle from zero for right-hand side r (level 0). */
static void precond(p2o_ctx *C, double **r, double **z)
{
    p2o_level *l = &C->L[0];
    double *sb[4], *sx[4];
    int c;
    for (c = 0; c < 4; c++) { sb[c] = l->b[c]; sx[c] = l->x[c]; l->b[c] = r[c]; l->x[c] = z[c]; }
    vec_zero(l->x, l->n);
    vcycle(C);
    for (c = 0; c < 4; c++) { l->b[c] = sb[c]; l->x[c] = sx[c]; }
}

/* q = A z (level 0, BC rows x - koef x_t, pin cell as continuity). */
static void apply_A(p2o_ctx *C, double **z, double **q)
{
    p2o_level *l = &C->L[0];
    double *sb[4], *sx[4], *sr[4];
    int c;
    long u;
    for (c = 0; c < 4; c++) { sb[c] = l->b[c]; sx[c] = l->x[c]; sr[c] = l->r[c]; l->b[c] = calloc(l->n, sizeof(double)); l->x[c] = z[c]; l->r[c] = q[c]; }
    residual(C, 0);
    for (c = 0; c < 4; c++) { for (u = 0; u < l->n; u++) q[c][u] = -q[c][u]; free(l->b[c]); l->b[c] = sb[c]; l->x[c] = sx[c]; l->r[c] = sr[c]; }
}

int p2o_zero_pin = 0;
int p2o_solve(void *h, double tol, int maxit, int restart, double *hist)
{
    p2o_ctx *C = h;
    p2o_level *l = &C->L[0];
    long n = l->n;
    int it = 0, c, m = restart > 0 ? restart : 1, k, j;
    double rel, **Z, **Q, *r[4], *qq = calloc(m, sizeof(double));
    Z = calloc((size_t)m * 4, sizeof(double *));
    Q = calloc((size_t)m * 4, sizeof(double *));
    for (k = 0; k < m * 4; k++) { Z[k] = calloc(n, sizeof(double)); Q[k] = calloc(n, sizeof(double)); }
    for (c = 0; c < 4; c++) r[c] = calloc(n, sizeof(double));
    rel = rel_residual(C, NULL, NULL);
    if (hist) hist[0] = rel;
    k = 0;
    while (rel > tol && it < maxit) {
        double **z = &Z[k * 4], **q = &Q[k * 4], alpha;
        residual(C, 0);
        vec_copy(r, l->r, n);
        if (p2o_zero_pin) zero_pin_row(l, r);
        precond(C, r, z);
        if (restart == 0) {
            vec_axpy(l->x, 1.0, z, n);
        } else {
            apply_A(C, z, q);
            if (p2o_zero_pin) zero_pin_row(l, q);
            for (j = 0; j < k; j++) {
                double beta = vec_dot(q, &Q[j * 4], n) / qq[j];
                vec_axpy(q, -beta, &Q[j * 4], n);
                vec_axpy(z, -beta, &Z[j * 4], n);
            }
            qq[k] = vec_dot(q, q, n);
            alpha = vec_dot(r, q, n) / qq[k];
            vec_axpy(l->x, alpha, z, n);
            k = (k + 1) % m;
        }
        rel = rel_residual(C, NULL, NULL);
        it++;
        if (hist) hist[it] = rel;
        if (!(rel == rel)) break;
    }
    normalize_pressure(C, 0);
    for (k = 0; k < m * 4; k++) { free(Z[k]); free(Q[k]); }
    free(Z); free(Q); free(qq);
    for (c = 0; c < 4; c++) free(r[c]);
    return it;
}

/* Level-0 solution in the node layout (entries that are not unknowns are 0). */
void p2o_get_solution(void *h, double *pr, double *vx, double *vy, double *vz)
{
    p2o_ctx *C = h;
    p2o_level *l = &C->L[0];
    int i, j, k;
    for (k = 0; k < l->nz; k++)
        for (i = 0; i < l->nx; i++)
            for (j = 0; j < l->ny; j++) {
                long u = IDX(l, i, j, k);
                pr[u] = valid(l, 0, i, j, k) ? l->x[0][u] : 0;
                vx[u] = valid(l, 1, i, j, k) ? l->x[1][u] : 0;
                vy[u] = valid(l, 2, i, j, k) ? l->x[2][u] : 0;
                vz[u] = valid(l, 3, i, j, k) ? l->x[3][u] : 0;
            }
}

void p2o_set_solution(void *h, const double *pr, const double *vx, const double *vy, const double *vz)
{
    p2o_ctx *C = h;
    p2o_level *l = &C->L[0];
    memcpy(l->x[0], pr, sizeof(double) * l->n);
    memcpy(l->x[1], vx, sizeof(double) * l->n);
    memcpy(l->x[2], vy, sizeof(double) * l->n);
    memcpy(l->x[3], vz, sizeof(double) * l->n);
}

/* A x for an arbitrary level-li vector in the interleaved [P,Vx,Vy,Vz] layout
 * (BC rows: x - koef x_t; ghosts: x) — compared against the reference's row store. */
void p2o_apply(void *h, int li, const double *xin, double *yout)
{
    p2o_ctx *C = h;
    p2o_level *l = &C->L[li];
    double *save[4];
    int c, i, j, k;
    for (c = 0; c < 4; c++) {
        long u;
        save[c] = l->x[c];
        l->x[c] = malloc(sizeof(double) * l->n);
        for (u = 0; u < l->n; u++) l->x[c][u] = xin[u * 4 + c];
    }
    for (k = 0; k < l->nz; k++)
        for (i = 0; i < l->nx; i++)
            for (j = 0; j < l->ny; j++) {
                long u = IDX(l, i, j, k);
                for (c = 0; c < 4; c++) {
                    double a;
                    if (!valid(l, c, i, j, k)) { a = l->x[c][u]; }
                    else if (l->bcmask[u] & (1 << c)) {
                        double cst, koef; long tn; int tc;
                        bc_of(C, li, u, c, &cst, &koef, &tn, &tc);
                        a = l->x[c][u] - (tn >= 0 ? koef * l->x[tc][tn] : 0.0);
                    } else if (c == 0) a = row_p(l, i, j, k);
                    else if (c == 1) a = row_vx(l, i, j, k, NULL);
                    else if (c == 2) a = row_vy(l, i, j, k, NULL);
                    else a = row_vz(l, i, j, k, NULL);
                    yout[u * 4 + c] = a;
                }
            }
    for (c = 0; c < 4; c++) { free(l->x[c]); l->x[c] = save[c]; }
}

void p2o_rhs(void *h, double *b)
{
    p2o_ctx *C = h;
    p2o_level *l = &C->L[0];
    long u;
    int c;
    for (u = 0; u < l->n; u++)
        for (c = 0; c < 4; c++) {
            int i = (int)((u / l->ny) % l->nx), j = (int)(u % l->ny), k = (int)(u / ((long)l->nx * l->ny));
            if (!valid(l, c, i, j, k)) b[u * 4 + c] = 0;
            else if ((l->bcmask[u] & (1 << c)) && !is_bc(l, u, c)) b[u * 4 + c] = l->pinval;
            else b[u * 4 + c] = l->b[c][u];
        }
}

void p2o_level_fields(void *h, int li, float *nu, float *ro, double *ec)
{
    p2o_ctx *C = h;
    p2o_level *l = &C->L[li];
    memcpy(nu, l->nu, sizeof(float) * l->n);
    memcpy(ro, l->ro, sizeof(float) * l->n);
    memcpy(ec, l->ec, sizeof(double) * l->n);
}

double p2o_rel_residual(void *h)
{
    return rel_residual((p2o_ctx *)h, NULL, NULL);
}

/* ---------------------------------------------------------------------- */
/* Marker -> node interpolation (ronurecalc, mark3mg.c:630-1133), single   */
/* thread, with the reference's float accumulators and double weights.     */
static long serch(const double *g, long n, double x)
{
    long m, a = 0, b = n - 1;
    do {
        m = (a + b) / 2;
        if (g[m] > x) b = m; else a = m;
    } while (b - a > 1);
    if (a > n - 2) a = n - 2;
    return a;
}

/* In/out: nu, ro, nxx, nxy, nxz, nyz (float[nodenum]); nodes without
 * markers keep their input value (then clamped), as in the reference. */
void p2o_ronurecalc(int nx, int ny, int nz, const double *gx, const double *gy, const double *gz,
                    long nmark, const float *mx, const float *my, const float *mz, const signed char *mt,
                    const double *markn0, const double *markro, double nubeg, double nuend, double nukoef,
                    int viscmod, float *nu, float *ro, float *nxx, float *nxy, float *nxz, float *nyz,
                    const double *markn1, const double *marknu, const double *markmm, const double *val1)
{
    long nn = (long)nx * ny * nz, mm, v;
    double xsize = gx[nx - 1], ysize = gy[ny - 1], zsize = gz[nz - 1];
    long xy = (long)nx * ny;
    float *A[6];
    double *W[6];
    int q;
    for (q = 0; q < 6; q++) { A[q] = calloc(nn, sizeof(float)); W[q] = calloc(nn, sizeof(double)); }
    /* A/W order: 0 ro, 1 nu, 2 nxx, 3 nxy, 4 nxz, 5 nyz */
    for (mm = 0; mm < nmark; mm++) {
        double mnu, mro, dx, dy, dz;
        long m10, m20, m30, m1, m2, m3;
        int t = mt[mm];
        if (!(mx[mm] > 0 && my[mm] > 0 && mz[mm] > 0 && mx[mm] < xsize && my[mm] < ysize && mz[mm] < zsize && t < 50)) continue;
        mnu = markn0[t];
        /* power-law rock (viscalc, mark3mg.c:1479-1498) when the tables are given */
        if (val1 && t <= 20 && markn0[t] != markn1[t]) {
            double n = markmm[t];
            mnu = marknu[t] * pow(val1[mm] / 1.0, (1 - n) / n);
            if (mnu < markn0[t]) mnu = markn0[t];
            if (mnu > markn1[t]) mnu = markn1[t];
        }
        mro = markro[t];
        if (mnu < nubeg) mnu = nubeg;
        if (mnu > nuend) mnu = nuend;
        m10 = serch(gx, nx, (double)mx[mm]);
        m20 = serch(gy, ny, (double)my[mm]);
        m30 = serch(gz, nz, (double)mz[mm]);
        dx = gx[m10 + 1] - gx[m10];
        dy = gy[m20 + 1] - gy[m20];
        dz = gz[m30 + 1] - gz[m30];
        for (m3 = m30; m3 <= m30 + 1; m3++) {
            double ddz = 1.0 - fabs((gz[m3] - mz[mm]) / dz);
            for (m1 = m10; m1 <= m10 + 1; m1++) {
                double ddx = 1.0 - fabs((gx[m1] - mx[mm]) / dx);
                for (m2 = m20; m2 <= m20 + 1; m2++) {
                    double ddy = 1.0 - fabs((gy[m2] - my[mm]) / dy);
                    double swt = ddx * ddy * ddz, f, s1;
                    long m4 = m3 * xy + m1 * ny + m2;
                    f = viscmod == 0 ? mnu : viscmod == 1 ? log(mnu) : 1.0 / mnu;
                    if (ddx > nukoef && ddy > nukoef && ddz > nukoef) { A[1][m4] += f * swt; W[1][m4] += swt; }
                    if (m1 > m10 && m2 > m20 && m3 > m30) {
                        s1 = 8.0 * (0.5 - fabs(ddx - 0.5)) * (0.5 - fabs(ddy - 0.5)) * (0.5 - fabs(ddz - 0.5));
                        A[2][m4] += f * s1; W[2][m4] += s1;
                    }
                    if (m3 == m30 && ddx > 0.5 && ddy > 0.5) {
                        s1 = 8.0 * (ddx - 0.5) * (ddy - 0.5) * (0.5 - fabs(ddz - 0.5));
                        A[3][m4] += f * s1; W[3][m4] += s1;
                    }
                    if (m2 == m20 && ddx > 0.5 && ddz > 0.5) {
                        s1 = 8.0 * (ddx - 0.5) * (0.5 - fabs(ddy - 0.5)) * (ddz - 0.5);
                        A[4][m4] += f * s1; W[4][m4] += s1;
                    }
                    if (m1 == m10 && ddy > 0.5 && ddz > 0.5) {
                        s1 = 8.0 * (0.5 - fabs(ddx - 0.5)) * (ddy - 0.5) * (ddz - 0.5);
                        A[5][m4] += f * s1; W[5][m4] += s1;
                    }
                    if (ddx > 0.5 && ddy > 0.5 && ddz > 0.5) {
                        s1 = 8.0 * (ddx - 0.5) * (ddy - 0.5) * (ddz - 0.5);
                        A[0][m4] += mro * s1; W[0][m4] += s1;
                    }
                }
            }
        }
    }
    for (v = 0; v < nn; v++) {
        float *out[6];
        out[0] = ro; out[1] = nu; out[2] = nxx; out[3] = nxy; out[4] = nxz; out[5] = nyz;
        for (q = 0; q < 6; q++) {
            if (W[q][v] > 0) {
                /* the reference sums per-thread float buffers into a float array first */
                float s = 0.0f;
                s += A[q][v];
                if (q == 0) out[q][v] = (float)(s / W[q][v]);
                else {
                    out[q][v] = (float)(s / W[q][v]);
                    if (viscmod == 1) out[q][v] = (float)exp(out[q][v]);
                    if (viscmod == 2) out[q][v] = (float)(1.0 / out[q][v]);
                }
            }
            if (q > 0) {
                if (out[q][v] < nubeg) out[q][v] = (float)nubeg;
                if (out[q][v] > nuend) out[q][v] = (float)nuend;
            }
        }
    }
    for (q = 0; q < 6; q++) { free(A[q]); free(W[q]); }
}

/* ---------------------------------------------------------------------- */
/* Marker advection (movemark, mark3mg.c:174-629, non-periodic box) with   */
/* the staggered velocity interpolation vxyzcalc1 (mark3mg.c:2963-3243).   */
typedef struct {
    const double *g[3];
    long n[3];
    double size[3];
} mv_grid;

/* weights along the component's own axis: node interval of the cell */
static void mv_node_axis(const double *g, long n, long m, double x, long *lo, double *w0, double *w1)
{
    long a = m;
    double d;
    if (a < 0) a = 0;
    if (a > n - 2) a = n - 2;
    d = g[a + 1] - g[a];
    *lo = a;
    *w0 = 1.0 - (-((g[a] - x) / d));
    *w1 = 1.0 - (g[a + 1] - x) / d;
}

/* weights along a cross axis: between cell mid-points, the point clamped
 * onto the first or last mid-point (mark3mg.c:2988-3024) */
static void mv_mid_axis(const double *g, long n, long m, double x, long *lo, double *w0, double *w1)
{
    long a = m;
    double X = x, d;
    if (X < (g[a] + g[a + 1]) / 2.0) a -= 1;
    if (a < 0) { a = 0; X = (g[0] + g[1]) / 2.0; }
    if (a > n - 3) { a = n - 3; X = (g[a + 1] + g[a + 2]) / 2.0; }
    d = (g[a + 2] - g[a]) / 2.0;
    *lo = a;
    *w0 = 1.0 - (-(((g[a] + g[a + 1]) / 2.0 - X) / d));
    *w1 = 1.0 - ((g[a + 1] + g[a + 2]) / 2.0 - X) / d;
}

static void mv_velocity(const mv_grid *G, const float *const v[3], double x, double y, double z, double out[3])
{
    double p[3], w[3][2];
    long cell[3], lo[3], nxy = G->n[0] * G->n[1];
    int comp, a, b, c;
    p[0] = x; p[1] = y; p[2] = z;
    for (a = 0; a < 3; a++) {
        if (p[a] < 0) p[a] = 0;
        if (p[a] > G->size[a]) p[a] = G->size[a];
        cell[a] = serch(G->g[a], G->n[a], p[a]);
    }
    for (comp = 0; comp < 3; comp++) {
        double sum = 0;
        for (a = 0; a < 3; a++) {
            if (a == comp) mv_node_axis(G->g[a], G->n[a], cell[a], p[a], &lo[a], &w[a][0], &w[a][1]);
            else mv_mid_axis(G->g[a], G->n[a], cell[a], p[a], &lo[a], &w[a][0], &w[a][1]);
        }
        /* z outer, x, y inner, as the three loops of vxyzcalc1 */
        for (c = 0; c < 2; c++)
            for (a = 0; a < 2; a++)
                for (b = 0; b < 2; b++)
                    sum += v[comp][(lo[2] + c) * nxy + (lo[0] + a) * G->n[1] + lo[1] + b] * (w[0][a] * w[1][b] * w[2][c]);
        out[comp] = sum;
    }
}

/* markmod 1: velocity at the marker; 2: fourth-order Runge-Kutta.  Markers
 * are moved when inside the box or, unless outgrid is 1, when their type is
 * below 50 or at least 100; outgrid 2 keeps the motion outside the box
 * orthogonal to the wall.  markk (may be NULL) is set to 0 for moved markers
 * of type below 100 that end outside the box (mark3mg.c:489-494). */
/* Strain rate at a point (epscalc1, mark3mg.c:3244-3642, non-periodic):
 * normal components from cell centres, exy/exz/eyz from edges. */
static void ep_centre(const double *g, long n, long m0, double x, long *lo, double *w0, double *w1)
{
    long m = m0;
    double X = x, d;
    if (X > (g[m] + g[m + 1]) / 2.0) m += 1;
    if (m < 1) { m = 1; X = (g[1] + g[0]) / 2.0; }
    if (m > n - 2) { m = n - 2; X = (g[m] + g[m + 1]) / 2.0; }
    d = (g[m + 1] - g[m - 1]) / 2.0;
    *lo = m;
    *w0 = 1.0 - (-(((g[m] + g[m - 1]) / 2.0 - X) / d));
    *w1 = 1.0 - ((g[m + 1] + g[m]) / 2.0 - X) / d;
}

static void ep_line(const double *g, long n, long m0, double x, long *lo, double *w0, double *w1)
{
    long m = m0;
    double X = x, d;
    if (m < 1) { m = 1; X = g[1]; }
    if (m > n - 3) { m = n - 3; X = g[m + 1]; }
    d = g[m + 1] - g[m];
    *lo = m;
    *w0 = 1.0 - (-((g[m] - X) / d));
    *w1 = 1.0 - (g[m + 1] - X) / d;
}

static void ep_mid(const double *g, long n, long m0, double x, long *lo, double *w0, double *w1)
{
    long m = m0;
    double X = x, d;
    if (X < (g[m] + g[m + 1]) / 2.0) m -= 1;
    if (m < 1) { m = 0; X = (g[0] + g[1]) / 2.0; }
    if (m > n - 3) { m = n - 3; X = (g[m + 1] + g[m + 2]) / 2.0; }
    d = (g[m + 2] - g[m]) / 2.0;
    *lo = m;
    *w0 = 1.0 - (-(((g[m] + g[m + 1]) / 2.0 - X) / d));
    *w1 = 1.0 - ((g[m + 1] + g[m + 2]) / 2.0 - X) / d;
}

static double ep_sum(const float *f, const long lo[3], double w[3][2], long nxy, long ny)
{
    double s = 0;
    int a, b, c;
    for (c = 0; c < 2; c++)
        for (a = 0; a < 2; a++)
            for (b = 0; b < 2; b++)
                s += f[(lo[2] + c) * nxy + (lo[0] + a) * ny + lo[1] + b] * (w[0][a] * w[1][b] * w[2][c]);
    return s;
}

/* kind per axis: 0 centre, 1 line, 2 mid */
static double ep_field(const mv_grid *G, const float *f, const long cell[3], const double p[3], const int kind[3])
{
    long lo[3];
    double w[3][2];
    int a;
    for (a = 0; a < 3; a++) {
        if (kind[a] == 0) ep_centre(G->g[a], G->n[a], cell[a], p[a], &lo[a], &w[a][0], &w[a][1]);
        else if (kind[a] == 1) ep_line(G->g[a], G->n[a], cell[a], p[a], &lo[a], &w[a][0], &w[a][1]);
        else ep_mid(G->g[a], G->n[a], cell[a], p[a], &lo[a], &w[a][0], &w[a][1]);
    }
    return ep_sum(f, lo, w, G->n[0] * G->n[1], G->n[1]);
}

/* second invariant of the strain rate at (x, y, z), as movemark forms val1 */
static double ep_invariant(const mv_grid *G, const float *const e[6], double x, double y, double z)
{
    static const int kc[3] = {0, 0, 0}, kxy[3] = {1, 1, 2}, kxz[3] = {1, 2, 1}, kyz[3] = {2, 1, 1};
    double p[3], ee[6];
    long cell[3];
    int a;
    p[0] = x; p[1] = y; p[2] = z;
    for (a = 0; a < 3; a++) {
        if (p[a] < 0) p[a] = 0;
        if (p[a] > G->size[a]) p[a] = G->size[a];
        cell[a] = serch(G->g[a], G->n[a], p[a]);
    }
    for (a = 0; a < 3; a++) ee[a] = ep_field(G, e[a], cell, p, kc);
    ee[3] = ep_field(G, e[3], cell, p, kxy);
    ee[4] = ep_field(G, e[4], cell, p, kxz);
    ee[5] = ep_field(G, e[5], cell, p, kyz);
    return pow(0.5 * (ee[0] * ee[0] + ee[1] * ee[1] + ee[2] * ee[2]) + ee[3] * ee[3] + ee[4] * ee[4] + ee[5] * ee[5],
               0.5);
}

/* strain: exx..eyz node fields or NULL; then val1 (per marker, written for
 * moved markers) and marke (brittle strain, in/out) are updated as movemark
 * does (mark3mg.c:218-220, 358-410, 488; in markmod 1 the marker's own
 * invariant stands for the stage average). */
void p2o_movemark(int nx, int ny, int nz, const double *gx, const double *gy, const double *gz, const float *vx,
                  const float *vy, const float *vz, double dt, int markmod, int outgrid, long nmark, float *mx,
                  float *my, float *mz, const signed char *mt, float *markk, const float *const *strain,
                  double *val1, float *marke)
{
    mv_grid G;
    const float *v[3];
    long q;
    int a;
    G.g[0] = gx; G.g[1] = gy; G.g[2] = gz;
    G.n[0] = nx; G.n[1] = ny; G.n[2] = nz;
    G.size[0] = gx[nx - 1]; G.size[1] = gy[ny - 1]; G.size[2] = gz[nz - 1];
    v[0] = vx; v[1] = vy; v[2] = vz;
    for (q = 0; q < nmark; q++) {
        double k1[3], k2[3], k3[3], k4[3], vel[3];
        double x0 = mx[q], y0 = my[q], z0 = mz[q];
        int t = mt[q];
        int inside = mx[q] >= 0 && my[q] >= 0 && mz[q] >= 0 && x0 <= G.size[0] && y0 <= G.size[1] && z0 <= G.size[2];
        if (!(inside || (outgrid != 1 && (t < 50 || t >= 100)))) continue;
        int brittle = 0;
        double e1 = 0, ee0 = 0;
        mv_velocity(&G, v, x0, y0, z0, k1);
        if (strain) {
            e1 = ep_invariant(&G, strain, x0, y0, z0);
            val1[q] = e1;
            brittle = marke[q] > 0;
            ee0 = e1;
        }
        if (markmod == 1) {
            for (a = 0; a < 3; a++) vel[a] = k1[a];
        } else {
            double e2 = 0, e3 = 0, e4 = 0;
            mv_velocity(&G, v, x0 + k1[0] * dt / 2.0, y0 + k1[1] * dt / 2.0, z0 + k1[2] * dt / 2.0, k2);
            if (brittle) e2 = ep_invariant(&G, strain, x0 + k1[0] * dt / 2.0, y0 + k1[1] * dt / 2.0, z0 + k1[2] * dt / 2.0);
            mv_velocity(&G, v, x0 + k2[0] * dt / 2.0, y0 + k2[1] * dt / 2.0, z0 + k2[2] * dt / 2.0, k3);
            if (brittle) e3 = ep_invariant(&G, strain, x0 + k2[0] * dt / 2.0, y0 + k2[1] * dt / 2.0, z0 + k2[2] * dt / 2.0);
            mv_velocity(&G, v, x0 + k3[0] * dt, y0 + k3[1] * dt, z0 + k3[2] * dt, k4);
            if (brittle) {
                e4 = ep_invariant(&G, strain, x0 + k3[0] * dt, y0 + k3[1] * dt, z0 + k3[2] * dt);
                ee0 = (e1 + 2.0 * e2 + 2.0 * e3 + e4) / 6.0;
            }
            for (a = 0; a < 3; a++) vel[a] = (k1[a] + 2.0 * k2[a] + 2.0 * k3[a] + k4[a]) / 6.0;
        }
        if (outgrid == 2) {
            if (mx[q] < 0 || x0 > G.size[0]) vel[1] = vel[2] = 0;
            if (my[q] < 0 || y0 > G.size[1]) vel[0] = vel[2] = 0;
            if (mz[q] < 0 || z0 > G.size[2]) vel[0] = vel[1] = 0;
        }
        mx[q] = (float)(x0 + dt * vel[0]);
        my[q] = (float)(y0 + dt * vel[1]);
        mz[q] = (float)(z0 + dt * vel[2]);
        if (brittle && t < 100) marke[q] += (float)(ee0 * dt);
        if (markk && t < 100 &&
            (mx[q] < 0 || my[q] < 0 || mz[q] < 0 || (double)mx[q] > G.size[0] || (double)my[q] > G.size[1] ||
             (double)mz[q] > G.size[2]))
            markk[q] = 0;
    }
}

/* ---------------------------------------------------------------------- */
/* Post-solve stresses and strain rates (vpiterate, move3mgNew.c:2908-3038, */
/* value mode of sxxcalc..syzcalc 3-794), non-periodic box.                */
static double st_nu(float v, double nubeg, double nuend)
{
    double n = v;
    if (n > nuend) n = nuend;
    if (n < nubeg) n = nubeg;
    return n;
}

/* float difference first, then scaled in double */
static double st_d(float a, float b, double kf)
{
    float d = a - b;
    return (double)d * kf;
}

static void st_put(float **out, int q, long u, double left, double nueff)
{
    out[6 + q][u] = (float)left;
    out[q][u] = (float)(2.0 * nueff * left);
}

/* out: sxx syy szz sxy sxz syz exx eyy ezz exy exz eyz (float[nodenum]);
 * positions the reference does not write are left alone. */
void p2o_stress_strain(int nx, int ny, int nz, const double *gx, const double *gy, const double *gz, const float *vx,
                       const float *vy, const float *vz, const float *nxx, const float *nxy, const float *nxz,
                       const float *nyz, double nubeg, double nuend, float **out)
{
    long nxy_ = (long)nx * ny, u;
    int i, j, k;
    for (k = 0; k < nz; k++)
        for (i = 0; i < nx; i++)
            for (j = 0; j < ny; j++) {
                u = k * nxy_ + (long)i * ny + j;
                if (i > 0 && j > 0 && k > 0) {
                    long v0 = u - nxy_ - ny - 1;
                    double xkf = 1.0 / (gx[i] - gx[i - 1]), ykf = 1.0 / (gy[j] - gy[j - 1]);
                    double zkf = 1.0 / (gz[k] - gz[k - 1]);
                    double dx = st_d(vx[v0 + ny], vx[v0], xkf), dy = st_d(vy[v0 + 1], vy[v0], ykf);
                    double dz = st_d(vz[v0 + nxy_], vz[v0], zkf);
                    double nu = st_nu(nxx[u], nubeg, nuend);
                    st_put(out, 0, u, dx - (dx + dy + dz) / 3.0, nu);
                    st_put(out, 1, u, dy - (dx + dy + dz) / 3.0, nu);
                    st_put(out, 2, u, dz - (dx + dy + dz) / 3.0, nu);
                }
                if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k < nz - 1) {
                    double xkf = 1.0 / (gx[i + 1] - gx[i - 1]), ykf = 1.0 / (gy[j + 1] - gy[j - 1]);
                    st_put(out, 3, u, st_d(vx[u], vx[u - 1], ykf) + st_d(vy[u], vy[u - ny], xkf),
                           st_nu(nxy[u], nubeg, nuend));
                }
                if (i > 0 && i < nx - 1 && k > 0 && k < nz - 1 && j < ny - 1) {
                    double xkf = 1.0 / (gx[i + 1] - gx[i - 1]), zkf = 1.0 / (gz[k + 1] - gz[k - 1]);
                    st_put(out, 4, u, st_d(vx[u], vx[u - nxy_], zkf) + st_d(vz[u], vz[u - ny], xkf),
                           st_nu(nxz[u], nubeg, nuend));
                }
                if (j > 0 && j < ny - 1 && k > 0 && k < nz - 1 && i < nx - 1) {
                    double ykf = 1.0 / (gy[j + 1] - gy[j - 1]), zkf = 1.0 / (gz[k + 1] - gz[k - 1]);
                    st_put(out, 5, u, st_d(vy[u], vy[u - nxy_], zkf) + st_d(vz[u], vz[u - 1], ykf),
                           st_nu(nyz[u], nubeg, nuend));
                }
            }
}

/* ---------------------------------------------------------------------- */
/* Effective bulk viscosity diagnostics (effbulkvisccalc mode 1,           */
/* mark3mg.c:2-150), in the reference's order and float/double mix.        */
/* in: ro nxx nxy nxz nyz exx eyy ezz exy exz eyz sxx syy szz sxy sxz syz;  */
/* out: eiin siin eiivp tau2 hsn nubulkn nubulk1..4, matrix[12], incl[12]; */
/* counts: numtot nummat numinc.                                          */
void p2o_effbulk(int nx, int ny, int nz, const float *const *in, double *out, long *counts)
{
    const float *ro = in[0], *nxx = in[1], *nxy = in[2], *nxz = in[3], *nyz = in[4];
    const float *exx = in[5], *eyy = in[6], *ezz = in[7], *exy = in[8], *exz = in[9], *eyz = in[10];
    const float *sxx = in[11], *syy = in[12], *szz = in[13], *sxy = in[14], *sxz = in[15], *syz = in[16];
    long m1, m2, m3, m4, v1[8], numtot = 0, numinc = 0, nummat = 0, sy = ny, sz = (long)nx * ny;
    double tau2 = 0, siin = 0, eiin = 0, eiivp = 0, hsn = 0, nubulkn = 0, ac[12] = {0}, ai[12] = {0};
    int q;
    for (m3 = 0; m3 < nz; m3++)
        for (m1 = 0; m1 < nx; m1++)
            for (m2 = 0; m2 < ny; m2++) {
                double Exy, Exz, Eyz, Sxy, Sxz, Syz, eiinloc, siinloc, eiivploc, hsnloc, *acc;
                float c[12];
                m4 = m3 * sz + m1 * sy + m2;
                if (!(ro[m4] > 1500 && m1 > 0 && m2 > 0 && m3 > 0)) continue;
                numtot += 1;
                nubulkn += 1 / nxx[m4];
                v1[0] = (m3 - 1) * sz + (m1 - 1) * sy + (m2 - 1); v1[1] = v1[0] + 1;
                v1[2] = v1[0] + sy; v1[3] = v1[2] + 1;
                v1[4] = v1[0] + sz; v1[5] = v1[4] + 1;
                v1[6] = v1[4] + sy; v1[7] = v1[6] + 1;
                Exy = (exy[v1[0]] * exy[v1[0]] + exy[v1[1]] * exy[v1[1]] + exy[v1[2]] * exy[v1[2]] + exy[v1[3]] * exy[v1[3]]) / 4;
                Exz = (exz[v1[0]] * exz[v1[0]] + exz[v1[2]] * exz[v1[2]] + exz[v1[4]] * exz[v1[4]] + exz[v1[6]] * exz[v1[6]]) / 4;
                Eyz = (eyz[v1[0]] * eyz[v1[0]] + eyz[v1[1]] * eyz[v1[1]] + eyz[v1[4]] * eyz[v1[4]] + eyz[v1[5]] * eyz[v1[5]]) / 4;
                Sxy = (sxy[v1[0]] * sxy[v1[0]] + sxy[v1[1]] * sxy[v1[1]] + sxy[v1[2]] * sxy[v1[2]] + sxy[v1[3]] * sxy[v1[3]]) / 4;
                Sxz = (sxz[v1[0]] * sxz[v1[0]] + sxz[v1[2]] * sxz[v1[2]] + sxz[v1[4]] * sxz[v1[4]] + sxz[v1[6]] * sxz[v1[6]]) / 4;
                Syz = (syz[v1[0]] * syz[v1[0]] + syz[v1[1]] * syz[v1[1]] + syz[v1[4]] * syz[v1[4]] + syz[v1[5]] * syz[v1[5]]) / 4;
                eiinloc = pow(0.5 * (exx[m4] * exx[m4] + eyy[m4] * eyy[m4] + ezz[m4] * ezz[m4]) + Exy + Exz + Eyz, 0.5);
                siinloc = pow(0.5 * (sxx[m4] * sxx[m4] + syy[m4] * syy[m4] + szz[m4] * szz[m4]) + Sxy + Sxz + Syz, 0.5);
                Exy = (pow(sxy[v1[0]] / 2 / nxy[v1[0]], 2) + pow(sxy[v1[1]] / 2 / nxy[v1[1]], 2) +
                       pow(sxy[v1[2]] / 2 / nxy[v1[2]], 2) + pow(sxy[v1[3]] / 2 / nxy[v1[3]], 2)) / 4;
                Exz = (pow(sxz[v1[0]] / 2 / nxz[v1[0]], 2) + pow(sxz[v1[2]] / 2 / nxz[v1[2]], 2) +
                       pow(sxz[v1[4]] / 2 / nxz[v1[4]], 2) + pow(sxz[v1[6]] / 2 / nxz[v1[6]], 2)) / 4;
                Eyz = (pow(syz[v1[0]] / 2 / nyz[v1[0]], 2) + pow(syz[v1[1]] / 2 / nyz[v1[1]], 2) +
                       pow(syz[v1[4]] / 2 / nyz[v1[4]], 2) + pow(syz[v1[5]] / 2 / nyz[v1[5]], 2)) / 4;
                eiivploc = pow(0.5 * (pow(sxx[m4] / 2 / nxx[m4], 2) + pow(syy[m4] / 2 / nxx[m4], 2) +
                                      pow(szz[m4] / 2 / nxx[m4], 2)) + Exy + Exz + Eyz, 0.5);
                Sxy = (sxy[v1[0]] * sxy[v1[0]] / 2 / nxy[v1[0]] + sxy[v1[1]] * sxy[v1[1]] / 2 / nxy[v1[1]] +
                       sxy[v1[2]] * sxy[v1[2]] / 2 / nxy[v1[2]] + sxy[v1[3]] * sxy[v1[3]] / 2 / nxy[v1[3]]) / 4;
                Sxz = (sxz[v1[0]] * sxz[v1[0]] / 2 / nxz[v1[0]] + sxz[v1[2]] * sxz[v1[2]] / 2 / nxz[v1[2]] +
                       sxz[v1[4]] * sxz[v1[4]] / 2 / nxz[v1[4]] + sxz[v1[6]] * sxz[v1[6]] / 2 / nxz[v1[6]]) / 4;
                Syz = (syz[v1[0]] * syz[v1[0]] / 2 / nyz[v1[0]] + syz[v1[1]] * syz[v1[1]] / 2 / nyz[v1[1]] +
                       syz[v1[4]] * syz[v1[4]] / 2 / nyz[v1[4]] + syz[v1[5]] * syz[v1[5]] / 2 / nyz[v1[5]]) / 4;
                hsnloc = (sxx[m4] * sxx[m4] + syy[m4] * syy[m4] + szz[m4] * szz[m4]) / 2 / nxx[m4] + 2.0 * (Sxy + Sxz + Syz);
                eiin += eiinloc;
                tau2 += nxx[m4] * eiinloc;
                siin += siinloc;
                hsn += hsnloc;
                eiivp += eiivploc;
                c[0] = exx[m4]; c[1] = eyy[m4]; c[2] = ezz[m4];
                c[3] = (exy[v1[0]] + exy[v1[1]] + exy[v1[2]] + exy[v1[3]]) / 4;
                c[4] = (exz[v1[0]] + exz[v1[2]] + exz[v1[4]] + exz[v1[6]]) / 4;
                c[5] = (eyz[v1[0]] + eyz[v1[1]] + eyz[v1[4]] + eyz[v1[5]]) / 4;
                c[6] = sxx[m4]; c[7] = syy[m4]; c[8] = szz[m4];
                c[9] = (sxy[v1[0]] + sxy[v1[1]] + sxy[v1[2]] + sxy[v1[3]]) / 4;
                c[10] = (sxz[v1[0]] + sxz[v1[2]] + sxz[v1[4]] + sxz[v1[6]]) / 4;
                c[11] = (syz[v1[0]] + syz[v1[1]] + syz[v1[4]] + syz[v1[5]]) / 4;
                if (ro[m4] > 3850) { numinc += 1; acc = ai; } else { nummat += 1; acc = ac; }
                for (q = 0; q < 12; q++) acc[q] += c[q];
            }
    eiin /= numtot; siin /= numtot; hsn /= numtot; eiivp /= numtot; nubulkn = numtot / nubulkn; tau2 /= numtot;
    for (q = 0; q < 12; q++) {
        if (nummat > 0) ac[q] /= nummat;
        if (numinc > 0) ai[q] /= numinc;
    }
    out[0] = eiin; out[1] = siin; out[2] = eiivp; out[3] = tau2; out[4] = hsn; out[5] = nubulkn;
    out[6] = tau2 / eiin; out[7] = hsn / 4 / eiin / eiin; out[8] = hsn / 4 / eiivp / eiivp; out[9] = siin / 2 / eiin;
    for (q = 0; q < 12; q++) { out[10 + q] = ac[q]; out[22 + q] = ai[q]; }
    counts[0] = numtot; counts[1] = nummat; counts[2] = numinc;
}

/* Debug/test helpers: sweeps of the level-0 smoother only; two-grid count. */
double p2o_smooth_only(void *h, int sweeps)
{
    p2o_ctx *C = h;
    smooth(C, 0, sweeps);
    return rel_residual(C, NULL, NULL);
}

/* Single transfers on interleaved [P,Vx,Vy,Vz] vectors of one level pair
 * (for pinning against the reference's vprestrict / vpprolong). */
void p2o_restrict(void *h, int lc, const double *fine_res, double *coarse_rhs, int compat)
{
    p2o_ctx *C = h;
    p2o_level *f = &C->L[lc - 1], *cl = &C->L[lc];
    long u;
    int c;
    double *sx[4];
    for (c = 0; c < 4; c++) sx[c] = cl->x[c];
    for (u = 0; u < f->n; u++)
        for (c = 0; c < 4; c++) f->r[c][u] = fine_res[u * 4 + c];
    p2o_compat = compat;
    restrict_level(C, lc);
    p2o_compat = 1;
    for (u = 0; u < cl->n; u++)
        for (c = 0; c < 4; c++) coarse_rhs[u * 4 + c] = cl->b[c][u];
    (void)sx;
}

void p2o_prolong(void *h, int lc, const double *coarse_x, double *fine_x)
{
    p2o_ctx *C = h;
    p2o_level *f = &C->L[lc - 1], *cl = &C->L[lc];
    long u;
    int c;
    for (u = 0; u < cl->n; u++)
        for (c = 0; c < 4; c++) cl->x[c][u] = coarse_x[u * 4 + c];
    for (u = 0; u < f->n; u++)
        for (c = 0; c < 4; c++) f->x[c][u] = fine_x[u * 4 + c];
    prolong_level(C, lc);
    for (u = 0; u < f->n; u++)
        for (c = 0; c < 4; c++) fine_x[u * 4 + c] = f->x[c][u];
}

/* ---------------------------------------------------------------------- */
/* Heat equation step (titerate, pardiso/heat3mg.c:292-829), single thread. */
/* Restated literally: the level-0 right-hand side heaterr mode 0 (6-291),  */
/* the step limit from maxtkstep (331-374), rocprestrict (1235-1332), the   */
/* implicit 7-point rows heaterr mode 1 and the boundary rows tbonderr      */
/* (841-893) stored as gausmat2 does (gaus3mg_SerieMG.c:312-365), the       */
/* damped lexicographic Gauss-Seidel gausmatt (1057-1120), trestrict        */
/* (1122-1233), tprolong (954-1054), the error heaterr mode 2 and the       */
/* marker temperatures with numerical diffusion (641-829, tkcalc1           */
/* pardiso/mark3mg.c:1212-1282).  Float arrays (tk, tk0, tk1, tk2, kt, cp,  */
/* ro, ht, et) and the float arithmetic of the reference's expressions on   */
/* them are kept.  The reference loops until the error is below HEATMIN     */
/* with no cap; here at most max_cycles batches of V-cycles run per step.   */
typedef struct {
    int nl;                        /* levels 0..nl-1 */
    int nx[MAXLEV], ny[MAXLEV], nz[MAXLEV];
    long off[MAXLEV], n[MAXLEV], tot;
    double *g[MAXLEV][3];
} ht_grid;

static void ht_grid_build(ht_grid *G, int nx, int ny, int nz, const double *gx, const double *gy, const double *gz,
                          int nl)
{
    int li, q, n2;
    long off = 0;
    G->nl = nl;
    for (li = 0; li < nl; li++) {
        int s = 1 << li;
        if (li == 0) { G->nx[0] = nx; G->ny[0] = ny; G->nz[0] = nz; }
        else {
            G->nx[li] = (G->nx[li - 1] - 5) / 2 + 5;
            G->ny[li] = (G->ny[li - 1] - 5) / 2 + 5;
            G->nz[li] = (G->nz[li - 1] - 5) / 2 + 5;
        }
        G->n[li] = (long)G->nx[li] * G->ny[li] * G->nz[li];
        G->off[li] = off;
        off += G->n[li];
        for (q = 0; q < 3; q++) {
            int n = q == 0 ? G->nx[li] : q == 1 ? G->ny[li] : G->nz[li], nf = q == 0 ? nx : q == 1 ? ny : nz;
            const double *g = q == 0 ? gx : q == 1 ? gy : gz;
            double *o = malloc(sizeof(double) * n);
            o[0] = g[0]; o[1] = g[1]; o[2] = g[2];
            o[n - 1] = g[nf - 1]; o[n - 2] = g[nf - 2]; o[n - 3] = g[nf - 3];
            for (n2 = 3; n2 < n - 3; n2++) o[n2] = g[(n2 - 2) * s + 2];
            G->g[li][q] = o;
        }
    }
    G->tot = off;
}

static void ht_grid_free(ht_grid *G)
{
    int li, q;
    for (li = 0; li < G->nl; li++)
        for (q = 0; q < 3; q++) free(G->g[li][q]);
}

/* coarse cell index of a fine line (heat3mg.c:979-990, 1160-1171, 1276-1287) */
static long ht_cmin(long m, long nf, long nc)
{
    long c = (m - 2) / 2 + 2;
    if (m < 3) c = m;
    if (m > nf - 4) c = nc - (nf - m);
    if (c > nc - 2) c = nc - 2;
    return c;
}

typedef struct {
    ht_grid G;
    const int *bct;                /* T boundary row number per node, all levels */
    const float *bondv1;
    const int *bondn1;
    float *kt, *cp, *ro;           /* all levels */
    double *sol0, *sol1, *fre0, *fre1, *val1;
    long *lin0, *pos0;
    int *num0;
    double t0koef, t1koef;
} ht_ctx;

/* Coarse level fields from the finer one: rocprestrict (heat3mg.c:1235-1332),
 * float accumulators with double weights as the reference's arrays are. */
static void ht_rocprestrict(ht_ctx *H, int lc)
{
    ht_grid *G = &H->G;
    int lf = lc - 1;
    long m1, m2, m3, u;
    for (u = G->off[lc]; u < G->off[lc] + G->n[lc]; u++) { H->cp[u] = 0; H->kt[u] = 0; H->ro[u] = 0; H->sol1[u] = 0; }
    for (m3 = 0; m3 < G->nz[lf]; m3++)
        for (m1 = 0; m1 < G->nx[lf]; m1++)
            for (m2 = 0; m2 < G->ny[lf]; m2++) {
                long m4 = G->off[lf] + m3 * G->nx[lf] * G->ny[lf] + m1 * G->ny[lf] + m2, m10, m20, m30;
                long c1 = ht_cmin(m1, G->nx[lf], G->nx[lc]), c2 = ht_cmin(m2, G->ny[lf], G->ny[lc]);
                long c3 = ht_cmin(m3, G->nz[lf], G->nz[lc]);
                double dx = G->g[lc][0][c1 + 1] - G->g[lc][0][c1], dy = G->g[lc][1][c2 + 1] - G->g[lc][1][c2];
                double dz = G->g[lc][2][c3 + 1] - G->g[lc][2][c3];
                for (m30 = c3; m30 <= c3 + 1; m30++) {
                    double ddz = 1.0 - fabs((G->g[lc][2][m30] - G->g[lf][2][m3]) / dz);
                    for (m10 = c1; m10 <= c1 + 1; m10++) {
                        double ddx = 1.0 - fabs((G->g[lc][0][m10] - G->g[lf][0][m1]) / dx);
                        for (m20 = c2; m20 <= c2 + 1; m20++) {
                            double ddy = 1.0 - fabs((G->g[lc][1][m20] - G->g[lf][1][m2]) / dy);
                            long m40 = G->off[lc] + m30 * G->nx[lc] * G->ny[lc] + m10 * G->ny[lc] + m20;
                            double swt = ddx * ddy * ddz;
                            H->cp[m40] += H->cp[m4] * swt;
                            H->kt[m40] += H->kt[m4] * swt;
                            H->ro[m40] += H->ro[m4] * swt;
                            H->sol1[m40] += swt;
                        }
                    }
                }
            }
    for (u = G->off[lc]; u < G->off[lc] + G->n[lc]; u++) {
        H->cp[u] /= H->sol1[u];
        H->kt[u] /= H->sol1[u];
        H->ro[u] /= H->sol1[u];
        H->sol1[u] = 0;
    }
}

/* trestrict (heat3mg.c:1122-1233) */
static void ht_restrict(ht_ctx *H, int lc)
{
    ht_grid *G = &H->G;
    int lf = lc - 1;
    long m1, m2, m3, u;
    for (u = G->off[lc]; u < G->off[lc] + G->n[lc]; u++) { H->fre1[u] = 0; H->sol1[u] = 0; }
    for (m3 = 0; m3 < G->nz[lf]; m3++)
        for (m1 = 0; m1 < G->nx[lf]; m1++)
            for (m2 = 0; m2 < G->ny[lf]; m2++) {
                long m4 = G->off[lf] + m3 * G->nx[lf] * G->ny[lf] + m1 * G->ny[lf] + m2, m10, m20, m30;
                long c1 = ht_cmin(m1, G->nx[lf], G->nx[lc]), c2 = ht_cmin(m2, G->ny[lf], G->ny[lc]);
                long c3 = ht_cmin(m3, G->nz[lf], G->nz[lc]);
                double dx = G->g[lc][0][c1 + 1] - G->g[lc][0][c1], dy = G->g[lc][1][c2 + 1] - G->g[lc][1][c2];
                double dz = G->g[lc][2][c3 + 1] - G->g[lc][2][c3];
                for (m30 = c3; m30 <= c3 + 1; m30++) {
                    double ddz = (G->g[lc][2][m30] - G->g[lf][2][m3]) / dz;
                    if (m30 == c3) ddz = -ddz;
                    ddz = 1.0 - ddz;
                    for (m10 = c1; m10 <= c1 + 1; m10++) {
                        double ddx = (G->g[lc][0][m10] - G->g[lf][0][m1]) / dx;
                        if (m10 == c1) ddx = -ddx;
                        ddx = 1.0 - ddx;
                        for (m20 = c2; m20 <= c2 + 1; m20++) {
                            double ddy = (G->g[lc][1][m20] - G->g[lf][1][m2]) / dy;
                            long m40 = G->off[lc] + m30 * G->nx[lc] * G->ny[lc] + m10 * G->ny[lc] + m20;
                            if (m20 == c2) ddy = -ddy;
                            ddy = 1.0 - ddy;
                            if (!H->bct[m40]) {
                                double swt = ddx * ddy * ddz;
                                H->fre1[m40] += H->fre0[m4] * swt;
                                H->sol1[m40] += swt;
                            }
                        }
                    }
                }
            }
    for (u = G->off[lc]; u < G->off[lc] + G->n[lc]; u++) {
        if (H->sol1[u]) { H->fre1[u] /= H->sol1[u]; H->sol1[u] = 0; }
        H->sol0[u] = 0;
    }
}

/* tprolong with ynreset 0 (heat3mg.c:954-1054) */
static void ht_prolong(ht_ctx *H, int lc)
{
    ht_grid *G = &H->G;
    int lf = lc - 1;
    long m1, m2, m3;
    for (m3 = 0; m3 < G->nz[lf]; m3++)
        for (m1 = 0; m1 < G->nx[lf]; m1++)
            for (m2 = 0; m2 < G->ny[lf]; m2++) {
                long m4 = G->off[lf] + m3 * G->nx[lf] * G->ny[lf] + m1 * G->ny[lf] + m2, m10, m20, m30;
                long c1, c2, c3;
                double dx, dy, dz;
                if (H->bct[m4]) continue;
                c1 = ht_cmin(m1, G->nx[lf], G->nx[lc]); c2 = ht_cmin(m2, G->ny[lf], G->ny[lc]);
                c3 = ht_cmin(m3, G->nz[lf], G->nz[lc]);
                dx = G->g[lc][0][c1 + 1] - G->g[lc][0][c1]; dy = G->g[lc][1][c2 + 1] - G->g[lc][1][c2];
                dz = G->g[lc][2][c3 + 1] - G->g[lc][2][c3];
                for (m30 = c3; m30 <= c3 + 1; m30++) {
                    double ddz = (G->g[lc][2][m30] - G->g[lf][2][m3]) / dz;
                    if (m30 == c3) ddz = -ddz;
                    ddz = 1.0 - ddz;
                    for (m10 = c1; m10 <= c1 + 1; m10++) {
                        double ddx = (G->g[lc][0][m10] - G->g[lf][0][m1]) / dx;
                        if (m10 == c1) ddx = -ddx;
                        ddx = 1.0 - ddx;
                        for (m20 = c2; m20 <= c2 + 1; m20++) {
                            double ddy = (G->g[lc][1][m20] - G->g[lf][1][m2]) / dy;
                            long m40 = G->off[lc] + m30 * G->nx[lc] * G->ny[lc] + m10 * G->ny[lc] + m20;
                            if (m20 == c2) ddy = -ddy;
                            ddy = 1.0 - ddy;
                            H->sol0[m4] += H->sol0[m40] * (ddx * ddy * ddz) * H->t1koef;
                        }
                    }
                }
            }
}

/* gausmatt (heat3mg.c:1057-1120) on the rows of one level */
static void ht_gausmatt(ht_ctx *H, int am, long mcmax, long mcmin)
{
    long m1;
    int m2, m3;
    for (m3 = 0; m3 < am; m3++)
        for (m1 = mcmin; m1 <= mcmax; m1++)
            if (H->num0[m1]) {
                double ival = -H->fre1[m1], ival1 = H->val1[H->pos0[m1]];
                for (m2 = 0; m2 < H->num0[m1]; m2++) ival += H->val1[H->pos0[m1] + m2] * H->sol0[H->lin0[H->pos0[m1] + m2]];
                H->sol0[m1] -= ival / ival1 * H->t0koef;
            }
    for (m1 = mcmin; m1 <= mcmax; m1++)
        if (H->num0[m1]) {
            double ival = H->fre1[m1];
            for (m2 = 0; m2 < H->num0[m1]; m2++) ival -= H->val1[H->pos0[m1] + m2] * H->sol0[H->lin0[H->pos0[m1] + m2]];
            H->fre0[m1] = ival;
        }
}

static void ht_row(ht_ctx *H, long u, int nn, const long *un, const double *ui, double rhs)
{
    int q;
    H->fre1[u] = rhs;
    H->pos0[u] = u * 7;
    H->num0[u] = nn;
    for (q = 0; q < nn; q++) { H->lin0[u * 7 + q] = un[q]; H->val1[u * 7 + q] = ui[q]; }
}

/* Inverse spacing factors of heaterr (heat3mg.c:21-24) */
#define HT_KF(g, m) (2.0 / ((g)[(m) + 1] - (g)[(m) - 1]))

/* dpar: timestep, maxtkstep, HEATMIN, t0koef, t1koef, heatdif, tdeep, zdeep, GX, GY, GZ
 * ipar: multicyct, frictyn, adiabyn, max_cycles, multittt[0][0..15], multittt[1][0..15]
 * se:   sxx, syy, szz, sxy, sxz, syz, exx, eyy, ezz, exy, exz, eyz (NULL: frictyn must be 0)
 * info: tktimestep, substeps, V-cycle batches, last error, min tk, max tk, status (0 ok, 1 cap reached),
 *       maxtkrate */
int p2o_titerate(int nx, int ny, int nz, const double *gx, const double *gy, const double *gz, int multinumt,
                 const int *bct, const float *bondv1, const int *bondn1, const double *dpar, const int *ipar,
                 float *tk, const float *kt0, const float *cp0, const float *ro0, const float *ht, const float *et,
                 const float *vx, const float *vy, const float *vz, const double *pr, const float *const *se,
                 long nmark, const float *markx, const float *marky, const float *markz, const signed char *markt,
                 float *markk, double *info)
{
    ht_ctx HC, *H = &HC;
    ht_grid *G = &H->G;
    long nxy = (long)nx * ny, nn = nxy * nz, u, m1, m2, m3, mk;
    double timestep = dpar[0], maxtkstep = dpar[1], heatmin = dpar[2], heatdif = dpar[5];
    double tdeep = dpar[6], zdeep = dpar[7], GXK = dpar[8], GYK = dpar[9], GZK = dpar[10];
    int multicyct = ipar[0], frictyn = ipar[1], adiabyn = ipar[2], maxcyc = ipar[3];
    double maxtkrate = 0, tktimestep = 1e30, tktimesum, tktimesum0, heatsum = 0, mintk = 1e30, maxtk = -1e30;
    float *tk0, *tk1, *tk2;
    int li, status = 0;
    long nsub = 0, ncyc = 0;
    const double *gl[3];
    mv_grid MG;
    const float *vel[3];
    memset(info, 0, sizeof(double) * 8);
    if (multinumt + 1 > MAXLEV || (frictyn && !se)) return -1;
    memset(H, 0, sizeof(*H));
    ht_grid_build(G, nx, ny, nz, gx, gy, gz, multinumt + 1);
    H->bct = bct; H->bondv1 = bondv1; H->bondn1 = bondn1;
    H->t0koef = dpar[3]; H->t1koef = dpar[4];
    H->kt = calloc(G->tot, sizeof(float)); H->cp = calloc(G->tot, sizeof(float)); H->ro = calloc(G->tot, sizeof(float));
    memcpy(H->kt, kt0, sizeof(float) * nn); memcpy(H->cp, cp0, sizeof(float) * nn); memcpy(H->ro, ro0, sizeof(float) * nn);
    H->sol0 = calloc(G->tot, sizeof(double)); H->sol1 = calloc(G->tot, sizeof(double));
    H->fre0 = calloc(G->tot, sizeof(double)); H->fre1 = calloc(G->tot, sizeof(double));
    H->val1 = calloc(G->tot * 7, sizeof(double)); H->lin0 = calloc(G->tot * 7, sizeof(long));
    H->pos0 = calloc(G->tot, sizeof(long)); H->num0 = calloc(G->tot, sizeof(int));
    tk0 = malloc(sizeof(float) * nn); tk1 = calloc(nn, sizeof(float)); tk2 = malloc(sizeof(float) * nn);
    gl[0] = gx; gl[1] = gy; gl[2] = gz;
    MG.g[0] = gx; MG.g[1] = gy; MG.g[2] = gz; MG.n[0] = nx; MG.n[1] = ny; MG.n[2] = nz;
    MG.size[0] = gx[nx - 1] - gx[0]; MG.size[1] = gy[ny - 1] - gy[0]; MG.size[2] = gz[nz - 1] - gz[0];
    vel[0] = vx; vel[1] = vy; vel[2] = vz;

    for (u = 0; u < nn; u++) { tk0[u] = tk[u]; if (tk[u] > maxtk) maxtk = tk[u]; if (tk[u] < mintk) mintk = tk[u]; }
    /* right-hand side per level-0 node and the step limit (heaterr mode 0) */
    for (m3 = 0; m3 < nz; m3++)
        for (m1 = 0; m1 < nx; m1++)
            for (m2 = 0; m2 < ny; m2++) {
                long v3 = m3 * nxy + m1 * ny + m2;
                double ival, rocpkf, xkf, ykf, zkf, x = 0, y = 0, z = 0, vxyz[3] = {0, 0, 0};
                long p[8];
                if (bct[v3]) continue;
                xkf = HT_KF(gx, m1); ykf = HT_KF(gy, m2); zkf = HT_KF(gz, m3);
                rocpkf = H->ro[v3] * H->cp[v3];
                if (rocpkf < 2e+6) rocpkf = 2e+6;
                ival = ht[v3];
                if (adiabyn == 2 || frictyn) {
                    p[0] = v3; p[1] = p[0] + 1; p[2] = p[0] + ny; p[3] = p[2] + 1;
                    p[4] = p[0] + nxy; p[5] = p[4] + 1; p[6] = p[4] + ny; p[7] = p[6] + 1;
                    x = (gx[m1] - gx[m1 - 1]) / 2.0 * xkf;
                    y = (gy[m2] - gy[m2 - 1]) / 2.0 * ykf;
                    z = (gz[m3] - gz[m3 - 1]) / 2.0 * zkf;
                }
                if (adiabyn) mv_velocity(&MG, vel, gx[m1], gy[m2], gz[m3], vxyz);
                if (adiabyn == 2 && H->ro[v3] > 2e+3) {
                    double dpdx = xkf * ((1.0 - y) * (1.0 - z) * (pr[p[2]] - pr[p[0]]) + y * (1.0 - z) * (pr[p[3]] - pr[p[1]]) +
                                         (1.0 - y) * z * (pr[p[6]] - pr[p[4]]) + y * z * (pr[p[7]] - pr[p[5]]));
                    double dpdy = ykf * ((1.0 - x) * (1.0 - z) * (pr[p[1]] - pr[p[0]]) + x * (1.0 - z) * (pr[p[3]] - pr[p[2]]) +
                                         (1.0 - x) * z * (pr[p[5]] - pr[p[4]]) + x * z * (pr[p[7]] - pr[p[6]]));
                    double dpdz = zkf * ((1.0 - x) * (1.0 - y) * (pr[p[4]] - pr[p[0]]) + x * (1.0 - y) * (pr[p[6]] - pr[p[2]]) +
                                         (1.0 - x) * y * (pr[p[5]] - pr[p[1]]) + x * y * (pr[p[7]] - pr[p[3]]));
                    ival += et[v3] * tk0[v3] * (vxyz[0] * dpdx + vxyz[1] * dpdy + vxyz[2] * dpdz);
                }
                if (adiabyn == 1 && H->ro[v3] > 2e+3)
                    ival += et[v3] * tk0[v3] * H->ro[v3] * (vxyz[0] * GXK + vxyz[1] * GYK + vxyz[2] * GZK);
                if (frictyn && H->ro[v3] > 2e+3) {
                    const float *sxx = se[0], *syy = se[1], *szz = se[2], *sxy = se[3], *sxz = se[4], *syz = se[5];
                    const float *exx = se[6], *eyy = se[7], *ezz = se[8], *exy = se[9], *exz = se[10], *eyz = se[11];
                    double ev;
#define HT_D(q) (sxx[p[q]] * exx[p[q]] + syy[p[q]] * eyy[p[q]] + szz[p[q]] * ezz[p[q]])
                    ev = (1.0 - x) * (1.0 - y) * (1.0 - z) * HT_D(0);
                    ev += (1.0 - x) * (y) * (1.0 - z) * HT_D(1);
                    ev += (x) * (1.0 - y) * (1.0 - z) * HT_D(2);
                    ev += (x) * (y) * (1.0 - z) * HT_D(3);
                    ev += (1.0 - x) * (1.0 - y) * (z) * HT_D(4);
                    ev += (1.0 - x) * (y) * (z) * HT_D(5);
                    ev += (x) * (1.0 - y) * (z) * HT_D(6);
                    ev += (x) * (y) * (z) * HT_D(7);
#undef HT_D
                    ev += 2.0 * ((1.0 - z) * (sxy[v3 - nxy] * exy[v3 - nxy]) + z * (sxy[v3] * exy[v3]));
                    ev += 2.0 * ((1.0 - y) * (sxz[v3 - 1] * exz[v3 - 1]) + y * (sxz[v3] * exz[v3]));
                    ev += 2.0 * ((1.0 - x) * (syz[v3 - ny] * eyz[v3 - ny]) + x * (syz[v3] * eyz[v3]));
                    ival += ev;
                }
                tk1[v3] = (float)ival;
                ival = fabs(ival / rocpkf);
                if (ival > maxtkrate) maxtkrate = ival;
            }
    if (maxtkrate) tktimestep = maxtkstep / maxtkrate;
    info[0] = tktimestep;
    info[7] = maxtkrate;
    if (timestep == 0 || tktimestep == 0) goto done;
    for (u = 0; u < nn; u++) tk2[u] = tk[u];
    for (li = 1; li <= multinumt; li++) ht_rocprestrict(H, li);
    tktimesum = 0;
    tktimesum0 = timestep;
    do {
        timestep = tktimesum0 < tktimestep ? tktimesum0 : tktimestep;
        if (timestep > (tktimesum0 - tktimesum)) timestep = tktimesum0 - tktimesum;
        for (u = 0; u < nn; u++) tk0[u] = tk[u];
        for (u = 0; u < nn; u++) H->sol0[u] = tk[u];
        nsub++;
        /* rows of every level (heaterr mode 1, tbonderr) */
        for (li = 0; li <= multinumt; li++) {
            const double *g0 = G->g[li][0], *g1 = G->g[li][1], *g2 = G->g[li][2];
            long lnx = G->nx[li], lny = G->ny[li], lnxy = lnx * lny;
            for (m3 = 0; m3 < G->nz[li]; m3++)
                for (m1 = 0; m1 < lnx; m1++)
                    for (m2 = 0; m2 < lny; m2++) {
                        long v[7], un[7];
                        double ui[7], rhs, rocpkf, ival, xkf, ykf, zkf;
                        v[3] = G->off[li] + m3 * lnxy + m1 * lny + m2;
                        if (bct[v[3]]) {
                            int b = bct[v[3]], k = 1;
                            un[0] = v[3]; ui[0] = 1.0;
                            if (bondn1[b]) { un[1] = bondn1[b] - 1; ui[1] = -bondv1[2 * b + 1]; k = 2; }
                            ht_row(H, v[3], k, un, ui, bondv1[2 * b]);
                            continue;
                        }
                        v[0] = v[3] - lnxy; v[1] = v[3] - lny; v[2] = v[3] - 1; v[4] = v[3] + 1; v[5] = v[3] + lny;
                        v[6] = v[3] + lnxy;
                        xkf = HT_KF(g0, m1); ykf = HT_KF(g1, m2); zkf = HT_KF(g2, m3);
                        rocpkf = H->ro[v[3]] * H->cp[v[3]];
                        if (rocpkf < 2e+6) rocpkf = 2e+6;
                        rhs = li == 0 ? tk1[v[3]] + tk0[v[3]] / timestep * rocpkf : 0;
                        ui[0] = rocpkf / timestep; un[0] = v[3];
                        ival = (H->kt[v[1]] + H->kt[v[3]]) / 2.0 * xkf / (g0[m1] - g0[m1 - 1]);
                        ui[1] = -ival; un[1] = v[1]; ui[0] += ival;
                        ival = (H->kt[v[3]] + H->kt[v[5]]) / 2.0 * xkf / (g0[m1 + 1] - g0[m1]);
                        ui[0] += ival; ui[2] = -ival; un[2] = v[5];
                        ival = (H->kt[v[2]] + H->kt[v[3]]) / 2.0 * ykf / (g1[m2] - g1[m2 - 1]);
                        ui[3] = -ival; un[3] = v[2]; ui[0] += ival;
                        ival = (H->kt[v[3]] + H->kt[v[4]]) / 2.0 * ykf / (g1[m2 + 1] - g1[m2]);
                        ui[0] += ival; ui[4] = -ival; un[4] = v[4];
                        ival = (H->kt[v[0]] + H->kt[v[3]]) / 2.0 * zkf / (g2[m3] - g2[m3 - 1]);
                        ui[5] = -ival; un[5] = v[0]; ui[0] += ival;
                        ival = (H->kt[v[3]] + H->kt[v[6]]) / 2.0 * zkf / (g2[m3 + 1] - g2[m3]);
                        ui[0] += ival; ui[6] = -ival; un[6] = v[6];
                        ht_row(H, v[3], 7, un, ui, rhs);
                    }
        }
        do {
            int n1, n2;
            double bsum = 0, hnum = 0;
            for (n1 = 0; n1 < multicyct; n1++) {
                if (multinumt > 0) {
                    for (n2 = 0; n2 < multinumt; n2++) {
                        ht_gausmatt(H, ipar[4 + n2], G->off[n2] + G->n[n2] - 1, G->off[n2]);
                        ht_restrict(H, n2 + 1);
                    }
                    for (n2 = multinumt; n2 > 0; n2--) {
                        ht_gausmatt(H, ipar[20 + n2], G->off[n2] + G->n[n2] - 1, G->off[n2]);
                        ht_prolong(H, n2);
                    }
                } else
                    ht_gausmatt(H, ipar[4], G->off[0] + G->n[0] - 1, G->off[0]);
            }
            ncyc++;
            mintk = 1e30; maxtk = -1e30;
            for (u = 0; u < nn; u++) {
                tk[u] = (float)H->sol0[u];
                if (tk[u] < mintk) mintk = tk[u];
                if (tk[u] > maxtk) maxtk = tk[u];
            }
            /* error of the heat rows (heaterr mode 2) */
            heatsum = 0;
            for (m3 = 0; m3 < nz; m3++)
                for (m1 = 0; m1 < nx; m1++)
                    for (m2 = 0; m2 < ny; m2++) {
                        long v[7];
                        double rocpkf, ival, ival1, xkf, ykf, zkf;
                        v[3] = m3 * nxy + m1 * ny + m2;
                        if (bct[v[3]]) continue;
                        v[0] = v[3] - nxy; v[1] = v[3] - ny; v[2] = v[3] - 1; v[4] = v[3] + 1; v[5] = v[3] + ny;
                        v[6] = v[3] + nxy;
                        xkf = HT_KF(gx, m1); ykf = HT_KF(gy, m2); zkf = HT_KF(gz, m3);
                        rocpkf = H->ro[v[3]] * H->cp[v[3]];
                        if (rocpkf < 2e+6) rocpkf = 2e+6;
                        ival1 = (tk[v[3]] - tk0[v[3]]) / timestep;
                        ival = (H->kt[v[1]] + H->kt[v[3]]) / 2.0 * xkf / (gx[m1] - gx[m1 - 1]) / rocpkf;
                        ival1 += (tk[v[3]] - tk[v[1]]) * ival;
                        ival = (H->kt[v[3]] + H->kt[v[5]]) / 2.0 * xkf / (gx[m1 + 1] - gx[m1]) / rocpkf;
                        ival1 -= (tk[v[5]] - tk[v[3]]) * ival;
                        ival = (H->kt[v[2]] + H->kt[v[3]]) / 2.0 * ykf / (gy[m2] - gy[m2 - 1]) / rocpkf;
                        ival1 += (tk[v[3]] - tk[v[2]]) * ival;
                        ival = (H->kt[v[3]] + H->kt[v[4]]) / 2.0 * ykf / (gy[m2 + 1] - gy[m2]) / rocpkf;
                        ival1 -= (tk[v[4]] - tk[v[3]]) * ival;
                        ival = (H->kt[v[0]] + H->kt[v[3]]) / 2.0 * zkf / (gz[m3] - gz[m3 - 1]) / rocpkf;
                        ival1 += (tk[v[3]] - tk[v[0]]) * ival;
                        ival = (H->kt[v[3]] + H->kt[v[6]]) / 2.0 * zkf / (gz[m3 + 1] - gz[m3]) / rocpkf;
                        ival1 -= (tk[v[6]] - tk[v[3]]) * ival;
                        ival1 -= tk1[v[3]] / rocpkf;
                        ival1 *= timestep;
                        heatsum += ival1 * ival1;
                        hnum += 1.0;
                    }
            heatsum = pow(heatsum / hnum, 0.5);
            (void)bsum;
            if (heatsum > heatmin && maxcyc > 0 && ncyc >= maxcyc) { status = 1; break; }
        } while (heatsum > heatmin);
        tktimesum += timestep;
        if (status) break;
    } while (tktimesum < tktimesum0);
    timestep = tktimesum0;
    (void)gl;

    /* marker temperatures (heat3mg.c:641-829) */
    if (nmark > 0 && markk) {
        double *S0 = calloc(nn, sizeof(double)), *S1 = calloc(nn, sizeof(double));
        double xs = gx[nx - 1] - gx[0], ys = gy[ny - 1] - gy[0], zs = gz[nz - 1] - gz[0];
        for (mk = 0; mk < nmark; mk++) {
            long wn[11];
            double wi[11], e2, e3;
            int inside = markx[mk] > 0 && marky[mk] > 0 && markz[mk] > 0 && (double)markx[mk] < xs &&
                         (double)marky[mk] < ys && (double)markz[mk] < zs;
            int t = markt[mk];
            if (!inside || t >= 100) continue;
            /* tkcalc1 (mark3mg.c:1212-1282) */
            {
                double x = markx[mk], y = marky[mk], z = markz[mk], dx, dy, dz;
                long a1 = serch(gx, nx, x), a2 = serch(gy, ny, y), a3 = serch(gz, nz, z), c3, c1, c2;
                int n1 = 0;
                wn[0] = a1; wn[1] = a2; wn[2] = a3;
                wi[0] = dx = gx[a1 + 1] - gx[a1]; wi[1] = dy = gy[a2 + 1] - gy[a2]; wi[2] = dz = gz[a3 + 1] - gz[a3];
                e2 = e3 = 0;
                for (c3 = a3; c3 <= a3 + 1; c3++) {
                    double ddz = 1.0 - fabs((gz[c3] - z) / dz);
                    for (c1 = a1; c1 <= a1 + 1; c1++) {
                        double ddx = 1.0 - fabs((gx[c1] - x) / dx);
                        for (c2 = a2; c2 <= a2 + 1; c2++) {
                            double ddy = 1.0 - fabs((gy[c2] - y) / dy), swt = ddx * ddy * ddz;
                            long m4 = c3 * nxy + c1 * ny + c2;
                            wi[3 + n1] = swt; wn[3 + n1] = m4;
                            e2 += swt * tk[m4];
                            e3 += swt * tk2[m4];
                            n1++;
                        }
                    }
                }
            }
            if (t >= 50) { markk[mk] = (float)e2; continue; }
            if (markk[mk] <= 0) {
                markk[mk] = (float)e3;
                if (marky[mk] > zdeep && markk[mk] < tdeep) markk[mk] = tdeep;
            }
            if (heatdif) {
                double mkt = 0, mcp = 0, mro = 0, mtk = tk[wn[3]], dtk, dtk1, rocpkf;
                int n1;
                for (n1 = 0; n1 < 8; n1++) {
                    long m4 = wn[3 + n1];
                    double w = wi[3 + n1];
                    mkt += H->kt[m4] * w; mcp += H->cp[m4] * w; mro += H->ro[m4] * w;
                    if (tk[m4] > mtk) mtk = tk[m4];
                }
                if ((wn[0] <= 0 || wn[0] >= nx - 2 || wn[1] <= 0 || wn[1] >= ny - 2 || wn[2] <= 0 || wn[2] >= nz - 2) &&
                    (markk[mk] + e2 - e3) > mtk)
                    markk[mk] = mtk - e2 + e3;
                dtk = e3 - (double)markk[mk];
                rocpkf = mro * mcp;
                if (rocpkf < 2e+6) rocpkf = 2e+6;
                dtk1 = -heatdif * mkt / rocpkf * 2.0 * (1.0 / wi[0] / wi[0] + 1.0 / wi[1] / wi[1] + 1.0 / wi[2] / wi[2]) * timestep;
                if (dtk1 < -150.0) dtk1 = -150.0;
                dtk1 = dtk * (1.0 - exp(dtk1));
                markk[mk] += (float)dtk1;
                for (n1 = 0; n1 < 8; n1++) { S1[wn[3 + n1]] += dtk1 * wi[3 + n1]; S0[wn[3 + n1]] += wi[3 + n1]; }
            }
            markk[mk] += (float)(e2 - e3);
        }
        if (heatdif) {
            for (u = 0; u < nn; u++)
                if (S0[u]) S1[u] /= S0[u];
            for (mk = 0; mk < nmark; mk++) {
                int inside = markx[mk] > 0 && marky[mk] > 0 && markz[mk] > 0 && (double)markx[mk] < xs &&
                             (double)marky[mk] < ys && (double)markz[mk] < zs;
                long a1, a2, a3, c1, c2, c3;
                double x, y, z, dx, dy, dz;
                if (!inside || markt[mk] >= 50) continue;
                x = markx[mk]; y = marky[mk]; z = markz[mk];
                a1 = serch(gx, nx, x); a2 = serch(gy, ny, y); a3 = serch(gz, nz, z);
                dx = gx[a1 + 1] - gx[a1]; dy = gy[a2 + 1] - gy[a2]; dz = gz[a3 + 1] - gz[a3];
                for (c3 = a3; c3 <= a3 + 1; c3++) {
                    double ddz = 1.0 - fabs((gz[c3] - z) / dz);
                    for (c1 = a1; c1 <= a1 + 1; c1++) {
                        double ddx = 1.0 - fabs((gx[c1] - x) / dx);
                        for (c2 = a2; c2 <= a2 + 1; c2++) {
                            double ddy = 1.0 - fabs((gy[c2] - y) / dy);
                            long m4 = c3 * nxy + c1 * ny + c2;
                            if (S1[m4]) markk[mk] -= (float)(S1[m4] * (ddx * ddy * ddz));
                        }
                    }
                }
            }
        }
        free(S0); free(S1);
    }
done:
    info[1] = (double)nsub; info[2] = (double)ncyc; info[3] = heatsum; info[4] = mintk; info[5] = maxtk;
    info[6] = status;
    free(H->kt); free(H->cp); free(H->ro); free(H->sol0); free(H->sol1); free(H->fre0); free(H->fre1);
    free(H->val1); free(H->lin0); free(H->pos0); free(H->num0); free(tk0); free(tk1); free(tk2);
    ht_grid_free(G);
    return status;
}
