/*
 * move3mg_cuda.c -- the reference's vpiterate(), ronurecalc(), movemark(),
 * effbulkvisccalc() and titerate() on top of libp2cuda.so (include/p2cuda.h).
 *
 * This file is compiled inside the reference's unity build (pardiso/i3mg.c
 * includes head3mg.c, load3mg.c, move3mgNew.c, mark3mg.c, ... into one
 * translation unit) and uses its globals (pardiso/head3mg.c) directly: the
 * entry points keep their signatures and their data exchange through
 * globals, so the time loop in i3mg.c is unchanged.  The CPU functions it
 * replaces are renamed out of the way before their files are included:
 *
 *     #define vpiterate  vpiterate_cpu     -- pardiso/move3mgNew.c:1791
 *     #define ronurecalc ronurecalc_cpu    -- pardiso/mark3mg.c:630
 *     #define movemark   movemark_cpu      -- pardiso/mark3mg.c:174
 *     #define effbulkvisccalc effbulkvisccalc_cpu  -- pardiso/mark3mg.c:2
 *     #include "move3mgNew.c"
 *     #include "mark3mg.c"
 *     #undef vpiterate
 *     #undef ronurecalc
 *     #undef movemark
 *     #undef effbulkvisccalc
 *     #include "gaus3mg_SerieMG.c"
 *     #define titerate titerate_cpu        -- pardiso/heat3mg.c:292
 *     #include "heat3mg.c"
 *     #undef titerate
 *     #include "move3mg_cuda.c"
 *
 * Inputs read: xnumx, ynumy, znumz, gx, gy, gz, x/y/zperiodic, multinum,
 * multinnn, mgp, mgn, bondm, bondv1, bondn1, bondnum, nu, ro, nxx, nxy, nxz,
 * nyz, vx, vy, vz, pr, p0koef, p1koef, p2koef, v0koef, v1koef, nubeg, nuend,
 * nukoef, viscmod, GXKOEF, GYKOEF, GZKOEF, pinit, pxinit, pyinit, pzinit;
 * markers markx, marky, markz, markt, marknum and the rock tables markn0,
 * markn1, markro (rocknum types); maxxystep and timestep for the time-step
 * limit; timestep, markmod, outgrid for movemark.
 * With power-law rocks (types <= 20 with markn0 != markn1) ronurecalc also
 * reads marknu, markmm and val1.
 * Outputs written: vx, vy, vz (float), pr (double), the stresses sxx..syz and
 * strain rates exx..eyz (float) and the limited timestep by vpiterate; nu,
 * ro, nxx, nxy, nxz, nyz and marke (0 -> 1e-20) by ronurecalc; markx, marky,
 * markz and the markk
 * reset of markers that leave the box, val1 (strain-rate invariant per
 * marker) and marke (brittle strain) by movemark.
 * titerate reads tk, kt, cp, ro, ht, et, the T rows of bondm (from
 * 8 * nodenum), HEATMIN, multinumt, multicyct, multittt, t0koef, t1koef,
 * heatdif, frictyn, adiabyn, tdeep, zdeep, maxtkstep, timestep, GX/GY/GZKOEF,
 * vx, vy, vz, pr, sxx..syz, exx..eyz and the markers, and writes tk and markk.
 *
 * Errors follow the reference's convention: a message on stdout and exit().
 * The device is 0, or the value of the environment variable P2CUDA_DEVICE.
 */

#include "p2cuda.h"

static p2_ctx *p2s_ctx = NULL;
static long p2s_grid_nodes = -1;

static void p2s_fail(const char *what, p2_status st)
{
    printf("%s failed (p2cuda status %d): %s\n", what, (int)st, p2s_ctx ? p2_last_error(p2s_ctx) : "no context");
    exit(0);
}

static void p2s_params(p2_params *p)
{
    int l;
    p2_default_params(p);
    p->p0koef = p0koef;
    p->p1koef = p1koef;
    p->p2koef = p2koef;
    p->v0koef = v0koef;
    p->v1koef = v1koef;
    p->nubeg = nubeg;
    p->nuend = nuend;
    p->nukoef = nukoef;
    p->gxkoef = GXKOEF;
    p->gykoef = GYKOEF;
    p->gzkoef = GZKOEF;
    p->pinit = pinit;
    p->pxinit = (int)pxinit;
    p->pyinit = (int)pyinit;
    p->pzinit = (int)pzinit;
    p->viscmod = viscmod;
    p->multinum = multinum;
    /* sweeps per level: multinnn[0][] before, multinnn[1][] after the coarse
       correction (mode.t3c); the level-0 counts set the base of the schedule */
    for (l = 0; l <= multinum && l < P2_MAX_LEVELS; l++) {
        p->npre[l] = multinnn[0][l] > 0 ? multinnn[0][l] : 1;
        p->npost[l] = multinnn[1][l] > 0 ? multinnn[1][l] : 1;
    }
}

/* Context, grid and boundary tables: once, and again if the grid changes. */
static void p2s_setup(void)
{
    p2_status st;
    p2_params prm;
    long nodes = xnumx * ynumy * znumz;
    if (!p2s_ctx) {
        const char *d = getenv("P2CUDA_DEVICE");
        st = p2_create(&p2s_ctx, d ? atoi(d) : 0);
        if (st != P2_OK) p2s_fail("p2_create", st);
    }
    if (p2s_grid_nodes == nodes) return;
    p2s_params(&prm);
    st = p2_set_grid(p2s_ctx, xnumx, ynumy, znumz, gx, gy, gz, xperiodic, yperiodic, zperiodic, &prm);
    if (st != P2_OK) p2s_fail("p2_set_grid", st);
    st = p2_set_bc(p2s_ctx, bondm, 4L * (mgp[multinum] + mgn[multinum]), &bondv1[0][0], bondn1, bondnum);
    if (st != P2_OK) p2s_fail("p2_set_bc", st);
    p2s_grid_nodes = nodes;
}

/* pardiso/move3mgNew.c:1791 (prototype pardiso/head3mg.c:362): the Stokes
 * solve on the current node fields; vx, vy, vz, pr are the initial guess on
 * entry and the solution on return.  m0 and f0 are the caller's loop
 * counters, unused here as in the reference apart from its printing. */
void vpiterate(int m0, int f0)
{
    p2_status st;
    p2_solve_info info;
    double vr[6];
    int c;
    (void)m0;
    (void)f0;
    p2s_setup();
    st = p2_set_nodes(p2s_ctx, nu, ro, nxx, nxy, nxz, nyz);
    if (st != P2_OK) p2s_fail("p2_set_nodes", st);
    st = p2_stokes_solve(p2s_ctx, vx, vy, vz, pr, &info);
    if (st != P2_OK) p2s_fail("p2_stokes_solve", st);
    /* stresses, strain rates and velocity ranges (move3mgNew.c:2908-3038) */
    st = p2_stress_strain(p2s_ctx, sxx, syy, szz, sxy, sxz, syz, exx, eyy, ezz, exy, exz, eyz, vr);
    if (st != P2_OK) p2s_fail("p2_stress_strain", st);
    /* marker time step: no marker moves more than maxxystep along an axis
       (move3mgNew.c:3293-3316) */
    for (c = 0; c < 3; c++) {
        double vmax = fabs(vr[2 * c]) > fabs(vr[2 * c + 1]) ? fabs(vr[2 * c]) : fabs(vr[2 * c + 1]);
        if (vmax) {
            vmax = maxxystep / vmax;
            if (timestep > vmax) timestep = vmax;
        }
    }
    printf("vpiterate (p2cuda): %d iterations, relative residual %e, %.2f ms\n", info.iterations, info.rel_residual,
           info.ms_total);
}

/* pardiso/mark3mg.c:630 (prototype pardiso/head3mg.c:417): marker -> node
 * viscosity and density; markers of type >= 50 are skipped as in the
 * reference; rock types <= 20 with markn0 != markn1 take the power-law
 * viscosity from val1 (viscalc, mark3mg.c:1463-1498). */
void ronurecalc(void)
{
    p2_status st;
    int nrock = rocknum > 0 && rocknum <= MAXTMR ? rocknum : MAXTMR;
    int t, power_law = 0;
    long m;
    p2s_setup();
    for (t = 0; t < nrock && t <= 20; t++)
        if (markn0[t] != markn1[t]) power_law = 1;
    if (power_law) {
        /* viscosity from each marker's strain-rate invariant val1 (viscalc) */
        st = p2_ronurecalc_powerlaw(p2s_ctx, marknum, markx, marky, markz, (const signed char *)markt, nrock, markn0,
                                    markn1, markro, marknu, markmm, val1, nu, ro, nxx, nxy, nxz, nyz);
        if (st != P2_OK) p2s_fail("p2_ronurecalc_powerlaw", st);
    } else {
        st = p2_ronurecalc(p2s_ctx, marknum, markx, marky, markz, (const signed char *)markt, nrock, markn0, markn1,
                           markro, nu, ro, nxx, nxy, nxz, nyz);
        if (st != P2_OK) p2s_fail("p2_ronurecalc", st);
    }
    /* viscalc's side effect (mark3mg.c:1477) on the markers ronurecalc visits
       (mark3mg.c:694): a zero brittle strain becomes 1e-20 */
    for (m = 0; m < marknum; m++)
        if (markx[m] > 0 && marky[m] > 0 && markz[m] > 0 && markx[m] < xsize && marky[m] < ysize &&
            markz[m] < zsize && markt[m] < 50 && marke[m] == 0.0)
            marke[m] = 1e-20;
}

/* pardiso/mark3mg.c:174 (prototype pardiso/head3mg.c:416): advect the markers
 * through the current vx, vy, vz over timestep (markmod 1 or 2); periodic
 * boxes are not supported.  Markers of type < 100 that end outside the box
 * get markk = 0, as in the reference (mark3mg.c:489-494), when markk has
 * storage (i3mg.c's dynmemall() leaves it null, and the CPU movemark would
 * then fault on that store). */
void movemark(void)
{
    p2_status st;
    long m;
    char *was_in = NULL;
    if (markmod != 1 && markmod != 2) return;
    p2s_setup();
    if (marknum > 0) {
        was_in = (char *)malloc((size_t)marknum);
        if (!was_in) {
            printf("movemark: out of host memory\n");
            exit(0);
        }
        for (m = 0; m < marknum; m++)
            was_in[m] = markx[m] >= 0 && marky[m] >= 0 && markz[m] >= 0 && (double)markx[m] <= xsize &&
                        (double)marky[m] <= ysize && (double)markz[m] <= zsize;
    }
    /* exx..eyz as vpiterate left them; val1 and marke per marker */
    st = p2_movemark_strain(p2s_ctx, timestep, markmod, outgrid, vx, vy, vz, exx, eyy, ezz, exy, exz, eyz, marknum,
                            markx, marky, markz, (const signed char *)markt, val1, marke);
    if (st != P2_OK) p2s_fail("p2_movemark_strain", st);
    for (m = 0; m < marknum; m++) {
        int t = markt[m];
        int moved = was_in[m] || (outgrid != 1 && (t < 50 || t >= 100));
        if (markk && moved && t < 100 &&
            (markx[m] < 0 || marky[m] < 0 || markz[m] < 0 || (double)markx[m] > xsize ||
             (double)marky[m] > ysize || (double)markz[m] > zsize))
            markk[m] = 0;
    }
    free(was_in);
}

/* pardiso/mark3mg.c:2 (prototype pardiso/head3mg.c:435): effective bulk
 * viscosity diagnostics.  Mode 1 (node fields) runs on the GPU
 * (p2_effbulk_visc) and prints and appends to effbulkvisc.txt what the
 * reference does; mode 2 (the brittle-strain budget of marker types 7-10)
 * stays the reference's own effbulkvisccalc_cpu. */
void effbulkvisccalc(int nodemark)
{
    p2_status st;
    p2_effbulk r;
    FILE *f;
    if (nodemark != 1) {
        effbulkvisccalc_cpu(nodemark);
        return;
    }
    p2s_setup();
    st = p2_effbulk_visc(p2s_ctx, ro, nxx, nxy, nxz, nyz, exx, eyy, ezz, exy, exz, eyz, sxx, syy, szz, sxy, sxz,
                         syz, &r);
    if (st != P2_OK) p2s_fail("p2_effbulk_visc", st);
    printf("\n Siin = %e Eiin = %e Eiivp = %e Tau2n = %e Hsn = %e Nubulkn = %e Tot Num = %ld\n", r.siin, r.eiin,
           r.eiivp, r.tau2, r.hsn, r.nubulkn, r.numtot);
    printf("\n Nubulk1 = Tau2n/Eiin %e \n", r.nubulk1);
    printf("\n Nubulk2 = Hs/4/Eiin^2 %e \n", r.nubulk2);
    printf("\n Nubulk3 = Hs/4/Eiivp^2 %e \n", r.nubulk3);
    printf("\n Nubulk4 = Siin/2/Eiin %e \n", r.nubulk4);
    f = fopen("effbulkvisc.txt", "at");
    if (!f) return;
    fprintf(f, "%e %e %ld %ld %ld %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e %e "
               "%e %e %e\n",
            timesum, timestep, r.numinc, r.nummat, r.numtot, r.matrix[0], r.matrix[1], r.matrix[2], r.matrix[3],
            r.matrix[4], r.matrix[5], r.matrix[6], r.matrix[7], r.matrix[8], r.matrix[9], r.matrix[10], r.matrix[11],
            r.incl[0], r.incl[1], r.incl[2], r.incl[3], r.incl[4], r.incl[5], r.incl[6], r.incl[7], r.incl[8],
            r.incl[9], r.incl[10], r.incl[11], r.siin, r.eiin, r.eiivp, r.hsn, r.nubulk2, r.nubulk3, r.nubulk4);
    fclose(f);
}

/* pardiso/heat3mg.c:292 (prototype pardiso/head3mg.c:386): one thermal step
 * of timestep seconds on tk and on the marker temperatures markk (markers are
 * skipped when markk has no storage).  The coarse-level kt, cp, ro and the
 * work arrays tk0, tk1, tk2 stay on the device.  The reference repeats its
 * V-cycles until the error is below HEATMIN; the library stops after 10000
 * error checks per sub-step and the shim reports it. */
static long p2s_heat_nodes = -1;

void titerate(int m0)
{
    p2_status st;
    p2_heat_params hp;
    p2_heat_info info;
    const float *se[12];
    int l;
    p2s_setup();
    if (p2s_heat_nodes != p2s_grid_nodes) {
        st = p2_heat_set_bc(p2s_ctx, bondm, nodenum8 + mgp[multinum] + mgn[multinum], &bondv1[0][0], bondn1,
                            bondnum);
        if (st != P2_OK) p2s_fail("p2_heat_set_bc", st);
        p2s_heat_nodes = p2s_grid_nodes;
    }
    p2_default_heat_params(&hp);
    hp.maxtkstep = maxtkstep;
    hp.heatmin = HEATMIN;
    hp.t0koef = t0koef;
    hp.t1koef = t1koef;
    hp.heatdif = heatdif;
    hp.tdeep = tdeep;
    hp.zdeep = zdeep;
    hp.multinumt = multinumt;
    hp.multicyct = multicyct;
    for (l = 0; l < P2_MAX_LEVELS; l++) {
        hp.multittt[0][l] = l <= multinumt ? multittt[0][l] : 0;
        hp.multittt[1][l] = l <= multinumt ? multittt[1][l] : 0;
    }
    hp.frictyn = frictyn;
    hp.adiabyn = adiabyn;
    hp.max_cycles = 0;
    se[0] = sxx; se[1] = syy; se[2] = szz; se[3] = sxy; se[4] = sxz; se[5] = syz;
    se[6] = exx; se[7] = eyy; se[8] = ezz; se[9] = exy; se[10] = exz; se[11] = eyz;
    st = p2_titerate(p2s_ctx, &hp, timestep, tk, kt, cp, ro, ht, et, vx, vy, vz, pr, se, markk ? marknum : 0, markx,
                     marky, markz, (const signed char *)markt, markk, &info);
    if (st != P2_OK) p2s_fail("p2_titerate", st);
    if (!info.converged)
        printf("\n T ITERATIONS STOPPED: %d checks, err = %e > HEATMIN = %e\n", info.cycles, info.heatsum, HEATMIN);
    if (printmod) {
        printf("\n KRUG %2d \n", m0 + 1);
        printf("THERMAL STEP = %e YEARS    SUBSTEPS = %d\n", timestep / 3.15576e+7, info.substeps);
        printf("TEMPERATURE    : min = %e max = %e \n", info.mintk, info.maxtk);
        printf("TERMAL EQUATION: err = %e \n", info.heatsum);
    }
}
