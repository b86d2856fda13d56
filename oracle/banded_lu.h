/*
 * Banded LU with partial pivoting, FP64 (test infrastructure: CPU oracle).
 *
 * Stands in for Intel MKL PARDISO, the third-party direct solver the
 * reference calls for the coarsest multigrid level
 * (pardiso/gaus3mg_SerieMG.c:64-309; phases 11/22/33/-1 at 170/185/198/216,
 * mtype=11 real unsymmetric, iparm[7]=2 refinement steps).  MKL is not
 * vendored and has no pinned version in the reference (compile.sh:5 links
 * -lmkl_intel_lp64 -lmkl_intel_thread -lmkl_core).  Its published algorithm
 * is a sparse direct LU factorisation with pivoting followed by iterative
 * refinement; for a nonsingular system any accurate pivoted LU returns the
 * same solution to rounding, so this file restates the textbook band
 * Gaussian elimination with row partial pivoting (the LAPACK *gbtf2 scheme:
 * column-major band storage with kl extra rows for pivoting fill-in),
 * plus residual-based iterative refinement on the original CSR rows.
 *
 * Header-only (static functions) so that both the reference harness and
 * the oracle restatement can include it.
 */
#ifndef P2_BANDED_LU_H
#define P2_BANDED_LU_H

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    long n, kl, ku, kv, ldab;
    double *ab;   /* (ldab x n) column-major band: A(i,j) at ab[j*ldab + kv + i - j] */
    long *ipiv;   /* row interchanged with row j at step j */
    int singular; /* first zero pivot column + 1, or 0 */
} p2_band_lu;

static void p2_band_free(p2_band_lu *f)
{
    if (!f) return;
    free(f->ab);
    free(f->ipiv);
    memset(f, 0, sizeof(*f));
}

/* Allocate a zeroed band of size n with lower/upper bandwidths kl, ku. */
static int p2_band_alloc(p2_band_lu *f, long n, long kl, long ku)
{
    memset(f, 0, sizeof(*f));
    f->n = n;
    f->kl = kl;
    f->ku = ku;
    f->kv = kl + ku;
    f->ldab = 2 * kl + ku + 1;
    f->ab = (double *)calloc((size_t)(f->ldab * n), sizeof(double));
    f->ipiv = (long *)calloc((size_t)n, sizeof(long));
    return (f->ab && f->ipiv) ? 0 : -1;
}

static double *p2_band_at(p2_band_lu *f, long i, long j)
{
    return &f->ab[j * f->ldab + f->kv + i - j];
}

/* Factor in place: P A = L U.  Returns 0, or (column+1) of the first zero pivot. */
static int p2_band_factor(p2_band_lu *f)
{
    long n = f->n, kl = f->kl, kv = f->kv, ldab = f->ldab;
    long j, i, c, ju = 0;
    double *ab = f->ab;
    f->singular = 0;
    for (j = 0; j < n; j++) {
        long km = kl < n - 1 - j ? kl : n - 1 - j;
        long p = j;
        double best = fabs(ab[j * ldab + kv]);
        for (i = 1; i <= km; i++) {
            double v = fabs(ab[j * ldab + kv + i]);
            if (v > best) { best = v; p = j + i; }
        }
        f->ipiv[j] = p;
        if (best == 0.0) {
            if (!f->singular) f->singular = (int)(j + 1);
            continue;
        }
        {
            long jlast = j + f->ku + (p - j);
            if (jlast > n - 1) jlast = n - 1;
            if (jlast > ju) ju = jlast;
        }
        if (p != j) {
            for (c = j; c <= ju; c++) {
                double *a = &ab[c * ldab + kv + j - c];
                double *b = &ab[c * ldab + kv + p - c];
                double t = *a; *a = *b; *b = t;
            }
        }
        {
            double inv = 1.0 / ab[j * ldab + kv];
            double *col = &ab[j * ldab + kv + 1];
            for (i = 0; i < km; i++) col[i] *= inv;
            for (c = j + 1; c <= ju; c++) {
                double *cc = &ab[c * ldab + kv + j - c];
                double t = cc[0];
                if (t != 0.0) {
                    for (i = 1; i <= km; i++) cc[i] -= col[i - 1] * t;
                }
            }
        }
    }
    return f->singular;
}

/* Solve A x = b in place (x holds b on entry). */
static void p2_band_solve(const p2_band_lu *f, double *x)
{
    long n = f->n, kl = f->kl, kv = f->kv, ldab = f->ldab;
    long j, i;
    const double *ab = f->ab;
    for (j = 0; j < n; j++) {
        long km = kl < n - 1 - j ? kl : n - 1 - j;
        long p = f->ipiv[j];
        double t;
        if (p != j) { t = x[p]; x[p] = x[j]; x[j] = t; }
        t = x[j];
        if (t != 0.0) {
            const double *col = &ab[j * ldab + kv + 1];
            for (i = 0; i < km; i++) x[j + 1 + i] -= col[i] * t;
        }
    }
    for (j = n - 1; j >= 0; j--) {
        long i0 = j - kv < 0 ? 0 : j - kv;
        const double *col = &ab[j * ldab + kv - (j - i0)];
        double d = ab[j * ldab + kv];
        if (d != 0.0) x[j] /= d;
        {
            double t = x[j];
            if (t != 0.0)
                for (i = i0; i < j; i++) x[i] -= col[i - i0] * t;
        }
    }
}

/*
 * Build the band from a 1-based CSR (the PARDISO input convention,
 * pardiso/move3mgNew.c:2665-2698), factor, and keep the CSR for refinement.
 */
typedef struct {
    p2_band_lu lu;
    long n;
    const int *ia, *ja;
    const double *a;
} p2_csr_lu;

static int p2_csr_lu_factor(p2_csr_lu *s, long n, const int *ia, const int *ja, const double *a)
{
    long i, k, kl = 0, ku = 0;
    s->n = n; s->ia = ia; s->ja = ja; s->a = a;
    for (i = 0; i < n; i++)
        for (k = ia[i] - 1; k < ia[i + 1] - 1; k++) {
            long j = ja[k] - 1;
            if (i - j > kl) kl = i - j;
            if (j - i > ku) ku = j - i;
        }
    if (p2_band_alloc(&s->lu, n, kl, ku)) return -1;
    for (i = 0; i < n; i++)
        for (k = ia[i] - 1; k < ia[i + 1] - 1; k++) {
            long j = ja[k] - 1;
            *p2_band_at(&s->lu, i, j) += a[k];
        }
    return p2_band_factor(&s->lu);
}

/* Solve with `nref` residual-based refinement steps on the CSR rows. */
static void p2_csr_lu_solve(p2_csr_lu *s, const double *b, double *x, int nref)
{
    long n = s->n, i, k;
    int it;
    double *r = (double *)malloc(sizeof(double) * (size_t)n);
    memcpy(x, b, sizeof(double) * (size_t)n);
    p2_band_solve(&s->lu, x);
    for (it = 0; it < nref; it++) {
        for (i = 0; i < n; i++) {
            double acc = b[i];
            for (k = s->ia[i] - 1; k < s->ia[i + 1] - 1; k++) acc -= s->a[k] * x[s->ja[k] - 1];
            r[i] = acc;
        }
        p2_band_solve(&s->lu, r);
        for (i = 0; i < n; i++) x[i] += r[i];
    }
    free(r);
}

#endif
