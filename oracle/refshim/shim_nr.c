/*
 * shim_nr.c -- TEST INFRASTRUCTURE ONLY.  The Numerical Recipes in C routines
 * (GrIMP's cRecipes, not part of the reference tree) that the reference's
 * hot-path sources call, implemented here from what they compute:
 *   vector/matrix and their double variants: arrays indexed [nl..nh];
 *   gaussj: Gauss-Jordan elimination with full pivoting, a -> inverse, b -> x;
 *   covsrt: spreads the covariance of the fitted parameters over all ma;
 *   svdfit: weighted linear least squares to basis functions through a
 *           singular value decomposition (one-sided Jacobi here), singular
 *           values below 1e-5 of the largest dropped.
 * A singular system reaches nrerror(), which returns to the harness.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "cRecipes/nrutil.h"

void refshim_abort(void);

void nrerror(char error_text[])
{
    fprintf(stderr, "Numerical Recipes run-time error: %s\n", error_text);
    refshim_abort();
}

/* element k of a block with first index nl lives at block[k - nl] */
#define OFFSET_ALLOC(T, nl, nh) ((T *)calloc((size_t)((nh) - (nl) + 1), sizeof(T)) - (nl))

float *vector(long nl, long nh) { return OFFSET_ALLOC(float, nl, nh); }
int *ivector(long nl, long nh) { return OFFSET_ALLOC(int, nl, nh); }
double *dvector(long nl, long nh) { return OFFSET_ALLOC(double, nl, nh); }
void free_vector(float *v, long nl, long nh) { (void)nh; free(v + nl); }
void free_ivector(int *v, long nl, long nh) { (void)nh; free(v + nl); }
void free_dvector(double *v, long nl, long nh) { (void)nh; free(v + nl); }

float **matrix(long nrl, long nrh, long ncl, long nch)
{
    float **rows = OFFSET_ALLOC(float *, nrl, nrh);
    float *cells = (float *)calloc((size_t)(nrh - nrl + 1) * (size_t)(nch - ncl + 1), sizeof(float));
    for (long r = nrl; r <= nrh; r++) rows[r] = cells + (size_t)(r - nrl) * (size_t)(nch - ncl + 1) - ncl;
    return rows;
}

double **dmatrix(long nrl, long nrh, long ncl, long nch)
{
    double **rows = OFFSET_ALLOC(double *, nrl, nrh);
    double *cells = (double *)calloc((size_t)(nrh - nrl + 1) * (size_t)(nch - ncl + 1), sizeof(double));
    for (long r = nrl; r <= nrh; r++) rows[r] = cells + (size_t)(r - nrl) * (size_t)(nch - ncl + 1) - ncl;
    return rows;
}

void free_matrix(float **m, long nrl, long nrh, long ncl, long nch)
{
    (void)nrh; (void)nch;
    free(m[nrl] + ncl);
    free(m + nrl);
}

void free_dmatrix(double **m, long nrl, long nrh, long ncl, long nch)
{
    (void)nrh; (void)nch;
    free(m[nrl] + ncl);
    free(m + nrl);
}

void gaussj(float **a, int n, float **b, int m)
{
    int *used = (int *)calloc((size_t)n + 1, sizeof(int));   /* column already pivoted */
    int *prow = (int *)calloc((size_t)n + 1, sizeof(int));   /* row the pivot came from */
    int *pcol = (int *)calloc((size_t)n + 1, sizeof(int));   /* column of the pivot */
    for (int step = 1; step <= n; step++) {
        float best = -1.0f;
        int br = 0, bc = 0;
        for (int r = 1; r <= n; r++) {
            if (used[r]) continue;
            for (int c = 1; c <= n; c++) {
                if (used[c]) continue;
                float v = fabsf(a[r][c]);
                if (v > best) { best = v; br = r; bc = c; }
            }
        }
        if (best <= 0.0f) {
            free(used); free(prow); free(pcol);
            nrerror("gaussj: Singular Matrix");
            return;
        }
        used[bc] = 1;
        if (br != bc) { /* bring the pivot onto the diagonal */
            for (int c = 1; c <= n; c++) { float t = a[br][c]; a[br][c] = a[bc][c]; a[bc][c] = t; }
            for (int c = 1; c <= m; c++) { float t = b[br][c]; b[br][c] = b[bc][c]; b[bc][c] = t; }
        }
        prow[step] = br;
        pcol[step] = bc;
        float inv = 1.0f / a[bc][bc];
        a[bc][bc] = 1.0f;
        for (int c = 1; c <= n; c++) a[bc][c] *= inv;
        for (int c = 1; c <= m; c++) b[bc][c] *= inv;
        for (int r = 1; r <= n; r++) {
            if (r == bc) continue;
            float f = a[r][bc];
            a[r][bc] = 0.0f;
            for (int c = 1; c <= n; c++) a[r][c] -= a[bc][c] * f;
            for (int c = 1; c <= m; c++) b[r][c] -= b[bc][c] * f;
        }
    }
    for (int step = n; step >= 1; step--) /* undo the row interchanges on the inverse's columns */
        if (prow[step] != pcol[step])
            for (int r = 1; r <= n; r++) {
                float t = a[r][prow[step]];
                a[r][prow[step]] = a[r][pcol[step]];
                a[r][pcol[step]] = t;
            }
    free(used); free(prow); free(pcol);
}

void covsrt(float **covar, int ma, int ia[], int mfit)
{
    for (int i = mfit + 1; i <= ma; i++)
        for (int j = 1; j <= i; j++) covar[i][j] = covar[j][i] = 0.0f;
    int k = mfit;
    for (int j = ma; j >= 1; j--) {
        if (!ia[j]) continue;
        for (int i = 1; i <= ma; i++) { float t = covar[i][k]; covar[i][k] = covar[i][j]; covar[i][j] = t; }
        for (int i = 1; i <= ma; i++) { float t = covar[k][i]; covar[k][i] = covar[j][i]; covar[j][i] = t; }
        k--;
    }
}

void svdfit(void *x, double y[], double sig[], int ndata, double a[], int ma, double **u, double **v, double w[],
            double *chisq, void (*funcs)(void *, int32_t, double *, int32_t))
{
    double *af = (double *)malloc(sizeof(double) * (size_t)(ma + 1));
    double *rhs = (double *)malloc(sizeof(double) * (size_t)(ndata + 1));
    for (int i = 1; i <= ndata; i++) {
        (*funcs)(x, i, af, ma);
        for (int j = 1; j <= ma; j++) u[i][j] = af[j] / sig[i];
        rhs[i] = y[i] / sig[i];
    }
    for (int j = 1; j <= ma; j++)
        for (int k = 1; k <= ma; k++) v[j][k] = (j == k) ? 1.0 : 0.0;
    /* one-sided Jacobi: rotate column pairs of u until they are orthogonal */
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = 0.0;
        for (int p = 1; p < ma; p++)
            for (int q = p + 1; q <= ma; q++) {
                double al = 0, be = 0, ga = 0;
                for (int i = 1; i <= ndata; i++) {
                    al += u[i][p] * u[i][p];
                    be += u[i][q] * u[i][q];
                    ga += u[i][p] * u[i][q];
                }
                if (ga == 0.0 || fabs(ga) <= 1e-15 * sqrt(al * be)) continue;
                off = fmax(off, fabs(ga) / sqrt(al * be));
                double zeta = (be - al) / (2.0 * ga);
                double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
                for (int i = 1; i <= ndata; i++) {
                    double up = u[i][p], uq = u[i][q];
                    u[i][p] = c * up - s * uq;
                    u[i][q] = s * up + c * uq;
                }
                for (int i = 1; i <= ma; i++) {
                    double vp = v[i][p], vq = v[i][q];
                    v[i][p] = c * vp - s * vq;
                    v[i][q] = s * vp + c * vq;
                }
            }
        if (off < 1e-15) break;
    }
    double wmax = 0.0;
    for (int j = 1; j <= ma; j++) {
        double nrm = 0.0;
        for (int i = 1; i <= ndata; i++) nrm += u[i][j] * u[i][j];
        w[j] = sqrt(nrm);
        if (w[j] > 0)
            for (int i = 1; i <= ndata; i++) u[i][j] /= w[j];
        wmax = fmax(wmax, w[j]);
    }
    for (int j = 1; j <= ma; j++)
        if (w[j] < 1.0e-5 * wmax) w[j] = 0.0;
    for (int k = 1; k <= ma; k++) a[k] = 0.0;
    for (int j = 1; j <= ma; j++) {
        if (w[j] == 0.0) continue;
        double s = 0.0;
        for (int i = 1; i <= ndata; i++) s += u[i][j] * rhs[i];
        s /= w[j];
        for (int k = 1; k <= ma; k++) a[k] += s * v[k][j];
    }
    double chi = 0.0;
    for (int i = 1; i <= ndata; i++) {
        (*funcs)(x, i, af, ma);
        double s = 0.0;
        for (int j = 1; j <= ma; j++) s += a[j] * af[j];
        chi += pow((y[i] - s) / sig[i], 2);
    }
    *chisq = chi;
    free(af);
    free(rhs);
}
