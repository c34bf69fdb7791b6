/*
 * cRecipes/nrutil.h -- TEST INFRASTRUCTURE ONLY.  Declarations of the
 * Numerical Recipes in C routines (GrIMP's cRecipes, not part of the
 * reference tree) that the reference's hot-path sources call.  The
 * implementations in oracle/refshim/nr_shim.c are this project's own, written
 * from what the routines compute: offset-indexed vectors and matrices, a
 * Gauss-Jordan solve with inverse, covariance expansion, and a linear least
 * squares fit to basis functions.
 */
#ifndef REFSHIM_NRUTIL_H
#define REFSHIM_NRUTIL_H
#include <stdint.h>

float *vector(long nl, long nh);
int *ivector(long nl, long nh);
double *dvector(long nl, long nh);
float **matrix(long nrl, long nrh, long ncl, long nch);
double **dmatrix(long nrl, long nrh, long ncl, long nch);
void free_vector(float *v, long nl, long nh);
void free_ivector(int *v, long nl, long nh);
void free_dvector(double *v, long nl, long nh);
void free_matrix(float **m, long nrl, long nrh, long ncl, long nch);
void free_dmatrix(double **m, long nrl, long nrh, long ncl, long nch);
void nrerror(char error_text[]);

/* a[1..n][1..n] x = b[1..n][1..m]: a is replaced by its inverse, b by the solutions */
void gaussj(float **a, int n, float **b, int m);
/* spread the mfit x mfit covariance of the fitted parameters over ma x ma */
void covsrt(float **covar, int ma, int ia[], int mfit);
/* least squares a[1..ma] of y[1..ndata] against funcs(x, i, afunc, ma)
 * (GrIMP's double-precision variant over an opaque x) */
void svdfit(void *x, double y[], double sig[], int ndata, double a[], int ma, double **u, double **v, double w[],
            double *chisq, void (*funcs)(void *, int32_t, double *, int32_t));

#endif
