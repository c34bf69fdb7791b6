/*
 * fft_ref.c -- test infrastructure only (CPU oracle): mixed-radix DFT with
 * FFTW 2 conventions.  See fft_ref.h.
 *
 * Algorithm: X[k + m*r] = sum_q W_n^{q(k+m r)} Y_q[k], where Y_q is the
 * length-m DFT of x[q::p] and n = p*m (decimation in time).  Twiddles are one
 * table W_N^e = exp(sign*2*pi*i*e/N) computed in double precision with libm and
 * rounded once to REAL.  Radix 2 and 4 have dedicated butterflies; any other
 * prime factor uses the direct p-point sum.
 */
#include "fft_ref.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OFFT_MAXFAC 32
#define OFFT_MAXRADIX 64

struct offt_plan {
    int n;
    int sign;
    int nfac;
    int fac[OFFT_MAXFAC];
    ocplx *tw; /* W_N^e, e in [0, n) */
};

offt_plan *offt_plan_1d(int n, int sign)
{
    offt_plan *p = (offt_plan *)calloc(1, sizeof(offt_plan));
    int rem = n, f;
    p->n = n;
    p->sign = sign;
    /* factor: 4s first, then 2, then odd primes */
    while (rem % 4 == 0 && rem > 1) { p->fac[p->nfac++] = 4; rem /= 4; }
    while (rem % 2 == 0 && rem > 1) { p->fac[p->nfac++] = 2; rem /= 2; }
    for (f = 3; rem > 1; f += 2) {
        while (rem % f == 0) { p->fac[p->nfac++] = f; rem /= f; }
    }
    p->tw = (ocplx *)malloc(sizeof(ocplx) * (size_t)(n > 0 ? n : 1));
    for (int e = 0; e < n; e++) {
        double ang = (double)sign * 2.0 * 3.14159265358979323846 * (double)e / (double)n;
        p->tw[e].re = (REAL)cos(ang);
        p->tw[e].im = (REAL)sin(ang);
    }
    return p;
}

void offt_destroy(offt_plan *p)
{
    if (!p) return;
    free(p->tw);
    free(p);
}

static inline ocplx cmul(ocplx a, ocplx b)
{
    ocplx c;
    c.re = a.re * b.re - a.im * b.im;
    c.im = a.re * b.im + a.im * b.re;
    return c;
}

static void rec(const offt_plan *P, ocplx *out, const ocplx *in, int n, int istride, int tstride,
                const int *fac)
{
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    const int p = fac[0], m = n / p;
    for (int q = 0; q < p; q++)
        rec(P, out + q * m, in + (size_t)q * istride, m, istride * p, tstride * p, fac + 1);
    const int N = P->n;
    const ocplx *W = P->tw;
    if (p == 2) {
        for (int k = 0; k < m; k++) {
            ocplx t0 = out[k];
            ocplx t1 = cmul(out[m + k], W[k * tstride]);
            out[k].re = t0.re + t1.re;
            out[k].im = t0.im + t1.im;
            out[m + k].re = t0.re - t1.re;
            out[m + k].im = t0.im - t1.im;
        }
    } else if (p == 4) {
        const REAL s = (REAL)P->sign;
        for (int k = 0; k < m; k++) {
            ocplx t0 = out[k];
            ocplx t1 = cmul(out[m + k], W[k * tstride]);
            ocplx t2 = cmul(out[2 * m + k], W[2 * k * tstride]);
            ocplx t3 = cmul(out[3 * m + k], W[3 * k * tstride]);
            ocplx a0 = {t0.re + t2.re, t0.im + t2.im};
            ocplx a1 = {t0.re - t2.re, t0.im - t2.im};
            ocplx b0 = {t1.re + t3.re, t1.im + t3.im};
            ocplx b1 = {t1.re - t3.re, t1.im - t3.im};
            /* (s*i) * b1 = (-s*b1.im, s*b1.re) */
            ocplx jb1 = {-s * b1.im, s * b1.re};
            out[k].re = a0.re + b0.re;
            out[k].im = a0.im + b0.im;
            out[2 * m + k].re = a0.re - b0.re;
            out[2 * m + k].im = a0.im - b0.im;
            out[m + k].re = a1.re + jb1.re;
            out[m + k].im = a1.im + jb1.im;
            out[3 * m + k].re = a1.re - jb1.re;
            out[3 * m + k].im = a1.im - jb1.im;
        }
    } else {
        ocplx t[OFFT_MAXRADIX];
        const int Np = N / p; /* W_p = W_N^{N/p} */
        for (int k = 0; k < m; k++) {
            for (int q = 0; q < p; q++) t[q] = cmul(out[q * m + k], W[(q * k * tstride) % N]);
            for (int r = 0; r < p; r++) {
                ocplx acc = t[0];
                for (int q = 1; q < p; q++) {
                    ocplx v = cmul(t[q], W[((q * r) % p) * Np]);
                    acc.re += v.re;
                    acc.im += v.im;
                }
                out[r * m + k] = acc;
            }
        }
    }
}

void offt_exec_1d(const offt_plan *p, const ocplx *in, ocplx *out)
{
    rec(p, out, in, p->n, 1, 1, p->fac);
}

offt2d *offt2d_plan(int na, int nr, int sign)
{
    offt2d *p = (offt2d *)calloc(1, sizeof(offt2d));
    int mx = na > nr ? na : nr;
    p->na = na;
    p->nr = nr;
    p->rows = offt_plan_1d(nr, sign);
    p->cols = offt_plan_1d(na, sign);
    p->tmpA = (ocplx *)malloc(sizeof(ocplx) * (size_t)mx);
    p->tmpB = (ocplx *)malloc(sizeof(ocplx) * (size_t)mx);
    return p;
}

void offt2d_destroy(offt2d *p)
{
    if (!p) return;
    offt_destroy(p->rows);
    offt_destroy(p->cols);
    free(p->tmpA);
    free(p->tmpB);
    free(p);
}

void offt2d_exec(offt2d *p, const ocplx *in, ocplx *out)
{
    const int na = p->na, nr = p->nr;
    for (int i = 0; i < na; i++) {
        memcpy(p->tmpA, in + (size_t)i * nr, sizeof(ocplx) * (size_t)nr);
        offt_exec_1d(p->rows, p->tmpA, p->tmpB);
        memcpy(out + (size_t)i * nr, p->tmpB, sizeof(ocplx) * (size_t)nr);
    }
    for (int j = 0; j < nr; j++) {
        for (int i = 0; i < na; i++) p->tmpA[i] = out[(size_t)i * nr + j];
        offt_exec_1d(p->cols, p->tmpA, p->tmpB);
        for (int i = 0; i < na; i++) out[(size_t)i * nr + j] = p->tmpB[i];
    }
}
