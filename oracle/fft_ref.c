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

/* ---------------------------------------------------------------- batched
 * Self-sorting (Stockham) decimation in frequency over the factors p of n:
 * a stage of length nc = p m with stride s maps
 *   y[q + s (p k + u)] = W_nc^{u k} sum_t x[q + s (k + t m)] W_p^{t u},
 * q < s, k < m, u < p, and the next stage runs on nc / p with stride s p; the
 * output comes out in natural order.  Every element is a vector of V
 * consecutive complex values (V transforms done together), so the inner loop
 * runs over s V contiguous values. */
#define OFFT_MAXSTAGE 32
#ifndef OFFT_BLOCK
#define OFFT_BLOCK 16
#endif

struct offt_batch {
    int n, sign, nst;
    int fac[OFFT_MAXSTAGE];
    ocplx *tw[OFFT_MAXSTAGE]; /* stage twiddles W_nc^{u k}: [k][u - 1] */
    ocplx *wp[OFFT_MAXSTAGE]; /* generic radix: W_p^e, e < p */
};

__attribute__((unused)) static offt_batch *ob_plan(int n, int sign)
{
    offt_batch *b = (offt_batch *)calloc(1, sizeof(offt_batch));
    int rem = n;
    b->n = n;
    b->sign = sign;
    while (rem % 4 == 0 && rem > 1) { b->fac[b->nst++] = 4; rem /= 4; }
    while (rem % 2 == 0 && rem > 1) { b->fac[b->nst++] = 2; rem /= 2; }
    for (int f = 3; rem > 1; f += 2)
        while (rem % f == 0) { b->fac[b->nst++] = f; rem /= f; }
    int nc = n;
    for (int st = 0; st < b->nst; st++) {
        const int p = b->fac[st], m = nc / p;
        b->tw[st] = (ocplx *)malloc(sizeof(ocplx) * (size_t)(m * (p - 1) > 0 ? m * (p - 1) : 1));
        for (int k = 0; k < m; k++)
            for (int u = 1; u < p; u++) {
                double ang = (double)sign * 2.0 * 3.14159265358979323846 * (double)(u * k) / (double)nc;
                b->tw[st][k * (p - 1) + u - 1].re = (REAL)cos(ang);
                b->tw[st][k * (p - 1) + u - 1].im = (REAL)sin(ang);
            }
        b->wp[st] = (ocplx *)malloc(sizeof(ocplx) * (size_t)p);
        for (int e = 0; e < p; e++) {
            double ang = (double)sign * 2.0 * 3.14159265358979323846 * (double)e / (double)p;
            b->wp[st][e].re = (REAL)cos(ang);
            b->wp[st][e].im = (REAL)sin(ang);
        }
        nc = m;
    }
    return b;
}

static void ob_destroy(offt_batch *b)
{
    if (!b) return;
    for (int st = 0; st < b->nst; st++) {
        free(b->tw[st]);
        free(b->wp[st]);
    }
    free(b);
}

/* One stage: x -> y, elements of L = s V consecutive complex values. */
static void ob_stage(const offt_batch *b, int st, int nc, size_t L, const ocplx *restrict x, ocplx *restrict y)
{
    const int p = b->fac[st], m = nc / p;
    const ocplx *tw = b->tw[st];
    const REAL sg = (REAL)b->sign;
    for (int k = 0; k < m; k++) {
        const ocplx *w = tw + (size_t)k * (p - 1);
        if (p == 4) {
            const ocplx *x0 = x + (size_t)k * L, *x1 = x + (size_t)(k + m) * L;
            const ocplx *x2 = x + (size_t)(k + 2 * m) * L, *x3 = x + (size_t)(k + 3 * m) * L;
            ocplx *y0 = y + (size_t)(4 * k) * L, *y1 = y0 + L, *y2 = y1 + L, *y3 = y2 + L;
            const ocplx w1 = w[0], w2 = w[1], w3 = w[2];
            for (size_t i = 0; i < L; i++) {
                const REAL ar = x0[i].re + x2[i].re, ai = x0[i].im + x2[i].im;
                const REAL br = x0[i].re - x2[i].re, bi = x0[i].im - x2[i].im;
                const REAL cr = x1[i].re + x3[i].re, ci = x1[i].im + x3[i].im;
                /* (sg i)(x1 - x3) */
                const REAL dr = -sg * (x1[i].im - x3[i].im), di = sg * (x1[i].re - x3[i].re);
                const REAL o0r = ar + cr, o0i = ai + ci, o2r = ar - cr, o2i = ai - ci;
                const REAL o1r = br + dr, o1i = bi + di, o3r = br - dr, o3i = bi - di;
                y0[i].re = o0r;
                y0[i].im = o0i;
                y1[i].re = o1r * w1.re - o1i * w1.im;
                y1[i].im = o1r * w1.im + o1i * w1.re;
                y2[i].re = o2r * w2.re - o2i * w2.im;
                y2[i].im = o2r * w2.im + o2i * w2.re;
                y3[i].re = o3r * w3.re - o3i * w3.im;
                y3[i].im = o3r * w3.im + o3i * w3.re;
            }
        } else if (p == 2) {
            const ocplx *x0 = x + (size_t)k * L, *x1 = x + (size_t)(k + m) * L;
            ocplx *y0 = y + (size_t)(2 * k) * L, *y1 = y0 + L;
            const ocplx w1 = w[0];
            for (size_t i = 0; i < L; i++) {
                const REAL dr = x0[i].re - x1[i].re, di = x0[i].im - x1[i].im;
                y0[i].re = x0[i].re + x1[i].re;
                y0[i].im = x0[i].im + x1[i].im;
                y1[i].re = dr * w1.re - di * w1.im;
                y1[i].im = dr * w1.im + di * w1.re;
            }
        } else if (p == 3) {
            const ocplx *x0 = x + (size_t)k * L, *x1 = x + (size_t)(k + m) * L, *x2 = x + (size_t)(k + 2 * m) * L;
            ocplx *y0 = y + (size_t)(3 * k) * L, *y1 = y0 + L, *y2 = y1 + L;
            const ocplx w1 = w[0], w2 = w[1];
            const REAL h = (REAL)0.5, r3 = sg * (REAL)0.86602540378443864676;
            for (size_t i = 0; i < L; i++) {
                const REAL sr = x1[i].re + x2[i].re, si = x1[i].im + x2[i].im;
                const REAL tr = x0[i].re - h * sr, ti = x0[i].im - h * si;
                const REAL ur = -r3 * (x1[i].im - x2[i].im), ui = r3 * (x1[i].re - x2[i].re);
                const REAL o1r = tr + ur, o1i = ti + ui, o2r = tr - ur, o2i = ti - ui;
                y0[i].re = x0[i].re + sr;
                y0[i].im = x0[i].im + si;
                y1[i].re = o1r * w1.re - o1i * w1.im;
                y1[i].im = o1r * w1.im + o1i * w1.re;
                y2[i].re = o2r * w2.re - o2i * w2.im;
                y2[i].im = o2r * w2.im + o2i * w2.re;
            }
        } else if (p == 7) {
            /* pairs t, 7 - t: with s_t = a_t + a_7-t, d_t = a_t - a_7-t,
             * b_u = a0 + sum_t s_t cos(2 pi t u / 7) + sg i sum_t d_t sin(2 pi t u / 7)
             * and b_7-u the same with the sine sum negated (u = 1, 2, 3) */
            const double tp = 2.0 * 3.14159265358979323846 / 7.0;
            const REAL c1 = (REAL)cos(tp), c2 = (REAL)cos(2 * tp), c3 = (REAL)cos(3 * tp);
            const REAL s1 = (REAL)(sg * sin(tp)), s2 = (REAL)(sg * sin(2 * tp)), s3 = (REAL)(sg * sin(3 * tp));
            const ocplx *x0 = x + (size_t)k * L, *x1 = x + (size_t)(k + m) * L, *x2 = x + (size_t)(k + 2 * m) * L;
            const ocplx *x3 = x + (size_t)(k + 3 * m) * L, *x4 = x + (size_t)(k + 4 * m) * L;
            const ocplx *x5 = x + (size_t)(k + 5 * m) * L, *x6 = x + (size_t)(k + 6 * m) * L;
            ocplx *y0 = y + (size_t)(7 * k) * L, *y1 = y0 + L, *y2 = y1 + L, *y3 = y2 + L;
            ocplx *y4 = y3 + L, *y5 = y4 + L, *y6 = y5 + L;
            const ocplx w1 = w[0], w2 = w[1], w3 = w[2], w4 = w[3], w5 = w[4], w6 = w[5];
            for (size_t i = 0; i < L; i++) {
                const REAL ar = x0[i].re, ai = x0[i].im;
                const REAL p1r = x1[i].re + x6[i].re, p1i = x1[i].im + x6[i].im;
                const REAL p2r = x2[i].re + x5[i].re, p2i = x2[i].im + x5[i].im;
                const REAL p3r = x3[i].re + x4[i].re, p3i = x3[i].im + x4[i].im;
                const REAL m1r = x1[i].re - x6[i].re, m1i = x1[i].im - x6[i].im;
                const REAL m2r = x2[i].re - x5[i].re, m2i = x2[i].im - x5[i].im;
                const REAL m3r = x3[i].re - x4[i].re, m3i = x3[i].im - x4[i].im;
                const REAL A1r = ar + p1r * c1 + p2r * c2 + p3r * c3, A1i = ai + p1i * c1 + p2i * c2 + p3i * c3;
                const REAL A2r = ar + p1r * c2 + p2r * c3 + p3r * c1, A2i = ai + p1i * c2 + p2i * c3 + p3i * c1;
                const REAL A3r = ar + p1r * c3 + p2r * c1 + p3r * c2, A3i = ai + p1i * c3 + p2i * c1 + p3i * c2;
                const REAL B1r = m1r * s1 + m2r * s2 + m3r * s3, B1i = m1i * s1 + m2i * s2 + m3i * s3;
                const REAL B2r = m1r * s2 - m2r * s3 - m3r * s1, B2i = m1i * s2 - m2i * s3 - m3i * s1;
                const REAL B3r = m1r * s3 - m2r * s1 + m3r * s2, B3i = m1i * s3 - m2i * s1 + m3i * s2;
                /* b_u = A_u + i B_u = (A_r - B_i, A_i + B_r); b_7-u = (A_r + B_i, A_i - B_r) */
                const REAL o1r = A1r - B1i, o1i = A1i + B1r, o6r = A1r + B1i, o6i = A1i - B1r;
                const REAL o2r = A2r - B2i, o2i = A2i + B2r, o5r = A2r + B2i, o5i = A2i - B2r;
                const REAL o3r = A3r - B3i, o3i = A3i + B3r, o4r = A3r + B3i, o4i = A3i - B3r;
                y0[i].re = ar + p1r + p2r + p3r;
                y0[i].im = ai + p1i + p2i + p3i;
                y1[i].re = o1r * w1.re - o1i * w1.im;
                y1[i].im = o1r * w1.im + o1i * w1.re;
                y2[i].re = o2r * w2.re - o2i * w2.im;
                y2[i].im = o2r * w2.im + o2i * w2.re;
                y3[i].re = o3r * w3.re - o3i * w3.im;
                y3[i].im = o3r * w3.im + o3i * w3.re;
                y4[i].re = o4r * w4.re - o4i * w4.im;
                y4[i].im = o4r * w4.im + o4i * w4.re;
                y5[i].re = o5r * w5.re - o5i * w5.im;
                y5[i].im = o5r * w5.im + o5i * w5.re;
                y6[i].re = o6r * w6.re - o6i * w6.im;
                y6[i].im = o6r * w6.im + o6i * w6.re;
            }
        } else {
            /* any other factor: the direct p-point sum, vectorised over i */
            const ocplx *wp = b->wp[st];
            for (int u = 0; u < p; u++) {
                ocplx *yu = y + (size_t)(p * k + u) * L;
                const ocplx wu = u == 0 ? (ocplx){1, 0} : w[u - 1];
                const ocplx *x0 = x + (size_t)k * L;
                for (size_t i = 0; i < L; i++) yu[i] = x0[i];
                for (int t = 1; t < p; t++) {
                    const ocplx *xt = x + (size_t)(k + t * m) * L;
                    const ocplx e = wp[(t * u) % p];
                    for (size_t i = 0; i < L; i++) {
                        yu[i].re += xt[i].re * e.re - xt[i].im * e.im;
                        yu[i].im += xt[i].re * e.im + xt[i].im * e.re;
                    }
                }
                for (size_t i = 0; i < L; i++) {
                    const REAL ar = yu[i].re, ai = yu[i].im;
                    yu[i].re = ar * wu.re - ai * wu.im;
                    yu[i].im = ar * wu.im + ai * wu.re;
                }
            }
        }
    }
}

/* V transforms of length n along the slow axis of a (n x V) array in a;
 * b is scratch of the same size; returns the array holding the result. */
__attribute__((unused)) static ocplx *ob_exec(const offt_batch *b, ocplx *a, ocplx *sc, size_t V)
{
    int nc = b->n;
    size_t s = 1;
    ocplx *x = a, *y = sc;
    for (int st = 0; st < b->nst; st++) {
        ob_stage(b, st, nc, s * V, x, y);
        nc /= b->fac[st];
        s *= (size_t)b->fac[st];
        ocplx *t = x;
        x = y;
        y = t;
    }
    return x;
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
#ifdef OFFT_BATCHED
    const size_t n = (size_t)na * nr;
    p->brows = ob_plan(nr, sign);
    p->bcols = ob_plan(na, sign);
    p->w0 = (ocplx *)malloc(sizeof(ocplx) * n);
    p->w1 = (ocplx *)malloc(sizeof(ocplx) * (size_t)mx * OFFT_BLOCK);
    p->w2 = (ocplx *)malloc(sizeof(ocplx) * (size_t)mx * OFFT_BLOCK);
#endif
    return p;
}

void offt2d_destroy(offt2d *p)
{
    if (!p) return;
    offt_destroy(p->rows);
    offt_destroy(p->cols);
    free(p->tmpA);
    free(p->tmpB);
    ob_destroy(p->brows);
    ob_destroy(p->bcols);
    free(p->w0);
    free(p->w1);
    free(p->w2);
    free(p);
}

void offt2d_exec(offt2d *p, const ocplx *in, ocplx *out)
{
#ifdef OFFT_BATCHED
    {
        /* columns, then rows, each in blocks of OFFT_BLOCK lines gathered
         * into a small contiguous buffer (n x block, cache-resident) and
         * transformed together */
        const int na = p->na, nr = p->nr, B = OFFT_BLOCK;
        for (int j0 = 0; j0 < nr; j0 += B) {
            const int bw = j0 + B < nr ? B : nr - j0;
            for (int i = 0; i < na; i++)
                for (int jj = 0; jj < bw; jj++) p->w1[(size_t)i * bw + jj] = in[(size_t)i * nr + j0 + jj];
            const ocplx *r = ob_exec(p->bcols, p->w1, p->w2, (size_t)bw);
            for (int i = 0; i < na; i++)
                for (int jj = 0; jj < bw; jj++) p->w0[(size_t)i * nr + j0 + jj] = r[(size_t)i * bw + jj];
        }
        for (int i0 = 0; i0 < na; i0 += B) {
            const int bh = i0 + B < na ? B : na - i0;
            for (int ii = 0; ii < bh; ii++)
                for (int j = 0; j < nr; j++) p->w1[(size_t)j * bh + ii] = p->w0[(size_t)(i0 + ii) * nr + j];
            const ocplx *r = ob_exec(p->brows, p->w1, p->w2, (size_t)bh);
            for (int ii = 0; ii < bh; ii++)
                for (int j = 0; j < nr; j++) out[(size_t)(i0 + ii) * nr + j] = r[(size_t)j * bh + ii];
        }
        return;
    }
#endif

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
