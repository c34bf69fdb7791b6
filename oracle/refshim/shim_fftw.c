/*
 * shim_fftw.c -- TEST INFRASTRUCTURE ONLY.  The FFTW 2.1.5 calls of the
 * reference's hot-path sources (fftw2d_create_plan, fftwnd_one,
 * fftw_create_plan_specific, fftw) over a DFT written here from its
 * definition: X[k] = sum_j x[j] exp(sign 2 pi i j k / n), unnormalised,
 * sign -1 for FFTW_FORWARD and +1 for FFTW_BACKWARD.  FFTW itself is not part
 * of the reference tree.  The transform is a self-sorting (Stockham) FFT over
 * the prime factors of n, any prime by its direct sum, evaluated in double
 * precision with twiddles from long double, and rounded to float
 * (fftw_real) once at the end; so the results are those of the exact DFT to
 * within float rounding.  Plans hold no pointers to the caller's arrays, and
 * out-of-place transforms leave their input unchanged.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fft/fftw-2.1.5/fftw/fftw.h"

typedef struct {
    double re, im;
} dcx;

struct refshim_fftw_plan {
    int n, sign, nfac;
    int fac[40];
    dcx *w; /* exp(sign 2 pi i e / n), e < n */
    dcx *a, *b;
};

struct refshim_fftwnd_plan {
    int nx, ny, inplace;
    fftw_plan px, py;
    dcx *buf; /* nx * ny */
    dcx *line;
};

static fftw_plan plan1(int n, int sign)
{
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    p->n = n;
    p->sign = sign;
    int r = n;
    for (int f = 2; r > 1; f++)
        while (r % f == 0) {
            p->fac[p->nfac++] = f;
            r /= f;
        }
    p->w = (dcx *)malloc(sizeof(dcx) * (size_t)(n > 0 ? n : 1));
    for (int e = 0; e < n; e++) {
        long double ang = (long double)sign * 2.0L * 3.141592653589793238462643383279502884L * e / n;
        p->w[e].re = (double)cosl(ang);
        p->w[e].im = (double)sinl(ang);
    }
    p->a = (dcx *)malloc(sizeof(dcx) * (size_t)(n > 0 ? n : 1));
    p->b = (dcx *)malloc(sizeof(dcx) * (size_t)(n > 0 ? n : 1));
    return p;
}

/* in-place transform of p->a (length n), self-sorting: after the stage with
 * radix q, the data are the length-(m q) DFTs of the decimated subsequences */
static void run1(fftw_plan p)
{
    const int n = p->n;
    dcx *x = p->a, *y = p->b;
    int m = 1; /* length of the sub-transforms done so far */
    for (int s = 0; s < p->nfac; s++) {
        const int q = p->fac[s];
        const int L = n / (m * q); /* number of interleaved sequences at this stage */
        /* x holds, for each residue l < L*q, the length-m DFT of x_l (the
         * subsequence with stride L*q): stored as x[l + (L q) k], k < m.
         * Combine q of them into length-(m q) DFTs stored as y[l + L k], k < m q */
        for (int l = 0; l < L; l++)
            for (int k = 0; k < m; k++)
                for (int t = 0; t < q; t++) { /* output index k + m t */
                    double re = 0.0, im = 0.0;
                    for (int u = 0; u < q; u++) {
                        const dcx v = x[(l + L * u) + (size_t)(L * q) * k];
                        /* twiddle exp(sign 2 pi i u (k + m t) / (m q)) */
                        const long e = ((long)u * (k + (long)m * t)) % (m * q);
                        const dcx w = p->w[e * (n / (m * q))];
                        re += v.re * w.re - v.im * w.im;
                        im += v.re * w.im + v.im * w.re;
                    }
                    y[l + (size_t)L * (k + m * t)].re = re;
                    y[l + (size_t)L * (k + m * t)].im = im;
                }
        dcx *t = x;
        x = y;
        y = t;
        m *= q;
    }
    if (x != p->a) memcpy(p->a, x, sizeof(dcx) * (size_t)n);
}

fftw_plan fftw_create_plan(int n, fftw_direction dir, int flags)
{
    (void)flags;
    return plan1(n, (int)dir);
}

fftw_plan fftw_create_plan_specific(int n, fftw_direction dir, int flags, fftw_complex *in, int istride,
                                    fftw_complex *out, int ostride)
{
    (void)in; (void)istride; (void)out; (void)ostride;
    return fftw_create_plan(n, dir, flags);
}

void fftw(fftw_plan p, int howmany, fftw_complex *in, int istride, int idist, fftw_complex *out, int ostride,
          int odist)
{
    for (int h = 0; h < howmany; h++) {
        const fftw_complex *src = in + (size_t)h * idist;
        for (int j = 0; j < p->n; j++) {
            p->a[j].re = src[(size_t)j * istride].re;
            p->a[j].im = src[(size_t)j * istride].im;
        }
        run1(p);
        fftw_complex *dst = (out ? out : in) + (size_t)h * (out ? odist : idist);
        const int os = out ? ostride : istride;
        for (int j = 0; j < p->n; j++) {
            dst[(size_t)j * os].re = (fftw_real)p->a[j].re;
            dst[(size_t)j * os].im = (fftw_real)p->a[j].im;
        }
    }
}

void fftw_one(fftw_plan p, fftw_complex *in, fftw_complex *out)
{
    fftw(p, 1, in, 1, p->n, out, 1, p->n);
}

void fftw_destroy_plan(fftw_plan p)
{
    if (!p) return;
    free(p->w);
    free(p->a);
    free(p->b);
    free(p);
}

fftwnd_plan fftw2d_create_plan(int nx, int ny, fftw_direction dir, int flags)
{
    fftwnd_plan p = (fftwnd_plan)calloc(1, sizeof(*p));
    p->nx = nx;
    p->ny = ny;
    p->inplace = (flags & FFTW_IN_PLACE) != 0;
    p->px = plan1(nx, (int)dir);
    p->py = plan1(ny, (int)dir);
    p->buf = (dcx *)malloc(sizeof(dcx) * (size_t)nx * ny);
    return p;
}

/* rows (length ny) then columns (length nx), all in double; one rounding */
void fftwnd_one(fftwnd_plan p, fftw_complex *in, fftw_complex *out)
{
    const int nx = p->nx, ny = p->ny;
    for (int i = 0; i < nx; i++) {
        for (int j = 0; j < ny; j++) {
            p->py->a[j].re = in[(size_t)i * ny + j].re;
            p->py->a[j].im = in[(size_t)i * ny + j].im;
        }
        run1(p->py);
        memcpy(p->buf + (size_t)i * ny, p->py->a, sizeof(dcx) * (size_t)ny);
    }
    for (int j = 0; j < ny; j++) {
        for (int i = 0; i < nx; i++) p->px->a[i] = p->buf[(size_t)i * ny + j];
        run1(p->px);
        for (int i = 0; i < nx; i++) p->buf[(size_t)i * ny + j] = p->px->a[i];
    }
    fftw_complex *dst = (p->inplace || !out) ? in : out;
    for (size_t k = 0; k < (size_t)nx * ny; k++) {
        dst[k].re = (fftw_real)p->buf[k].re;
        dst[k].im = (fftw_real)p->buf[k].im;
    }
}

void fftwnd(fftwnd_plan p, int howmany, fftw_complex *in, int istride, int idist, fftw_complex *out, int ostride,
            int odist)
{
    (void)istride; (void)ostride; /* the reference calls it with unit strides only */
    for (int h = 0; h < howmany; h++)
        fftwnd_one(p, in + (size_t)h * idist, out ? out + (size_t)h * odist : NULL);
}

void fftwnd_destroy_plan(fftwnd_plan p)
{
    if (!p) return;
    fftw_destroy_plan(p->px);
    fftw_destroy_plan(p->py);
    free(p->buf);
    free(p);
}
