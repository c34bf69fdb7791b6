/*
 * fft_ref.h -- test infrastructure only (CPU oracle).  Mixed-radix complex DFT
 * with the conventions of FFTW 2.1.5 as the reference uses it
 * (fftw2d_create_plan / fftwnd_one, Strack/speckleTrack.c:1507-1550):
 * unnormalised, FFTW_FORWARD = exp(-2*pi*i*j*k/N), FFTW_BACKWARD = exp(+...),
 * 2-D transforms over row-major [rows][cols] arrays.
 * FFTW 2.1.5 itself is not in the reference tree; this is an independent
 * implementation of the same mathematical transform, written from the DFT
 * definition (recursive decimation in time over the prime factors of N).
 * Built with OFFT_BATCHED (the float library, the timed CPU baseline), the 2-D
 * transform is instead a self-sorting (Stockham) decimation-in-frequency FFT
 * applied to whole rows at a time, which a compiler vectorises: FFTW is an
 * optimised library, so the baseline's FFT has to be a competitive one.
 */
#ifndef ORACLE_FFT_REF_H
#define ORACLE_FFT_REF_H

#ifndef REAL
#define REAL double
#endif

typedef struct {
    REAL re;
    REAL im;
} ocplx;

#define OFFT_FORWARD (-1)
#define OFFT_BACKWARD (1)

typedef struct offt_plan offt_plan;

offt_plan *offt_plan_1d(int n, int sign);
void offt_destroy(offt_plan *p);
/* out-of-place 1-D transform; in and out must not overlap */
void offt_exec_1d(const offt_plan *p, const ocplx *in, ocplx *out);

typedef struct offt_batch offt_batch;

typedef struct {
    int na, nr;
    offt_plan *rows; /* length nr */
    offt_plan *cols; /* length na */
    ocplx *tmpA, *tmpB;
    /* OFFT_BATCHED builds: self-sorting transforms batched across the other
     * axis (see fft_ref.c), with three na x nr work arrays */
    offt_batch *brows, *bcols;
    ocplx *w0, *w1, *w2;
} offt2d;

offt2d *offt2d_plan(int na, int nr, int sign);
void offt2d_destroy(offt2d *p);
/* out-of-place or in-place 2-D transform of a row-major na x nr array */
void offt2d_exec(offt2d *p, const ocplx *in, ocplx *out);

#endif
