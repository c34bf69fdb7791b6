/*
 * fft/fftw-2.1.5/fftw/fftw.h -- TEST INFRASTRUCTURE ONLY.  The subset of the
 * FFTW 2.1.5 interface (single precision: fftw_real is float, as the
 * reference's float32 image reads require) that the reference's hot-path
 * sources call, over an independent DFT written from the definition
 * (oracle/refshim/fftw_shim.c).  FFTW 2.1.5 is not part of the reference tree.
 * Semantics kept: unnormalised transforms, FFTW_FORWARD = exp(-2 pi i jk/N),
 * FFTW_BACKWARD = exp(+...), 2-D transforms over row-major arrays, plans
 * out of place unless FFTW_IN_PLACE is given.
 */
#ifndef REFSHIM_FFTW_H
#define REFSHIM_FFTW_H

typedef float fftw_real;
typedef struct {
    fftw_real re, im;
} fftw_complex;

typedef enum { FFTW_FORWARD = -1, FFTW_BACKWARD = 1 } fftw_direction;

#define FFTW_ESTIMATE (0)
#define FFTW_MEASURE (1)
#define FFTW_OUT_OF_PLACE (0)
#define FFTW_IN_PLACE (8)
#define FFTW_USE_WISDOM (16)

typedef struct refshim_fftw_plan *fftw_plan;
typedef struct refshim_fftwnd_plan *fftwnd_plan;

fftw_plan fftw_create_plan(int n, fftw_direction dir, int flags);
fftw_plan fftw_create_plan_specific(int n, fftw_direction dir, int flags, fftw_complex *in, int istride,
                                    fftw_complex *out, int ostride);
void fftw(fftw_plan plan, int howmany, fftw_complex *in, int istride, int idist, fftw_complex *out, int ostride,
          int odist);
void fftw_one(fftw_plan plan, fftw_complex *in, fftw_complex *out);
void fftw_destroy_plan(fftw_plan plan);

fftwnd_plan fftw2d_create_plan(int nx, int ny, fftw_direction dir, int flags);
void fftwnd_one(fftwnd_plan p, fftw_complex *in, fftw_complex *out);
void fftwnd(fftwnd_plan p, int howmany, fftw_complex *in, int istride, int idist, fftw_complex *out, int ostride,
            int odist);
void fftwnd_destroy_plan(fftwnd_plan plan);

#endif
