/*
 * strack_ref.c -- TEST INFRASTRUCTURE ONLY (CPU oracle, pinned to the reference build by tests/test_ref_pin.py).
 *
 * Restatement of speckleTrack() and its helpers, Strack/speckleTrack.c and
 * Strack/dopplerEstimation.c.  Each function cites the reference lines it
 * follows.  Module globals of the reference become fields of StCtx so the
 * oracle is reentrant; the control flow, the index maps and the arithmetic
 * types follow the reference.  REAL is the FFT sample type (the reference's
 * fftw_real; float, since the SLC buffers are read as 8-byte fftw_complex
 * samples of float32 files, speckleTrack.c:1380-1384), FLT the type of the
 * reference's `float` working variables.  The f64 build makes both double.
 *
 * Pinned undefined behaviour of the reference (documented, reproduced here):
 *  - rangeShift is never assigned in strack: pinned to 0 (:632-634).
 *  - r2/a2 are uninitialised before the first point: pinned to 0 (fails the
 *    strict bounds test); a grid lookup with no value keeps the previous
 *    point's r2/a2 (:820-826).
 *  - aZDefocus is never initialised: pinned to 0 (:1980-1986 mallocs it);
 *    ampTrackFast's write through uninitialised i,j (:537) is a no-op.
 *  - a NaN Doppler angle (a constant patch) gives roll 0.
 *  - gaussj on a singular 3x3 system (process exit in Numerical Recipes)
 *    ends that fit with the current parameters.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "fft_ref.h"
#include "oracle.h"

#ifndef FLT
#define FLT REAL
#endif

#define NOVER 12
#define NFAST 8
#define LA 2
#define OS 2
#define OSA 2
#define NGAUSS 18
#define AZ 1
#define RG 2
#define ST_PI 3.14159265358979323846
#define LARGEINT 2000000000
#define TRUE 1
#define FALSE 0

/* ---------------------------------------------------------------- image */

static inline uint32_t bswap32(uint32_t v)
{
    return (v >> 24) | ((v >> 8) & 0xff00u) | ((v << 8) & 0xff0000u) | (v << 24);
}

/* One sample of an SLC image, as loadBuffer delivers it (speckleTrack.c:1369-1399):
 * float32 complex swapped when MSB; int16 complex as integers. */
static inline void sample_at(const sb_image *im, int row, int col, REAL *re, REAL *imv)
{
    size_t k = (size_t)row * (size_t)im->nr + (size_t)col;
    if (im->sampleType == SB_CFLOAT32) {
        const uint32_t *w = (const uint32_t *)im->data + 2 * k;
        uint32_t a = w[0], b = w[1];
        float fa, fb;
        if (im->byteOrder == SB_MSB) { a = bswap32(a); b = bswap32(b); }
        memcpy(&fa, &a, 4);
        memcpy(&fb, &b, 4);
        *re = (REAL)fa;
        *imv = (REAL)fb;
    } else {
        const uint16_t *w = (const uint16_t *)im->data + 2 * k;
        uint16_t a = w[0], b = w[1];
        if (im->byteOrder == SB_MSB) {
            a = (uint16_t)((a >> 8) | (a << 8));
            b = (uint16_t)((b >> 8) | (b << 8));
        }
        *re = (REAL)(int16_t)a;
        *imv = (REAL)(int16_t)b;
    }
}

/* ---------------------------------------------------------------- context */

typedef struct {
    int wr, wa; /* patch size (not oversampled) */
    ocplx *in1, *in2, *f1, *f2, *f1a, *f2a, *im1, *im2, *fa1, *fa2, *ps, *ca;
    FLT *caMag;
    offt2d *fwdIn, *revPad, *fwd, *rev;
} AmpBufs;

typedef struct {
    const sb_track_params *p;
    const sb_image *img1, *img2;
    int wR, wA, wRa, wAa;
    int azShift;
    int rangeShift;
    double p1, p2;
    FLT *hanning;
    ocplx *patch1, *patch2, *fftF1os, *fftF2os, *psNoPad, *cNoPad;
    FLT *cNoPadMag;
    offt2d *cForwardIn, *cReverseNoPad, *cForwardFast, *cReverseFast;
    ocplx *cFast, *psFast, *psFastOver, *cFastOver;
    AmpBufs amp[2];
    /* interferogram phase correction (initPhaseCorrect, speckleTrack.c:1576-1601) */
    int intPs, intPSA, intPSR;
    ocplx *intPatch, *fftIntPatch, *fftIntPatchOver, *intPatchOver;
    offt2d *intForward, *intBackward;
    float *aZDefocus; /* output grid */
    int64_t nComplex, nAmp, nAmpL, nFail;
} StCtx;

static ocplx *cbuf(size_t n) { return (ocplx *)calloc(n, sizeof(ocplx)); }

/* ---------------------------------------------------------------- utilities */

static int inBounds(int r1, int a1, int wR, int wA, int sR, int sA)
{
    /* speckleTrack.c:1943-1946 (strict) */
    return (r1 > 0 && (r1 + wR) < sR && a1 > 0 && (a1 + wA) < sA);
}

static int boundsCheck(StCtx *c, int r1, int a1, int r2, int a2, int wR, int wA)
{
    /* speckleTrack.c:1822-1828 */
    int in1 = inBounds(r1, a1, wR, wA, c->img1->nr, c->img1->na);
    int in2 = inBounds(r2, a2, wR, wA, c->img2->nr, c->img2->na);
    return in1 && in2;
}

static FLT absCmpx(ocplx x, int noSquareRoot)
{
    /* speckleTrack.c:1810-1817: float result */
    FLT x2 = (FLT)(x.re * x.re + x.im * x.im);
    if (noSquareRoot) return x2;
    return (FLT)sqrt((double)x2);
}

static int maskValue(StCtx *c, int r1, int a1)
{
    /* speckleTrack.c:1951-1965 (C division truncates toward zero) */
    const sb_mask *m = c->p->mask;
    if (m == NULL) return 1;
    int ia1 = (a1 + c->wA / 2 - m->a0) / m->nal;
    int ir1 = (r1 + c->wR / 2 - m->r0) / m->nrl;
    if (ia1 < 0 || ia1 >= m->na || ir1 < 0 || ir1 >= m->nr) return 0;
    return (int)(signed char)m->mask[(size_t)ia1 * m->nr + ir1];
}

static void getShifts(double range, double azimuth, const sb_offset_grid *o, double *dr, double *da)
{
    /* speckleTrack.c:1857-1940 */
    float t, u, p1, p2, p3, p4;
    float minvalue = (float)((float)-LARGEINT * 0.9);
    range = (range - o->r0) / o->deltaR;
    azimuth = (azimuth - o->a0) / o->deltaA;
    if (range < 0.0 || azimuth < 0.0 || (int)range >= o->nr || (int)azimuth >= o->na) {
        *dr = -LARGEINT;
        *da = -LARGEINT;
        return;
    }
    int j = (int)range, i = (int)azimuth;
    const float *R = o->dr, *A = o->da;
    const int nr = o->nr;
#define RI(ii, jj) R[(size_t)(ii) * nr + (jj)]
#define AI(ii, jj) A[(size_t)(ii) * nr + (jj)]
    if (j == (o->nr - 1) || i == (o->na - 1)) {
        *dr = RI(i, j);
        *da = AI(i, j);
        if (*dr < minvalue || *da < minvalue) {
            *dr = -LARGEINT;
            *da = -LARGEINT;
        }
        return;
    }
    t = (float)(range - (double)j);
    u = (float)(azimuth - (double)i);
    p1 = RI(i, j); p2 = RI(i, j + 1); p3 = RI(i + 1, j + 1); p4 = RI(i + 1, j);
    if (p1 <= minvalue || p2 <= minvalue || p3 <= minvalue || p4 <= minvalue) {
        float mx = fmaxf(fmaxf(fmaxf(p1, p2), p3), p4);
        *dr = mx;
        if (*dr < minvalue) {
            *dr = -LARGEINT;
            *da = -LARGEINT;
            return;
        }
    } else {
        *dr = (float)((1.0 - t) * (1.0 - u) * p1 + t * (1.0 - u) * p2 + t * u * p3 + (1.0 - t) * u * p4);
    }
    p1 = AI(i, j); p2 = AI(i, j + 1); p3 = AI(i + 1, j + 1); p4 = AI(i + 1, j);
    if (p1 <= minvalue || p2 <= minvalue || p3 <= minvalue || p4 <= minvalue) {
        float mx = fmaxf(fmaxf(fmaxf(p1, p2), p3), p4);
        *da = mx;
        if (*da < minvalue) {
            *dr = -LARGEINT;
            *da = -LARGEINT;
            return;
        }
    } else {
        *da = (float)((1.0 - t) * (1.0 - u) * p1 + t * (1.0 - u) * p2 + t * u * p3 + (1.0 - t) * u * p4);
    }
#undef RI
#undef AI
}

static void findImage2Pos(StCtx *c, int r1, int a1, int *r2, int *a2)
{
    /* speckleTrack.c:810-847 */
    const sb_track_params *p = c->p;
    double aShift = 0, rShift = 0, sc = (double)p->scaleFactor;
    int haveShift = FALSE;
    if (p->polyShift == FALSE) {
        getShifts(r1, a1, p->initOffsets, &rShift, &aShift);
        if (rShift > (-LARGEINT + 1))
            haveShift = TRUE;
        else
            return; /* keeps the previous r2, a2 */
    }
    if (p->polyShift == TRUE || haveShift == FALSE) {
        rShift = p->rShiftPoly[0] + (double)(r1 * sc) * p->rShiftPoly[1] + (double)(a1 * sc) * p->rShiftPoly[2];
        aShift = p->aShiftPoly[0] + (double)(r1 * sc) * p->aShiftPoly[1] + (double)(a1 * sc) * p->aShiftPoly[2];
    }
    rShift /= sc;
    aShift /= sc;
    *r2 = (rShift >= 0) ? r1 + (int)(rShift + 0.5) : r1 + (int)(rShift - 0.5);
    *a2 = (aShift >= 0) ? a1 + (int)(aShift + 0.5) : a1 + (int)(aShift - 0.5);
}

static void computeHanning(StCtx *c)
{
    /* speckleTrack.c:1830-1852 (square windows: the j index uses wA/2) */
    int wA = c->wA, wR = c->wR;
    for (int i = 0; i < wA / 2; i++) {
        int i1 = wA / 2 + i, i2 = wA / 2 - i - 1;
        double wi = 0.5 * (1.0 + cos((2.0 * ST_PI) * (double)i / (double)(wA - 1)));
        for (int j = 0; j < wR / 2; j++) {
            int j1 = wA / 2 + j, j2 = wA / 2 - j - 1;
            double wj = 0.5 * (1.0 + cos((2.0 * ST_PI) * (double)j / (double)(wR - 1)));
            FLT h = (FLT)(wi * wj);
            c->hanning[i1 * wR + j1] = h;
            c->hanning[i2 * wR + j2] = h;
            c->hanning[i2 * wR + j1] = h;
            c->hanning[i1 * wR + j2] = h;
        }
    }
}

/* zeroPadFFT, speckleTrack.c:2014-2038: spectrum quadrants to the corners of
 * a larger zeroed array with an optional roll (dA, dR). */
static void zeroPadFFT(ocplx *pad, int pSA, int pSR, const ocplx *orig, int oSA, int oSR, int dA, int dR)
{
    memset(pad, 0, sizeof(ocplx) * (size_t)pSA * pSR);
    for (int i = 0; i < oSA / 2; i++) {
        int i1 = pSA - oSA / 2 + i;
        int i2 = (oSA / 2 + i + dA) % oSA;
        int ia = (i + dA) % oSA;
        int j1 = pSR - oSR / 2;
        int j2 = oSR / 2 + dR;
        for (int j = 0; j < oSR / 2; j++) {
            int ja = (j + dR) % oSR;
            int j2a = j2 % oSR;
            pad[i * pSR + j] = orig[ia * oSR + ja];
            pad[i1 * pSR + j] = orig[i2 * oSR + ja];
            pad[i1 * pSR + j1] = orig[i2 * oSR + j2a];
            pad[i * pSR + j1] = orig[ia * oSR + j2a];
            j1++;
            j2++;
        }
    }
}

/* ---------------------------------------------------------------- Doppler */

static double computeSingleDop(const ocplx *image, int nAz, int nRg)
{
    /* dopplerEstimation.c:42-88: complex mean removal, lag-1 azimuth product */
    double mean_re = 0., mean_im = 0., sum_re = 0.0, sum_im = 0.0;
    long double denom = (long double)nRg * (long double)nAz;
    for (int j = 0; j < nRg; ++j)
        for (int i = 0; i < nAz; ++i) {
            mean_re += (long double)image[i * nRg + j].re;
            mean_im += (long double)image[i * nRg + j].im;
        }
    mean_re /= denom;
    mean_im /= denom;
    for (int j = 0; j < nRg; ++j)
        for (int i = 0; i < nAz - 1; ++i) {
            const ocplx *p0 = &image[i * nRg + j], *p1 = &image[(i + 1) * nRg + j];
            double a_re = (long double)p1->re - mean_re;
            double a_im = (long double)p1->im - mean_im;
            double b_re = (long double)p0->re - mean_re;
            double b_im = (long double)p0->im - mean_im;
            sum_re += a_re * b_re + a_im * b_im;
            sum_im += a_im * b_re - a_re * b_im;
        }
    if (sum_re == 0.0 && sum_im == 0.0) return NAN;
    return atan2(sum_im, sum_re);
}

static int iround(double x) { return (x >= 0.0) ? (int)(x + 0.5) : (int)(x - 0.5); }

static int estDopCarrier1(int wA, const ocplx *im1, const ocplx *im2, int nAz, int nRg)
{
    /* dopplerEstimation.c:25-40; returns the new trackPar->azShift */
    double angle1 = computeSingleDop(im1, nAz, nRg);
    double angle2 = computeSingleDop(im2, nAz, nRg);
    double v = (double)(nAz / 2) * (angle1 + angle2) * .5 / ST_PI;
    int shift = (v != v) ? 0 : iround(v); /* pinned: NaN angle -> 0 */
    if (shift < 0) shift += nAz;
    return (int)((float)shift * (float)wA / (float)nAz);
}

/* ---------------------------------------------------------------- LM fit */

typedef struct {
    FLT x;
} XY;

static void myGauss1D(FLT x, const FLT a[], FLT *y, FLT dyda[])
{
    /* speckleTrack.c:2445-2465 */
    FLT sig = a[3];
    FLT t = x - a[2];
    FLT argx = (FLT)(0.5 * t * t / (sig * sig));
    FLT ex = (FLT)exp((double)-argx);
    *y = a[1] * ex;
    dyda[1] = ex;
    dyda[2] = *y * t / (sig * sig);
    dyda[3] = *y * t * t / (sig * sig * sig);
}

static void mrqcof(const FLT *x, const FLT *y, const FLT *sig, int ndata, const FLT a[], FLT alpha[4][4],
                   FLT beta[4], FLT *chisq)
{
    /* mrqcofMod, speckleTrack.c:2309-2351 (ia = {_,1,1,1}, ma = mfit = 3) */
    FLT ymod, wt, sig2i, dy, dyda[4];
    for (int j = 1; j <= 3; j++) {
        for (int k = 1; k <= j; k++) alpha[j][k] = 0.0;
        beta[j] = 0.0;
    }
    *chisq = 0.0;
    for (int i = 1; i <= ndata; i++) {
        myGauss1D(x[i], a, &ymod, dyda);
        sig2i = (FLT)(1.0 / (sig[i] * sig[i]));
        dy = y[i] - ymod;
        for (int l = 1; l <= 3; l++) {
            wt = dyda[l] * sig2i;
            for (int m = 1; m <= l; m++) alpha[l][m] += wt * dyda[m];
            beta[l] += dy * wt;
        }
        *chisq += dy * dy * sig2i;
    }
    for (int j = 2; j <= 3; j++)
        for (int k = 1; k < j; k++) alpha[k][j] = alpha[j][k];
}

/* Gauss-Jordan elimination with full pivoting on an n x n system with one
 * right-hand side (the Numerical Recipes gaussj algorithm).  Returns 0 if the
 * matrix is singular. */
static int gaussj3(FLT a[4][4], int n, FLT b[4])
{
    int indxc[4], indxr[4], ipiv[4] = {0, 0, 0, 0};
    int irow = 0, icol = 0;
    for (int i = 1; i <= n; i++) {
        FLT big = 0.0;
        for (int j = 1; j <= n; j++)
            if (ipiv[j] != 1)
                for (int k = 1; k <= n; k++) {
                    if (ipiv[k] == 0) {
                        if (fabs((double)a[j][k]) >= big) {
                            big = (FLT)fabs((double)a[j][k]);
                            irow = j;
                            icol = k;
                        }
                    } else if (ipiv[k] > 1)
                        return 0;
                }
        ++(ipiv[icol]);
        if (irow != icol) {
            for (int l = 1; l <= n; l++) { FLT t = a[irow][l]; a[irow][l] = a[icol][l]; a[icol][l] = t; }
            FLT t = b[irow]; b[irow] = b[icol]; b[icol] = t;
        }
        indxr[i] = irow;
        indxc[i] = icol;
        if (a[icol][icol] == 0.0) return 0;
        FLT pivinv = (FLT)(1.0 / a[icol][icol]);
        a[icol][icol] = 1.0;
        for (int l = 1; l <= n; l++) a[icol][l] *= pivinv;
        b[icol] *= pivinv;
        for (int ll = 1; ll <= n; ll++)
            if (ll != icol) {
                FLT dum = a[ll][icol];
                a[ll][icol] = 0.0;
                for (int l = 1; l <= n; l++) a[ll][l] -= a[icol][l] * dum;
                b[ll] -= b[icol] * dum;
            }
    }
    for (int l = n; l >= 1; l--) {
        if (indxr[l] != indxc[l])
            for (int k = 1; k <= n; k++) {
                FLT t = a[k][indxr[l]]; a[k][indxr[l]] = a[k][indxc[l]]; a[k][indxc[l]] = t;
            }
    }
    return 1;
}

typedef struct {
    FLT alamda, ochisq;
    FLT alpha[4][4], beta[4];
} LMState;

/* mrqminMod, speckleTrack.c:2353-2416: one Levenberg-Marquardt step. Returns 0
 * when gaussj meets a singular matrix. */
static int mrqmin(const FLT *x, const FLT *y, const FLT *sig, int ndata, FLT a[4], LMState *s, FLT *chisq)
{
    FLT covar[4][4], da[4], atry[4];
    if (s->alamda < 0.0) {
        s->alamda = (FLT)0.001;
        mrqcof(x, y, sig, ndata, a, s->alpha, s->beta, chisq);
        s->ochisq = *chisq;
    }
    for (int j = 1; j <= 3; j++) {
        for (int k = 1; k <= 3; k++) covar[j][k] = s->alpha[j][k];
        covar[j][j] = s->alpha[j][j] * (FLT)(1.0 + s->alamda);
        da[j] = s->beta[j];
    }
    if (!gaussj3(covar, 3, da)) return 0;
    for (int l = 1; l <= 3; l++) atry[l] = a[l] + da[l];
    atry[0] = a[0];
    mrqcof(x, y, sig, ndata, atry, covar, da, chisq);
    if (*chisq < s->ochisq) {
        s->alamda *= (FLT)0.1;
        s->ochisq = *chisq;
        for (int j = 1; j <= 3; j++) {
            for (int k = 1; k <= 3; k++) s->alpha[j][k] = covar[j][k];
            s->beta[j] = da[j];
        }
        for (int l = 1; l <= 3; l++) a[l] = atry[l];
    } else {
        s->alamda *= (FLT)10.0;
        *chisq = s->ochisq;
    }
    return 1;
}

/* gaussPeak1D, speckleTrack.c:2137-2202: 18 samples through the coarse peak,
 * normalised to their max; <=5 LM steps; sigma = a[3]/2. */
static void gaussPeak1D(const FLT *cMag, int ncol, int iMax, int jMax, int AzOrRg, FLT *sigma, FLT *peakRatio)
{
    FLT xs[NGAUSS + 1], ys[NGAUSS + 1], sg[NGAUSS + 1];
    FLT maxC = 0;
    int iData = 1;
    for (int i = 0; i < NGAUSS; i++) {
        int i1;
        if (AzOrRg == AZ) {
            i1 = iMax - NGAUSS / 2 + i;
            ys[iData] = cMag[i1 * ncol + jMax];
        } else {
            i1 = jMax - NGAUSS / 2 + i;
            ys[iData] = cMag[iMax * ncol + i1];
        }
        sg[iData] = (FLT)0.1;
        xs[iData] = (FLT)i1;
        maxC = (maxC > ys[iData]) ? maxC : ys[iData];
        iData++;
    }
    for (int i = 0; i < NGAUSS; i++) ys[i + 1] /= maxC;
    FLT a[4], chisq;
    LMState st;
    st.alamda = -1.;
    a[0] = 0;
    a[1] = 1;
    a[2] = xs[NGAUSS / 2 + 1];
    a[3] = 2;
    FLT lasti = (FLT)2e9;
    for (int i = 0; i < 5; i++) {
        if (!mrqmin(xs, ys, sg, iData - 1, a, &st, &chisq)) break;
        if (fabs((double)(a[2] - lasti)) < 0.001) break;
        lasti = a[2];
    }
    *sigma = (FLT)(a[3] * .5);
    *peakRatio = a[1];
}

/* ---------------------------------------------------------------- 2-D fit (-gauss) */

/* Gauss-Jordan with full pivoting for the 5 x 5 system of the 2-D fit (the
 * same Numerical Recipes algorithm as gaussj3). */
static int gaussj5(FLT a[6][6], int n, FLT b[6])
{
    int indxc[6], indxr[6], ipiv[6] = {0, 0, 0, 0, 0, 0};
    int irow = 0, icol = 0;
    for (int i = 1; i <= n; i++) {
        FLT big = 0.0;
        for (int j = 1; j <= n; j++)
            if (ipiv[j] != 1)
                for (int k = 1; k <= n; k++) {
                    if (ipiv[k] == 0) {
                        if (fabs((double)a[j][k]) >= big) {
                            big = (FLT)fabs((double)a[j][k]);
                            irow = j;
                            icol = k;
                        }
                    } else if (ipiv[k] > 1)
                        return 0;
                }
        ++(ipiv[icol]);
        if (irow != icol) {
            for (int l = 1; l <= n; l++) { FLT t = a[irow][l]; a[irow][l] = a[icol][l]; a[icol][l] = t; }
            FLT t = b[irow]; b[irow] = b[icol]; b[icol] = t;
        }
        indxr[i] = irow;
        indxc[i] = icol;
        if (a[icol][icol] == 0.0) return 0;
        FLT pivinv = (FLT)(1.0 / a[icol][icol]);
        a[icol][icol] = 1.0;
        for (int l = 1; l <= n; l++) a[icol][l] *= pivinv;
        b[icol] *= pivinv;
        for (int ll = 1; ll <= n; ll++)
            if (ll != icol) {
                FLT dum = a[ll][icol];
                a[ll][icol] = 0.0;
                for (int l = 1; l <= n; l++) a[ll][l] -= a[icol][l] * dum;
                b[ll] -= b[icol] * dum;
            }
    }
    (void)indxc;
    (void)indxr;
    return 1;
}

/* myGauss, speckleTrack.c:2421-2443: amplitude, mux, sigx, muy, sigy */
static void myGauss2D(FLT px, FLT py, const FLT a[6], FLT *y, FLT dyda[6])
{
    FLT dx = px - a[2], dy = py - a[4];
    FLT argx = (FLT)0.5 * (dx * dx) / (a[3] * a[3]);
    FLT argy = (FLT)0.5 * (dy * dy) / (a[5] * a[5]);
    FLT ex = (FLT)exp((double)(-argx - argy));
    *y = a[1] * ex;
    dyda[1] = ex;
    dyda[2] = (*y) * (px - a[2]) / (a[3] * a[3]);
    dyda[3] = *y * (px - a[2]) * (px - a[2]) / (a[3] * a[3] * a[3]);
    dyda[4] = *y * (py - a[4]) / (a[5] * a[5]);
    dyda[5] = *y * (py - a[4]) * (py - a[4]) / (a[5] * a[5] * a[5]);
}

static void mrqcof2D(const FLT *px, const FLT *py, const FLT *z, int n, const FLT a[6], FLT alpha[6][6], FLT beta[6],
                     FLT *chisq)
{
    /* mrqcofMod with ma = mfit = 5, sig = 1 */
    FLT ymod, dyda[6];
    for (int j = 1; j <= 5; j++) {
        for (int k = 1; k <= j; k++) alpha[j][k] = 0.0;
        beta[j] = 0.0;
    }
    *chisq = 0.0;
    for (int i = 1; i <= n; i++) {
        myGauss2D(px[i], py[i], a, &ymod, dyda);
        FLT dy = z[i] - ymod;
        for (int l = 1; l <= 5; l++) {
            FLT wt = dyda[l];
            for (int m = 1; m <= l; m++) alpha[l][m] += wt * dyda[m];
            beta[l] += dy * wt;
        }
        *chisq += dy * dy;
    }
    for (int j = 2; j <= 5; j++)
        for (int k = 1; k < j; k++) alpha[k][j] = alpha[j][k];
}

/* cmpTrackGauss, speckleTrack.c:2205-2303: 18 x 18 samples of |c| around the
 * coarse peak, scaled to correlation units, a 2-D Gaussian by <= 8 LM steps
 * (stop when both centres move < 0.001); peak in NOVER units of the 2x grid. */
static void cmpTrackGauss(StCtx *c, int *iMax, int *jMax, double *cMax, int wR, int wA, const FLT *cFunc, double p1,
                          double p2, int isComplex)
{
    const int nG = NGAUSS;
    if ((*iMax - nG / 2) < 0 || (*iMax + nG / 2) >= (wA * OS - 1) || (*jMax - nG / 2) < 0 ||
        (*jMax + nG / 2) >= (wR * OS - 1)) {
        *iMax = -LARGEINT;
        *jMax = -LARGEINT;
        *cMax = 0;
        return;
    }
    FLT px[NGAUSS * NGAUSS + 1], py[NGAUSS * NGAUSS + 1], z[NGAUSS * NGAUSS + 1];
    const double hc = (c->p->hanningFlag == TRUE && isComplex == TRUE) ? 1.5 : 1.0;
    const double scale = hc / (sqrt(p1 * p2) * pow((double)(wR * wA), 2));
    int iData = 1;
    for (int i = 0; i < nG; i++) {
        int i1 = *iMax - nG / 2 + i, j1 = *jMax - nG / 2;
        for (int j = 0; j < nG; j++) {
            px[iData] = (FLT)i1;
            py[iData] = (FLT)j1;
            z[iData] = (FLT)(cFunc[i1 * wR * OSA + j1] * scale);
            iData++;
            j1++;
        }
    }
    FLT a[6] = {0, (FLT)(*cMax * scale), (FLT)*iMax, 3, (FLT)*jMax, 3};
    FLT alpha[6][6], beta[6], chisq = 0, ochisq = 0, alamda = -1;
    FLT lasti = (FLT)2e9, lastj = (FLT)2e9;
    for (int it = 0; it < 8; it++) {
        FLT covar[6][6], da[6], atry[6];
        if (alamda < 0.0) {
            alamda = (FLT)0.001;
            mrqcof2D(px, py, z, iData - 1, a, alpha, beta, &chisq);
            ochisq = chisq;
        }
        for (int j = 1; j <= 5; j++) {
            for (int k = 1; k <= 5; k++) covar[j][k] = alpha[j][k];
            covar[j][j] = alpha[j][j] * (FLT)(1.0 + alamda);
            da[j] = beta[j];
        }
        if (!gaussj5(covar, 5, da)) break; /* Numerical Recipes would exit: the fit ends */
        for (int l = 1; l <= 5; l++) atry[l] = a[l] + da[l];
        atry[0] = a[0];
        mrqcof2D(px, py, z, iData - 1, atry, covar, da, &chisq);
        if (chisq < ochisq) {
            alamda *= (FLT)0.1;
            ochisq = chisq;
            for (int j = 1; j <= 5; j++) {
                for (int k = 1; k <= 5; k++) alpha[j][k] = covar[j][k];
                beta[j] = da[j];
            }
            for (int l = 1; l <= 5; l++) a[l] = atry[l];
        } else {
            alamda *= (FLT)10.0;
            chisq = ochisq;
        }
        if (fabs((double)(a[2] - lasti)) < 0.001 && fabs((double)(a[4] - lastj)) < 0.001) break;
        lasti = a[2];
        lastj = a[4];
    }
    *iMax = (int)round((double)(a[2] * NOVER)); /* float product, as the reference's float a[] */
    *jMax = (int)round((double)(a[4] * NOVER));
    *cMax = a[1] < 1.0 ? a[1] : 1.0;
    if ((0.5 * a[3]) > 1000.0 || (0.5 * a[5]) > 1000.0) {
        *iMax = -LARGEINT;
        *jMax = -LARGEINT;
        *cMax = 0;
    }
}

/* ---------------------------------------------------------------- peaks */

/* findCPeak, speckleTrack.c:744-805: fftshift |c| into corrF while taking the
 * first maximum in the reference's scan order; reject near-edge peaks. */
static void findCPeak(FLT *corrF, const ocplx *cnp, int wR, int wA, int *iMax, int *jMax, double *cMax)
{
    *cMax = 0.0;
    *iMax = 0; /* pinned: the reference leaves them unset when |c| == 0 everywhere */
    *jMax = 0;
    for (int i = 0; i < wA / 2; i++) {
        int i1 = wA / 2 + i;
        int j1 = wR / 2;
        for (int j = 0; j < wR / 2; j++) {
            FLT v;
            v = corrF[i * wR + j] = absCmpx(cnp[i1 * wR + j1], FALSE);
            if (v > *cMax) { *cMax = v; *iMax = i; *jMax = j; }
            v = corrF[i1 * wR + j1] = absCmpx(cnp[i * wR + j], FALSE);
            if (v > *cMax) { *cMax = v; *iMax = i1; *jMax = j1; }
            v = corrF[i1 * wR + j] = absCmpx(cnp[i * wR + j1], FALSE);
            if (v > *cMax) { *cMax = v; *iMax = i1; *jMax = j; }
            v = corrF[i * wR + j1] = absCmpx(cnp[i1 * wR + j], FALSE);
            if (v > *cMax) { *cMax = v; *iMax = i; *jMax = j1; }
            j1++;
        }
    }
    if (*iMax < (NFAST / 2) || *iMax > (wA - NFAST / 2) || *jMax < (NFAST / 2) || *jMax > (wR - NFAST / 2)) {
        *cMax = -1.0;
        *jMax = -1000;
        *iMax = -1000;
    }
}

/* overSampleC, speckleTrack.c:852-863: 8x8 DFT, zero pad to 96x96, inverse. */
static void overSampleC(StCtx *c)
{
    offt2d_exec(c->cForwardFast, c->cFast, c->psFast);
    zeroPadFFT(c->psFastOver, NFAST * NOVER, NFAST * NOVER, c->psFast, NFAST, NFAST, 0, 0);
    offt2d_exec(c->cReverseFast, c->psFastOver, c->cFastOver);
}

/* Loads the 8x8 |c| block around (iMax,jMax), oversamples it, and returns the
 * argmax over [24,72)^2 (cmpTrackFast :683-699 and ampTrackFast :565-581). */
static double overSamplePeak(StCtx *c, const FLT *mag, int ncol, int iMax, int jMax, int *iMax1o, int *jMax1o)
{
    for (int i = 0; i < NFAST; i++) {
        int i1 = iMax - NFAST / 2 + i;
        int j1 = jMax - NFAST / 2;
        for (int j = 0; j < NFAST; j++) {
            c->cFast[i * NFAST + j].re = (REAL)mag[i1 * ncol + j1];
            c->cFast[i * NFAST + j].im = 0.0;
            j1++;
        }
    }
    overSampleC(c);
    int iMax1 = 0, jMax1 = 0;
    double cMax = 0.0;
    const int n = NFAST * NOVER;
    for (int i = n / 2 - NOVER * 2; i < n / 2 + NOVER * 2; i++)
        for (int j = n / 2 - NOVER * 2; j < n / 2 + NOVER * 2; j++) {
            double corr = absCmpx(c->cFastOver[i * n + j], FALSE);
            if (corr > cMax) { cMax = corr; iMax1 = i; jMax1 = j; }
        }
    *iMax1o = iMax1;
    *jMax1o = jMax1;
    return cMax;
}

/* ---------------------------------------------------------------- complex */

static int getPatches(StCtx *c, int r1, int a1, int r2, int a2)
{
    /* speckleTrack.c:1194-1330 */
    const sb_track_params *p = c->p;
    const int wA = c->wA, wR = c->wR;
    const int floatFlag = (c->img1->sampleType == SB_CFLOAT32);
    float threshold = floatFlag ? 1e-15f : 1e-9f;
    float thresholdAll = threshold * wA * wR;
    double p1 = 0., p2 = 0.;
    int nZero = 0;
    for (int i = 0; i < wA; i++) {
        for (int j = 0; j < wR; j++) {
            ocplx *q1 = &c->patch1[i * wR + j], *q2 = &c->patch2[i * wR + j];
            REAL re, im;
            sample_at(c->img1, a1 + i, r1 + j, &re, &im);
            if (floatFlag) { q1->re = re * 1000; q1->im = im * 1000; } else { q1->re = re; q1->im = im; }
            sample_at(c->img2, a2 + i, r2 + j, &re, &im);
            if (floatFlag) { q2->re = re * 1000; q2->im = im * 1000; } else { q2->re = re; q2->im = im; }
            if (p->hanningFlag == TRUE) {
                q2->re *= c->hanning[i * wR + j];
                q2->im *= c->hanning[i * wR + j];
            }
            FLT power1 = absCmpx(*q1, TRUE);
            FLT power2 = absCmpx(*q2, TRUE);
            if (power1 < threshold || power2 < threshold) nZero++;
            if (nZero > 20) return FALSE;
            p1 += power1;
            p2 += power2;
        }
    }
    if (p1 < thresholdAll || p2 < thresholdAll) return FALSE;
    c->azShift = estDopCarrier1(c->wA, c->patch1, c->patch2, wA, wR);
    c->p1 = p1 / (double)(wA * wR);
    c->p2 = p2 / (double)(wA * wR);
    return TRUE;
}

static void phaseCorrectBaseline(StCtx *c, int r1, int a1)
{
    /* speckleTrack.c:868-907; an all-zero baseline leaves the patch unchanged */
    const sb_baseline *b = c->p->baseline;
    if (b == NULL) return;
    if (b->Bn == 0 && b->Bp == 0 && b->dBn == 0 && b->dBp == 0 && b->dBnQ == 0 && b->dBpQ == 0) return;
    const int nSlpA = c->img1->na;
    double x = (a1 - c->wA / 2 - (nSlpA / 2)) / (double)nSlpA;
    double deltaX = 1. / (double)nSlpA;
    double bn = b->Bn + x * b->dBn + x * x * b->dBnQ;
    double ptod = -(4.0 * ST_PI) / b->lambda;
    for (int i = 0; i < c->wA; i++) {
        double bp = b->Bp + x * b->dBp + x * x * b->dBpQ;
        double bsq = bn * bn + bp * bp;
        for (int j = 0; j < c->wR; j++) {
            int j1 = (r1 - c->wR / 2 > 0 ? r1 - c->wR / 2 : 0) + j;
            double bnPhase = -bn * b->sinThetaD[j1] - bp * b->cosThetaD[j1] + (0.5 * bsq * b->overRange[j1]);
            bnPhase *= ptod;
            double pr = cos(bnPhase), pi = sin(bnPhase);
            double cr = c->patch1[i * c->wR + j].re, ci = c->patch1[i * c->wR + j].im;
            c->patch1[i * c->wR + j].re = (REAL)(cr * pr - ci * pi);
            c->patch1[i * c->wR + j].im = (REAL)(cr * pi + ci * pr);
        }
        x += deltaX;
    }
}

/* Interferogram sample (getInt, Strack/getInt.c:66-73: int16 pairs read with
 * byte swapping when the file is big-endian, converted to float). */
static void int_sample(const sb_interferogram *f, int row, int col, REAL *re, REAL *im)
{
    const unsigned char *b = (const unsigned char *)f->data + ((size_t)row * f->nr + col) * 4;
    int16_t r, i;
    if (f->byteOrder == SB_MSB) {
        r = (int16_t)((b[0] << 8) | b[1]);
        i = (int16_t)((b[2] << 8) | b[3]);
    } else {
        r = (int16_t)((b[1] << 8) | b[0]);
        i = (int16_t)((b[3] << 8) | b[2]);
    }
    *re = (REAL)(float)r;
    *im = (REAL)(float)i;
}

static void phaseCorrectInt(StCtx *c, int r1, int a1)
{
    /* speckleTrack.c:909-1000, osF = 1 */
    const sb_interferogram *f = c->p->intf;
    if (f == NULL || c->intPs == 0) return;
    const int ps = c->intPs, pSA = c->intPSA, pSR = c->intPSR;
    const int ia1 = (a1 + c->wA / 2) / f->nal - ps / 2;
    const int ir1 = (r1 + c->wR / 2) / f->nrl - ps / 2;
    if (!inBounds(ir1, ia1, ps, ps, f->nr, f->na)) return;
    for (int i = 0; i < ps; i++)
        for (int j = 0; j < ps; j++)
            int_sample(f, ia1 + i, ir1 + j, &c->intPatch[i * ps + j].re, &c->intPatch[i * ps + j].im);
    offt2d_exec(c->intForward, c->intPatch, c->fftIntPatch);
    double maxf = 0.;
    for (int k = 0; k < ps * ps; k++) {
        const double p = (double)c->fftIntPatch[k].re * c->fftIntPatch[k].re +
                         (double)c->fftIntPatch[k].im * c->fftIntPatch[k].im;
        maxf = maxf > p ? maxf : p;
    }
    /* The reference's loop body has no braces: the real part is cleared
       below 0.99 of the peak power, the imaginary part of every bin is cleared. */
    for (int k = 0; k < ps * ps; k++) {
        const double p = (double)c->fftIntPatch[k].re * c->fftIntPatch[k].re +
                         (double)c->fftIntPatch[k].im * c->fftIntPatch[k].im;
        if (p < 0.99 * maxf) c->fftIntPatch[k].re = 0.0;
        c->fftIntPatch[k].im = 0.0;
    }
    zeroPadFFT(c->fftIntPatchOver, pSA, pSR, c->fftIntPatch, ps, ps, 0, 0);
    offt2d_exec(c->intBackward, c->fftIntPatchOver, c->intPatchOver);
    int i1 = pSA / 2 - c->wA / 2;
    for (int i = 0; i < c->wA; i++) {
        int j1 = pSR / 2 - c->wR / 2;
        for (int j = 0; j < c->wR; j++) {
            double pr = c->intPatchOver[(size_t)i1 * pSR + j1].re;
            double pi = -c->intPatchOver[(size_t)i1 * pSR + j1].im;
            double scale;
            if (fabs(pr) < 1.0e-6 && fabs(pi) < 1.0e-6) {
                pr = 1.0;
                pi = 0.0;
                scale = 1.0;
            } else
                scale = 1.0 / sqrt(pr * pr + pi * pi);
            ocplx *q = &c->patch1[i * c->wR + j];
            const double cr = q->re, ci = q->im;
            q->re = (REAL)((cr * pr - ci * pi) * scale);
            q->im = (REAL)((cr * pi + ci * pr) * scale);
            j1++;
        }
        i1++;
    }
}

static void cmpPSWithPad(StCtx *c)
{
    /* speckleTrack.c:604-643 */
    const int wA = c->wA, wR = c->wR, W2 = wR * OSA;
    offt2d_exec(c->cForwardIn, c->patch1, c->fftF1os);
    offt2d_exec(c->cForwardIn, c->patch2, c->fftF2os);
    memset(c->psNoPad, 0, sizeof(ocplx) * (size_t)(wA * OSA) * W2);
    const ocplx *F1 = c->fftF1os, *F2 = c->fftF2os;
    ocplx *ps = c->psNoPad;
#define XS(dst, src)                                                                  \
    do {                                                                              \
        ps[dst].re = F1[src].re * F2[src].re + F1[src].im * F2[src].im;               \
        ps[dst].im = F1[src].im * F2[src].re - F1[src].re * F2[src].im;               \
    } while (0)
    for (int i = 0; i < wA / 2; i++) {
        int i1 = OSA * wA - wA / OSA + i;
        int i2 = (wA / OSA + i + c->azShift) % wA;
        int ia = (i + c->azShift) % wA;
        int j1 = wR * OSA - wR / OSA;
        int j2 = wR / OSA + c->rangeShift;
        for (int j = 0; j < wR / 2; j++) {
            int ja = (j + c->rangeShift) % wR;
            int j2a = j2 % wR;
            XS(i * W2 + j, ia * wR + ja);
            XS(i1 * W2 + j, i2 * wR + ja);
            XS(i1 * W2 + j1, i2 * wR + j2a);
            XS(i * W2 + j1, ia * wR + j2a);
            j1++;
            j2++;
        }
    }
#undef XS
}

static void cmpTrackFast(StCtx *c, int *iMax, int *jMax, double *cMax)
{
    /* speckleTrack.c:648-709 */
    double hanningCorrection = (c->p->hanningFlag == TRUE) ? 1.5 : 1.0;
    int wA2 = c->wA * OSA, wR2 = c->wR * OSA;
    offt2d_exec(c->cReverseNoPad, c->psNoPad, c->cNoPad);
    *cMax = 0.;
    findCPeak(c->cNoPadMag, c->cNoPad, wR2, wA2, iMax, jMax, cMax);
    if (*iMax < -999) return;
    int iMax1, jMax1;
    *cMax = overSamplePeak(c, c->cNoPadMag, wR2, *iMax, *jMax, &iMax1, &jMax1);
    *cMax = *cMax / (NFAST * NFAST);
    *cMax = hanningCorrection * (*cMax) / (sqrt(c->p1 * c->p2) * pow(c->wR * c->wA, 2));
    *iMax = (*iMax * NOVER) + iMax1 - (NOVER * NFAST) / 2;
    *jMax = (*jMax * NOVER) + jMax1 - (NOVER * NFAST) / 2;
}

static void finalizeCmpxMatch(StCtx *c, double cMax, int iMax, int jMax, double wRover2exp, double wAover2exp,
                              double invNOVER, int *good, int *type, float *rShift1, float *aShift1)
{
    /* speckleTrack.c:714-739 */
    *good = FALSE;
    if (cMax > .185 && c->p->noComplex == FALSE) {
        *rShift1 = (float)(((float)jMax - wRover2exp) * invNOVER / OS);
        *aShift1 = (float)(((float)iMax - wAover2exp) * invNOVER / OS);
        if (fabs((double)*rShift1) < 0.125 * c->wR * OS && fabs((double)*aShift1) < 0.125 * c->wA * OS) {
            *good = TRUE;
            c->nComplex++;
            *type = SB_CMATCH;
        }
    }
}

static int complexMatch(StCtx *c, int r1, int a1, int *iMax, int *jMax, double *cMax, float *rShift1,
                        float *aShift1, size_t outIdx)
{
    /* speckleTrack.c:349-394 */
    FLT sigmaRg, sigmaAz, peakRatioRg, peakRatioAz;
    int good, type;
    double invNOVER = 1.0 / (float)NOVER;
    double wRover2exp = c->wR / 2. * NOVER * OSA;
    double wAover2exp = c->wA / 2. * NOVER * OSA;
    phaseCorrectBaseline(c, r1, a1);
    phaseCorrectInt(c, r1, a1);
    cmpPSWithPad(c);
    if (c->p->gaussFlag == TRUE) {
        /* speckleTrack.c:366-371 */
        offt2d_exec(c->cReverseNoPad, c->psNoPad, c->cNoPad);
        findCPeak(c->cNoPadMag, c->cNoPad, c->wR * OS, c->wA * OS, iMax, jMax, cMax);
        cmpTrackGauss(c, iMax, jMax, cMax, c->wR, c->wA, c->cNoPadMag, c->p1, c->p2, TRUE);
    } else
        cmpTrackFast(c, iMax, jMax, cMax);
    good = FALSE;
    int iM = *iMax / NOVER; /* lround of an integer quotient */
    int jM = *jMax / NOVER;
    c->aZDefocus[outIdx] = (float)-LARGEINT;
    if ((iM - NGAUSS / 2) >= 0 && (iM + NGAUSS / 2) < (c->wA * OS) && (jM - NGAUSS / 2) >= 0 &&
        (jM + NGAUSS / 2) < (c->wR * OS)) {
        gaussPeak1D(c->cNoPadMag, c->wR * OSA, iM, jM, RG, &sigmaRg, &peakRatioRg);
        gaussPeak1D(c->cNoPadMag, c->wR * OSA, iM, jM, AZ, &sigmaAz, &peakRatioAz);
        c->aZDefocus[outIdx] = (float)(sigmaAz / sigmaRg);
        if (fabs(c->aZDefocus[outIdx]) < c->p->azDefocusThresh || c->p->checkAzFocus == FALSE) {
            finalizeCmpxMatch(c, *cMax, *iMax, *jMax, wRover2exp, wAover2exp, invNOVER, &good, &type, rShift1,
                              aShift1);
        }
    }
    return good;
}

/* ---------------------------------------------------------------- amplitude */

static int getAmpPatches(StCtx *c, int r1, int a1, int r2, int a2, int large)
{
    /* speckleTrack.c:1006-1189 */
    AmpBufs *b = &c->amp[large ? 1 : 0];
    const int floatFlag = (c->img1->sampleType == SB_CFLOAT32);
    float threshold = floatFlag ? 1.0e-15f : 1.0e-6f;
    const size_t wAa = (size_t)b->wa, wRa = (size_t)b->wr;
    float scale = (float)(1. / (wRa * wAa * wRa * wAa * OS * OS * OS));
    int nZero = 0;
    for (size_t i = 0; i < wAa; i++)
        for (size_t j = 0; j < wRa; j++) {
            sample_at(c->img1, a1 + (int)i, r1 + (int)j, &b->in1[i * wRa + j].re, &b->in1[i * wRa + j].im);
            sample_at(c->img2, a2 + (int)i, r2 + (int)j, &b->in2[i * wRa + j].re, &b->in2[i * wRa + j].im);
        }
    offt2d_exec(b->fwdIn, b->in1, b->f1);
    offt2d_exec(b->fwdIn, b->in2, b->f2);
    if (c->p->noComplex == TRUE && large == FALSE)
        c->azShift = estDopCarrier1(c->wA, b->in1, b->in2, c->wAa, c->wRa);
    int azShift = (int)((float)c->azShift * (float)wAa / (float)c->wA);
    zeroPadFFT(b->f1a, (int)wAa * OS, (int)wRa * OS, b->f1, (int)wAa, (int)wRa, azShift, 0);
    zeroPadFFT(b->f2a, (int)wAa * OS, (int)wRa * OS, b->f2, (int)wAa, (int)wRa, azShift, 0);
    offt2d_exec(b->revPad, b->f1a, b->im1);
    offt2d_exec(b->revPad, b->f2a, b->im2);
    double i1Sum = 0.0, i2Sum = 0.0;
    const size_t n2 = wAa * OS * wRa * OS;
    for (size_t k = 0; k < n2; k++) {
        b->im1[k].re = (REAL)(absCmpx(b->im1[k], TRUE) * scale);
        b->im1[k].im = 0.0;
        b->im2[k].re = (REAL)(absCmpx(b->im2[k], TRUE) * scale);
        b->im2[k].im = 0.0;
        if (b->im1[k].re < threshold || b->im2[k].re < threshold) nZero++;
        i1Sum += b->im1[k].re;
        i2Sum += b->im2[k].re;
    }
    if (nZero > 20) return FALSE;
    if (i1Sum < 1.0e-6 || i2Sum < 1.0e-6) return FALSE;
    return TRUE;
}

static void ampTrackFast(StCtx *c, int *iMax, int *jMax, double *cMax, double p1, double p2, int large,
                         size_t outIdx)
{
    /* speckleTrack.c:489-597 */
    AmpBufs *b = &c->amp[large ? 1 : 0];
    const int wA = b->wa, wR = b->wr;
    FLT sigmaAz, sigmaRg, peakRatioAz, peakRatioRg;
    offt2d_exec(b->rev, b->ps, b->ca);
    findCPeak(b->caMag, b->ca, wR * OSA, wA * OSA, iMax, jMax, cMax);
    if (*iMax > NGAUSS / 2 && *iMax < (wA * OSA - NGAUSS / 2) && *jMax > NGAUSS / 2 &&
        *jMax < (wR * OSA - NGAUSS / 2)) {
        gaussPeak1D(b->caMag, wR * OSA, *iMax, *jMax, RG, &sigmaRg, &peakRatioRg);
        gaussPeak1D(b->caMag, wR * OSA, *iMax, *jMax, AZ, &sigmaAz, &peakRatioAz);
        c->aZDefocus[outIdx] = (float)(sigmaAz / sigmaRg);
    }
    if (*iMax < -999 || (fabs(c->aZDefocus[outIdx]) >= c->p->azDefocusThresh && c->p->checkAzFocus == TRUE))
        return;
    if (c->p->gaussFlag == TRUE) {
        /* speckleTrack.c:551-557: pScale 16 matches the complex normalisation */
        cmpTrackGauss(c, iMax, jMax, cMax, wR, wA, b->caMag, p1 * 16., p2 * 16., FALSE);
        return;
    }
    int iMax1, jMax1;
    *cMax = overSamplePeak(c, b->caMag, wR * OSA, *iMax, *jMax, &iMax1, &jMax1);
    *cMax = *cMax / (pow((double)(wA * OS), 2) * pow((double)(wR * OS), 2) * pow((double)NFAST, 2));
    *cMax = *cMax / sqrt(p1 * p2);
    *iMax = (*iMax * NOVER) + iMax1 - (NOVER * NFAST) / 2;
    *jMax = (*jMax * NOVER) + jMax1 - (NOVER * NFAST) / 2;
}

static void ampMatch(StCtx *c, int *iMax, int *jMax, double *cMax, int large, size_t outIdx)
{
    /* speckleTrack.c:398-484 */
    AmpBufs *b = &c->amp[large ? 1 : 0];
    const int n = b->wa * OS * b->wr * OS;
    double avgAmp1 = 0.0, avgAmp2 = 0.0, p1 = 0.0, p2 = 0.0;
    for (int k = 0; k < n; k++) {
        b->im1[k].re = (REAL)sqrt((double)b->im1[k].re);
        b->im2[k].re = (REAL)sqrt((double)b->im2[k].re);
        avgAmp1 += b->im1[k].re;
        avgAmp2 += b->im2[k].re;
    }
    avgAmp1 = avgAmp1 / (double)n;
    avgAmp2 = avgAmp2 / (double)n;
    for (int k = 0; k < n; k++) {
        if (b->im1[k].re > 1.0e-20) b->im1[k].re = (REAL)(b->im1[k].re - avgAmp1);
        b->im2[k].re = (REAL)(b->im2[k].re - avgAmp2);
        p1 += b->im1[k].re * b->im1[k].re;
        p2 += b->im2[k].re * b->im2[k].re;
    }
    p1 = p1 / (double)n;
    p2 = p2 / (double)n;
    offt2d_exec(b->fwd, b->im1, b->fa1);
    offt2d_exec(b->fwd, b->im2, b->fa2);
    for (int k = 0; k < n; k++) {
        b->ps[k].re = b->fa1[k].re * b->fa2[k].re + b->fa1[k].im * b->fa2[k].im;
        b->ps[k].im = b->fa1[k].im * b->fa2[k].re - b->fa1[k].re * b->fa2[k].im;
    }
    ampTrackFast(c, iMax, jMax, cMax, p1, p2, large, outIdx);
}

/* ---------------------------------------------------------------- setup */

static void ampAlloc(AmpBufs *b, int wr, int wa)
{
    size_t n = (size_t)wr * wa, n4 = n * OS * OS;
    b->wr = wr;
    b->wa = wa;
    b->in1 = cbuf(n); b->in2 = cbuf(n); b->f1 = cbuf(n); b->f2 = cbuf(n);
    b->f1a = cbuf(n4); b->f2a = cbuf(n4); b->im1 = cbuf(n4); b->im2 = cbuf(n4);
    b->fa1 = cbuf(n4); b->fa2 = cbuf(n4); b->ps = cbuf(n4); b->ca = cbuf(n4);
    b->caMag = (FLT *)calloc(n4, sizeof(FLT));
    b->fwdIn = offt2d_plan(wa, wr, OFFT_FORWARD);
    b->revPad = offt2d_plan(wa * OS, wr * OS, OFFT_BACKWARD);
    b->fwd = offt2d_plan(wa * OS, wr * OS, OFFT_FORWARD);
    b->rev = offt2d_plan(wa * OS, wr * OS, OFFT_BACKWARD);
}

static void ampFree(AmpBufs *b)
{
    free(b->in1); free(b->in2); free(b->f1); free(b->f2); free(b->f1a); free(b->f2a);
    free(b->im1); free(b->im2); free(b->fa1); free(b->fa2); free(b->ps); free(b->ca); free(b->caMag);
    offt2d_destroy(b->fwdIn); offt2d_destroy(b->revPad); offt2d_destroy(b->fwd); offt2d_destroy(b->rev);
}

int oracle_real_size(void) { return (int)sizeof(REAL); }

int oracle_strack(const sb_track_params *p, const sb_image *img1, const sb_image *img2, sb_track_result *out,
                  int32_t row0, int32_t row1)
{
    if (!p || !img1 || !img2 || !out) return SB_ERR_ARG;
    if (p->hanningFlag && p->wR != p->wA) return SB_ERR_UNSUPPORTED;
    if (p->polyShift == 0 && p->initOffsets == NULL) return SB_ERR_ARG;
    if (p->intf && (p->intf->nal <= 0 || p->intf->nrl <= 0 || p->intf->nr <= 0 || p->intf->na <= 0 ||
                    !p->intf->data || p->intf->onDevice))
        return SB_ERR_ARG;
    StCtx C, *c = &C;
    memset(c, 0, sizeof(C));
    c->p = p;
    c->img1 = img1;
    c->img2 = img2;
    c->wR = p->wR; c->wA = p->wA; c->wRa = p->wRa; c->wAa = p->wAa;
    c->rangeShift = 0;
    const int wR = p->wR, wA = p->wA;
    c->hanning = (FLT *)calloc((size_t)wR * wA, sizeof(FLT));
    c->patch1 = cbuf((size_t)wR * wA); c->patch2 = cbuf((size_t)wR * wA);
    c->fftF1os = cbuf((size_t)wR * wA); c->fftF2os = cbuf((size_t)wR * wA);
    c->psNoPad = cbuf((size_t)wR * wA * 4); c->cNoPad = cbuf((size_t)wR * wA * 4);
    c->cNoPadMag = (FLT *)calloc((size_t)wR * wA * 4, sizeof(FLT));
    c->cForwardIn = offt2d_plan(wA, wR, OFFT_FORWARD);
    c->cReverseNoPad = offt2d_plan(wA * OSA, wR * OSA, OFFT_BACKWARD);
    c->cForwardFast = offt2d_plan(NFAST, NFAST, OFFT_FORWARD);
    c->cReverseFast = offt2d_plan(NFAST * NOVER, NFAST * NOVER, OFFT_BACKWARD);
    c->cFast = cbuf(NFAST * NFAST); c->psFast = cbuf(NFAST * NFAST);
    c->psFastOver = cbuf(NFAST * NOVER * NFAST * NOVER); c->cFastOver = cbuf(NFAST * NOVER * NFAST * NOVER);
    ampAlloc(&c->amp[0], p->wRa, p->wAa);
    ampAlloc(&c->amp[1], p->wRa * LA, p->wAa * LA);
    if (p->hanningFlag == TRUE && p->noComplex == FALSE) computeHanning(c);
    if (p->intf != NULL && p->noComplex == FALSE) {
        /* initPhaseCorrect: patch of max(wA/nal, wR/nrl, INTPATCHSIZE = 8) samples */
        const sb_interferogram *f = p->intf;
        int ps = wA / f->nal > wR / f->nrl ? wA / f->nal : wR / f->nrl;
        ps = ps > 8 ? ps : 8;
        /* a padded patch smaller than the window makes the reference read
           outside it (speckleTrack.c:978-983): refused */
        if (ps * f->nal < wA || ps * f->nrl < wR) {
            free(c->hanning); /* the rest is released by the process; test infrastructure */
            return SB_ERR_UNSUPPORTED;
        }
        c->intPs = ps;
        c->intPSA = ps * f->nal;
        c->intPSR = ps * f->nrl;
        c->intPatch = cbuf((size_t)ps * ps); c->fftIntPatch = cbuf((size_t)ps * ps);
        c->fftIntPatchOver = cbuf((size_t)c->intPSA * c->intPSR);
        c->intPatchOver = cbuf((size_t)c->intPSA * c->intPSR);
        c->intForward = offt2d_plan(ps, ps, OFFT_FORWARD);
        c->intBackward = offt2d_plan(c->intPSA, c->intPSR, OFFT_BACKWARD);
    }

    const int nR = p->nR, nA = p->nA;
    if (row1 <= 0 || row1 > nA) row1 = nA;
    if (row0 < 0) row0 = 0;
    c->aZDefocus = out->azd;
    for (int i = row0; i < row1; i++)
        for (int j = 0; j < nR; j++) {
            size_t k = (size_t)i * nR + j;
            out->offR[k] = (float)(-LARGEINT);
            out->offA[k] = (float)(-LARGEINT);
            out->corr[k] = 0;
            out->type[k] = SB_BAD;
            if (out->azd) out->azd[k] = 0.0f;
        }
    float *azdScratch = NULL;
    if (!out->azd) {
        azdScratch = (float *)calloc((size_t)nR * nA, sizeof(float));
        c->aZDefocus = azdScratch;
    }
    int64_t nTot = 0;
    double invNOVER = 1.0 / (float)NOVER;
    int r2 = 0, a2 = 0; /* pinned initial values */
    int iMax = 0, jMax = 0;
    float rShift1 = 0, aShift1 = 0;
    c->azShift = 0;
    for (int i = row0; i < row1; i++) {
        int a1 = p->aStart + i * p->deltaA - p->wA / 2;
        int nSkip = 0;
        for (int j = 0; j < nR; j++) {
            size_t k = (size_t)i * nR + j;
            int haveData = TRUE, type = SB_BAD, good, maskVal, nTries, large, ampWScale, ampType;
            double cMax = 0., cThresh;
            int r1 = p->rStart + j * p->deltaR - p->wR / 2;
            findImage2Pos(c, r1, a1, &r2, &a2);
            float rShiftAmp = (float)(r2 - r1), aShiftAmp = (float)(a2 - a1);
            maskVal = maskValue(c, r1 * p->scaleFactor, a1 * p->scaleFactor);
            maskVal = maskVal < 1 ? maskVal : 1;
            good = FALSE;
            if (boundsCheck(c, r1, a1, r2, a2, p->wR, p->wA) && maskVal > 0 && p->noComplex == FALSE) {
                haveData = getPatches(c, r1, a1, r2, a2);
                good = FALSE;
                if (haveData == TRUE) {
                    good = complexMatch(c, r1, a1, &iMax, &jMax, &cMax, &rShift1, &aShift1, k);
                    if (good == TRUE) type = SB_CMATCH;
                } else
                    nSkip++;
            }
            nTries = 0;
            while (good == FALSE && haveData == TRUE && maskVal > 0 && nTries < p->maxTries) {
                int64_t *nAmp;
                if (nTries == 0) {
                    large = FALSE; ampWScale = 1; ampType = SB_AMPMATCH; nAmp = &c->nAmp; cThresh = 0.07;
                } else {
                    large = TRUE; ampWScale = LA; ampType = SB_AMPMATCHLARGE; nAmp = &c->nAmpL; cThresh = 0.028;
                }
                int a1a = p->aStart + i * p->deltaA - p->wA / 2 * ampWScale;
                int r1a = p->rStart + j * p->deltaR - p->wR / 2 * ampWScale;
                int r2a = r1a + (int)rShiftAmp, a2a = a1a + (int)aShiftAmp;
                if (boundsCheck(c, r1a, a1a, r2a, a2a, p->wRa * ampWScale, p->wAa * ampWScale) && maskVal > 0) {
                    haveData = getAmpPatches(c, r1a, a1a, r2a, a2a, large);
                    if (haveData == TRUE) {
                        ampMatch(c, &iMax, &jMax, &cMax, large, k);
                        rShift1 = (float)(((float)jMax - p->wRa * 0.5 * OS * NOVER * ampWScale) * invNOVER / OS);
                        aShift1 = (float)(((float)iMax - p->wAa * 0.5 * OS * NOVER * ampWScale) * invNOVER / OS);
                    } else {
                        cMax = 0.0;
                        nSkip++;
                    }
                } else
                    cMax = 0.0;
                if (fabs((double)rShift1) < 0.15 * p->wRa * OS * ampWScale &&
                    fabs((double)aShift1) < 0.15 * p->wAa * OS * ampWScale && cMax > cThresh) {
                    good = TRUE;
                    (*nAmp)++;
                    type = ampType;
                }
                nTries++;
            }
            float rShift, aShift;
            if (good == TRUE && maskVal > 0) {
                rShift = rShiftAmp - rShift1;
                aShift = aShiftAmp - aShift1;
            } else {
                rShift = (float)-LARGEINT;
                aShift = (float)-LARGEINT;
                if (haveData == TRUE) c->nFail++;
            }
            out->offR[k] = rShift;
            out->offA[k] = aShift;
            if (rShift > -100000) {
                out->offR[k] *= (float)p->scaleFactor;
                out->offA[k] *= (float)p->scaleFactor;
            }
            out->corr[k] = (float)cMax;
            out->type[k] = (uint8_t)type;
        }
        nTot += (nR - nSkip);
    }
    out->nComplex = c->nComplex;
    out->nAmp = c->nAmp;
    out->nAmpL = c->nAmpL;
    out->nFail = c->nFail;
    out->nAttempted = nTot;

    free(azdScratch);
    free(c->hanning); free(c->patch1); free(c->patch2); free(c->fftF1os); free(c->fftF2os);
    free(c->psNoPad); free(c->cNoPad); free(c->cNoPadMag);
    offt2d_destroy(c->cForwardIn); offt2d_destroy(c->cReverseNoPad);
    offt2d_destroy(c->cForwardFast); offt2d_destroy(c->cReverseFast);
    free(c->cFast); free(c->psFast); free(c->psFastOver); free(c->cFastOver);
    ampFree(&c->amp[0]);
    ampFree(&c->amp[1]);
    if (c->intPs) {
        free(c->intPatch); free(c->fftIntPatch); free(c->fftIntPatchOver); free(c->intPatchOver);
        offt2d_destroy(c->intForward); offt2d_destroy(c->intBackward);
    }
    return SB_OK;
}

int oracle_est_dop_carrier(const float *p1, const float *p2, int32_t nAz, int32_t nRg, int32_t wA)
{
    size_t n = (size_t)nAz * nRg;
    ocplx *a = cbuf(n), *b = cbuf(n);
    for (size_t k = 0; k < n; k++) {
        a[k].re = p1[2 * k]; a[k].im = p1[2 * k + 1];
        b[k].re = p2[2 * k]; b[k].im = p2[2 * k + 1];
    }
    int s = estDopCarrier1(wA, a, b, nAz, nRg);
    free(a);
    free(b);
    return s;
}

/* Seconds per forward 2-D transform of na x nr in this build's precision:
 * the plan is made once, then reps executions are timed (one thread).  Used
 * to compare the CPU baseline's FFT with another FFT library's. */
int oracle_fft2d_time(int32_t na, int32_t nr, int32_t reps, double *secs)
{
    size_t n = (size_t)na * nr;
    ocplx *a = cbuf(n), *o = cbuf(n);
    for (size_t k = 0; k < n; k++) {
        a[k].re = (REAL)((double)((k * 7919u) % 1000u) / 1000.0 - 0.5);
        a[k].im = (REAL)((double)((k * 104729u) % 1000u) / 1000.0 - 0.5);
    }
    offt2d *pl = offt2d_plan(na, nr, OFFT_FORWARD);
    offt2d_exec(pl, a, o);
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (int32_t r = 0; r < reps; r++) offt2d_exec(pl, a, o);
    clock_gettime(CLOCK_MONOTONIC, &t1);
    *secs = ((double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec)) / (reps > 0 ? reps : 1);
    offt2d_destroy(pl);
    free(a);
    free(o);
    return SB_OK;
}

int oracle_fft2d(double *data, int32_t na, int32_t nr, int32_t sign)
{
    size_t n = (size_t)na * nr;
    ocplx *a = cbuf(n), *o = cbuf(n);
    for (size_t k = 0; k < n; k++) { a[k].re = (REAL)data[2 * k]; a[k].im = (REAL)data[2 * k + 1]; }
    offt2d *pl = offt2d_plan(na, nr, sign < 0 ? OFFT_FORWARD : OFFT_BACKWARD);
    offt2d_exec(pl, a, o);
    offt2d_destroy(pl);
    for (size_t k = 0; k < n; k++) { data[2 * k] = o[k].re; data[2 * k + 1] = o[k].im; }
    free(a);
    free(o);
    return SB_OK;
}
