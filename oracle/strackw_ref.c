/*
 * strackw_ref.c -- TEST INFRASTRUCTURE ONLY (CPU oracle, pinned to the reference build by tests/test_ref_pin.py).
 *
 * Restatement of corrTrackFast() and its helpers, Strackw/corrTrackFast.c.
 * REAL = the reference's fftw_real, FLT = its `float` working variables
 * (double in the f64 build).  Like the reference, patches whose far edge lies
 * outside the image are not rejected (only the near corner is checked,
 * :170-171); the reference then reads stale buffer rows, which this oracle
 * cannot reproduce, so callers keep such windows inside the image.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "fft_ref.h"
#include "oracle.h"

#ifndef FLT
#define FLT REAL
#endif

#define NOVER 16
#define NFAST 20
#define OS 2
#define ST_PI 3.14159265358979323846
#define LARGEINT 2000000000
#define TRUE 1
#define FALSE 0

static inline uint32_t bswap32w(uint32_t v)
{
    return (v >> 24) | ((v >> 8) & 0xff00u) | ((v << 8) & 0xff0000u) | (v << 24);
}

static inline void sample_w(const sb_image *im, int row, int col, REAL *re, REAL *imv)
{
    size_t k = (size_t)row * (size_t)im->nr + (size_t)col;
    if (im->sampleType == SB_CFLOAT32) {
        const uint32_t *w = (const uint32_t *)im->data + 2 * k;
        uint32_t a = w[0], b = w[1];
        float fa, fb;
        if (im->byteOrder == SB_MSB) { a = bswap32w(a); b = bswap32w(b); }
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

typedef struct {
    const sb_track_params *p;
    const sb_image *src1, *src2;
    int wRa, wAa, eR, eA; /* eR/eA include the internal +NFAST/4 */
    int wR2, wA2;         /* chip size (oversampled) */
    int azShift;
    ocplx *in1, *in2, *f1, *f2, *f1a, *f2a, *img1, *img2, *fa1, *fa2, *ps, *ca;
    FLT *caMag;
    FLT *dataS, *dataR;
    double *tmpS1, *tmpS2, *meanS, *sigmaS, *corrResult;
    ocplx *cFast, *psFast, *psFastOver, *cFastOver;
    offt2d *aForwardIn, *aForward, *aReverseNoPad, *cForwardFast, *cReverseFast;
} SwCtx;

static ocplx *wbuf(size_t n) { return (ocplx *)calloc(n, sizeof(ocplx)); }

static int iroundw(double x) { return (x >= 0.0) ? (int)(x + 0.5) : (int)(x - 0.5); }

static double singleDop(const ocplx *image, int nAz, int nRg)
{
    /* dopplerEstimation.c:42-88 */
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
            double a_re = (long double)p1->re - mean_re, a_im = (long double)p1->im - mean_im;
            double b_re = (long double)p0->re - mean_re, b_im = (long double)p0->im - mean_im;
            sum_re += a_re * b_re + a_im * b_im;
            sum_im += a_im * b_re - a_re * b_im;
        }
    if (sum_re == 0.0 && sum_im == 0.0) return NAN;
    return atan2(sum_im, sum_re);
}

static int dopShift(int wA, const ocplx *im1, const ocplx *im2, int nAz, int nRg)
{
    double v = (double)(nAz / 2) * (singleDop(im1, nAz, nRg) + singleDop(im2, nAz, nRg)) * .5 / ST_PI;
    int shift = (v != v) ? 0 : iroundw(v);
    if (shift < 0) shift += nAz;
    return (int)((float)shift * (float)wA / (float)nAz);
}

static int maskValueW(SwCtx *c, int r1, int a1)
{
    /* corrTrackFast.c:1135-1154 */
    const sb_mask *m = c->p->mask;
    if (m == NULL) return 1;
    int dr = (c->wRa / 2 - m->r0) * c->p->scaleFactor;
    int da = (c->wAa / 2 - m->a0) * c->p->scaleFactor;
    int ia1 = (a1 + da) / m->nal;
    int ir1 = (r1 + dr) / m->nrl;
    if (ia1 < 0 || ia1 >= m->na || ir1 < 0 || ir1 >= m->nr) return 0;
    return (int)(signed char)m->mask[(size_t)ia1 * m->nr + ir1];
}

/* Bilinear interpolation with sentinel handling, standing in for
 * mosaicSource's bilinearInterp (absent from the reference tree), as called by
 * getShifts (corrTrackFast.c:843-858): any corner at or below minvalue, or a
 * position outside the grid, yields noData. */
static float bilinearW(const float *img, double x, double y, int nx, int ny, float minvalue, float noData)
{
    if (x < 0 || y < 0 || x > (double)(nx - 1) || y > (double)(ny - 1)) return noData;
    int j = (int)x, i = (int)y;
    if (j >= nx - 1) j = nx - 2 < 0 ? 0 : nx - 2;
    if (i >= ny - 1) i = ny - 2 < 0 ? 0 : ny - 2;
    if (nx < 2 || ny < 2) return noData;
    double t = x - j, u = y - i;
    float p1 = img[(size_t)i * nx + j], p2 = img[(size_t)i * nx + j + 1];
    float p3 = img[(size_t)(i + 1) * nx + j + 1], p4 = img[(size_t)(i + 1) * nx + j];
    if (p1 <= minvalue || p2 <= minvalue || p3 <= minvalue || p4 <= minvalue) return noData;
    return (float)((1.0 - t) * (1.0 - u) * p1 + t * (1.0 - u) * p2 + t * u * p3 + (1.0 - t) * u * p4);
}

static void findImage2PosW(SwCtx *c, int r1, int a1, int *r2, int *a2)
{
    /* corrTrackFast.c:257-292 */
    const sb_track_params *p = c->p;
    double aShift, rShift, sc = (double)p->scaleFactor;
    if (p->polyShift == TRUE) {
        rShift = p->rShiftPoly[0] + (double)(r1 * sc) * p->rShiftPoly[1] + (double)(a1 * sc) * p->rShiftPoly[2];
        aShift = p->aShiftPoly[0] + (double)(r1 * sc) * p->aShiftPoly[1] + (double)(a1 * sc) * p->aShiftPoly[2];
    } else {
        const sb_offset_grid *o = p->initOffsets;
        float minvalue = (float)((float)-LARGEINT * 0.9);
        double range = (r1 - o->r0) / o->deltaR, azimuth = (a1 - o->a0) / o->deltaA;
        rShift = bilinearW(o->dr, range, azimuth, o->nr, o->na, minvalue, (float)-LARGEINT);
        aShift = bilinearW(o->da, range, azimuth, o->nr, o->na, minvalue, (float)-LARGEINT);
        if (rShift <= minvalue || aShift <= minvalue) { rShift = minvalue; aShift = minvalue; }
        if (rShift < (-LARGEINT + 1)) {
            rShift = p->rShiftPoly[0] + (double)(r1 * sc) * p->rShiftPoly[1] + (double)(a1 * sc) * p->rShiftPoly[2];
            aShift = p->aShiftPoly[0] + (double)(r1 * sc) * p->aShiftPoly[1] + (double)(a1 * sc) * p->aShiftPoly[2];
        }
    }
    rShift /= sc;
    aShift /= sc;
    *r2 = (rShift >= 0) ? r1 + (int)(rShift + 0.5) : r1 + (int)(rShift - 0.5);
    *a2 = (aShift >= 0) ? a1 + (int)(aShift + 0.5) : a1 + (int)(aShift - 0.5);
}

static void zeroPadW(SwCtx *c)
{
    /* zeroPad, corrTrackFast.c:718-761 */
    const int wRa = c->wRa, wAa = c->wAa, W2 = wRa * OS;
    memset(c->f1a, 0, sizeof(ocplx) * (size_t)wAa * OS * W2);
    memset(c->f2a, 0, sizeof(ocplx) * (size_t)wAa * OS * W2);
    int da = c->azShift;
    if (da < 0 || da >= wAa) da = 0;
    for (int i = 0; i < wAa / 2; i++) {
        int i1 = OS * wAa - wAa / OS + i;
        int i2 = (wAa / OS + i + da) % wAa;
        int ia = (i + da) % wAa;
        int j1 = wRa * OS - wRa / OS;
        int j2 = wRa / OS;
        for (int j = 0; j < wRa / 2; j++) {
            int ja = j % wRa, j2a = j2 % wRa;
            c->f1a[i * W2 + j] = c->f1[ia * wRa + ja];
            c->f1a[i1 * W2 + j] = c->f1[i2 * wRa + ja];
            c->f1a[i1 * W2 + j1] = c->f1[i2 * wRa + j2a];
            c->f1a[i * W2 + j1] = c->f1[ia * wRa + j2a];
            c->f2a[i * W2 + j] = c->f2[ia * wRa + ja];
            c->f2a[i1 * W2 + j] = c->f2[i2 * wRa + ja];
            c->f2a[i1 * W2 + j1] = c->f2[i2 * wRa + j2a];
            c->f2a[i * W2 + j1] = c->f2[ia * wRa + j2a];
            j1++;
            j2++;
        }
    }
}

static void detectPatch(SwCtx *c, FLT *data, ocplx *im, int wR, int wA, int edgePadR, int edgePadA, float scale,
                        int largePatch)
{
    /* corrTrackFast.c:765-839 (note: the azimuth clamp uses edgePadR) */
    const sb_track_params *p = c->p;
    const int W2 = c->wRa * OS;
    int extraR = largePatch ? 0 : p->navgR;
    int extraA = largePatch ? 0 : p->navgA;
    for (int i = 0; i < wA; i++) {
        int i1 = edgePadA * OS + i;
        for (int j = 0; j < wR; j++) {
            int j1 = edgePadR * OS + j;
            FLT *d = &data[i * wR + j];
            if (p->navgA > 1 || p->navgR > 1) {
                *d = 0;
                for (int m = -p->navgA; m <= p->navgA; m++) {
                    int k = i1 + m > 0 ? i1 + m : 0;
                    int kmax = edgePadR * OS + wA + extraA - 1;
                    k = k < kmax ? k : kmax;
                    for (int n = -p->navgR; n <= p->navgR; n++) {
                        int l = j1 + n > 0 ? j1 + n : 0;
                        int lmax = edgePadR * OS + wR + extraR - 1;
                        l = l < lmax ? l : lmax;
                        const ocplx *z = &im[k * W2 + l];
                        *d += (FLT)((z->re * z->re + z->im * z->im) * scale);
                    }
                }
            } else {
                const ocplx *z = &im[i1 * W2 + j1];
                *d = (FLT)((z->re * z->re + z->im * z->im) * scale);
            }
        }
    }
    for (int i = 0; i < wA; i++) {
        int i1 = edgePadA * OS + i;
        for (int j = 0; j < wR; j++) {
            int j1 = edgePadR * OS + j;
            data[i * wR + j] = (FLT)sqrt((double)data[i * wR + j]);
            im[i1 * W2 + j1].re = (REAL)data[i * wR + j];
            im[i1 * W2 + j1].im = 0.0;
        }
    }
    const int H2 = c->wAa * OS;
    for (int i = 0; i < H2; i++)
        for (int j = 0; j < edgePadR * OS; j++) {
            im[i * W2 + j].re = im[i * W2 + j].im = 0;
            im[i * W2 + W2 - j - 1].re = im[i * W2 + W2 - j - 1].im = 0;
        }
    for (int i = 0; i < edgePadA * OS; i++)
        for (int j = 0; j < W2; j++) {
            im[i * W2 + j].re = im[i * W2 + j].im = 0;
            im[(H2 - i - 1) * W2 + j].re = im[(H2 - i - 1) * W2 + j].im = 0;
        }
}

static void getCorrPatchesFast(SwCtx *c, int r1, int a1, int r2, int a2)
{
    /* corrTrackFast.c:299-372 */
    const sb_track_params *p = c->p;
    const int wRa = c->wRa, wAa = c->wAa;
    float scale = 1.f / ((float)wRa * (float)wAa * (float)wRa * (float)wAa * (float)(OS * OS * OS * OS) *
                         (float)(OS * OS * (p->navgA + 1) * (p->navgR + 1)));
    for (int i = 0; i < wAa; i++)
        for (int j = 0; j < wRa; j++) {
            sample_w(c->src1, a1 + i, r1 + j, &c->in1[i * wRa + j].re, &c->in1[i * wRa + j].im);
            sample_w(c->src2, a2 + i, r2 + j, &c->in2[i * wRa + j].re, &c->in2[i * wRa + j].im);
        }
    c->azShift = dopShift(wAa, c->in1, c->in2, wAa, wRa);
    offt2d_exec(c->aForwardIn, c->in1, c->f1);
    offt2d_exec(c->aForwardIn, c->in2, c->f2);
    zeroPadW(c);
    offt2d_exec(c->aReverseNoPad, c->f1a, c->img1);
    offt2d_exec(c->aReverseNoPad, c->f2a, c->img2);
    detectPatch(c, c->dataR, c->img2, c->wR2, c->wA2, c->eR, c->eA, scale, FALSE);
    detectPatch(c, c->dataS, c->img1, wRa * OS, wAa * OS, 0, 0, scale, TRUE);
}

static void computeMeanSigma(SwCtx *c, double *meanR, double *sigmaR)
{
    /* corrTrackFast.c:407-477 */
    const int wR2 = c->wR2, wA2 = c->wA2, W = c->wRa * OS, H = c->wAa * OS;
    const int nS = 2 * c->eR * OS + 1;
    *sigmaR = 0;
    *meanR = 0;
    for (int la = 0; la < wA2; la++)
        for (int lr = 0; lr < wR2; lr++) {
            FLT v = c->dataR[la * wR2 + lr];
            *sigmaR += (FLT)(v * v);
            *meanR += v;
        }
    *meanR /= (double)(wR2 * wA2);
    *sigmaR = *sigmaR / (double)(wR2 * wA2 - 1.);
    *sigmaR -= *meanR * (*meanR);
    for (int l = 0; l < H; l++) {
        double sum1 = 0.0, sum2 = 0.0;
        int s1 = 0;
        for (int s = 0; s < W; s++) {
            FLT v = c->dataS[l * W + s];
            sum1 += v;
            sum2 += (FLT)(v * v);
            if (s >= (wR2 - 1)) {
                int s2 = s - (wR2 - 1);
                c->tmpS1[l * W + s1] = sum1;
                c->tmpS2[l * W + s1] = sum2;
                FLT v2 = c->dataS[l * W + s2];
                sum1 -= v2;
                sum2 -= (FLT)(v2 * v2);
                s1++;
            }
        }
    }
    for (int s = 0; s < nS; s++) {
        double sum1 = 0.0, sum2 = 0.0;
        int l1 = 0;
        for (int l = 0; l < H; l++) {
            sum1 += c->tmpS1[l * W + s];
            sum2 += c->tmpS2[l * W + s];
            if (l >= (wA2 - 1)) {
                int l2 = l - (wA2 - 1);
                double m = sum1 / (double)(wR2 * wA2);
                c->meanS[l1 * nS + s] = m;
                c->sigmaS[l1 * nS + s] = sum2 / (double)(wR2 * wA2 - 1) - m * m;
                sum1 -= c->tmpS1[l2 * W + s];
                sum2 -= c->tmpS2[l2 * W + s];
                l1++;
            }
        }
    }
}

static void ampMatchEdge(SwCtx *c)
{
    /* corrTrackFast.c:903-947 */
    const int W = c->wRa * OS, H = c->wAa * OS;
    offt2d_exec(c->aForward, c->img1, c->fa1);
    offt2d_exec(c->aForward, c->img2, c->fa2);
    for (int k = 0; k < W * H; k++) {
        c->ps[k].re = c->fa1[k].re * c->fa2[k].re + c->fa1[k].im * c->fa2[k].im;
        c->ps[k].im = c->fa1[k].im * c->fa2[k].re - c->fa1[k].re * c->fa2[k].im;
    }
    offt2d_exec(c->aReverseNoPad, c->ps, c->ca);
#define MAG(z) ((FLT)sqrt((double)((z).re * (z).re + (z).im * (z).im)))
    for (int i = 0; i < H / 2; i++) {
        int i1 = H / 2 + i, j1 = W / 2;
        for (int j = 0; j < W / 2; j++) {
            c->caMag[i * W + j] = MAG(c->ca[i1 * W + j1]);
            c->caMag[i1 * W + j1] = MAG(c->ca[i * W + j]);
            c->caMag[i1 * W + j] = MAG(c->ca[i * W + j1]);
            c->caMag[i * W + j1] = MAG(c->ca[i1 * W + j]);
            j1++;
        }
    }
#undef MAG
}

static void getPeakCorr(SwCtx *c, int *iMax, int *jMax, double meanR, double sigmaR, double *maxCorr)
{
    /* corrTrackFast.c:862-899 */
    const int eA = c->eA, eR = c->eR, W = c->wRa * OS, nS = 2 * eR * OS + 1;
    double wR2 = c->wRa - 2 * eR, wA2 = c->wAa - 2 * eA;
    double scaleW = 1.0 / ((OS * OS * OS * OS) * c->wAa * wA2 * c->wRa * wR2);
    *maxCorr = -1e30;
    for (int l = -OS * eA; l <= OS * eA; l++) {
        int i = l + OS * eA, m = l + c->wAa * OS / 2;
        for (int s = -OS * eR; s <= OS * eR; s++) {
            int j = s + OS * eR, n = s + c->wRa * OS / 2;
            double v = c->caMag[m * W + n] * scaleW;
            v = v - (meanR * c->meanS[i * nS + j]);
            v = v / sqrt(sigmaR * c->sigmaS[i * nS + j]);
            c->corrResult[i * nS + j] = v;
            if (v > *maxCorr && l >= -OS * (eA - NFAST / 4) && s >= -OS * (eR - NFAST / 4) &&
                l <= OS * (eA - NFAST / 4) && s <= OS * (eR - NFAST / 4)) {
                *maxCorr = v;
                *iMax = i;
                *jMax = j;
            }
        }
    }
}

static void overSampleW(SwCtx *c)
{
    /* corrTrackFast.c:951-990: 21x21 DFT, symmetric zero pad to 336x336, inverse */
    const int N1 = NFAST + 1, NO = N1 * NOVER, half = NFAST / 2;
    offt2d_exec(c->cForwardFast, c->cFast, c->psFast);
    memset(c->psFastOver, 0, sizeof(ocplx) * (size_t)NO * NO);
    for (int i = 0; i <= half; i++) {
        int i1 = NO - half - 1 + i, i2 = half + i;
        int j1 = NO - half - 1, j2 = half;
        for (int j = 0; j <= half; j++) {
            c->psFastOver[i * NO + j] = c->psFast[i * N1 + j];
            if (j != 0) c->psFastOver[i * NO + j1] = c->psFast[i * N1 + j2];
            if (i != 0) {
                c->psFastOver[i1 * NO + j] = c->psFast[i2 * N1 + j];
                if (j != 0) c->psFastOver[i1 * NO + j1] = c->psFast[i2 * N1 + j2];
            }
            j1++;
            j2++;
        }
    }
    offt2d_exec(c->cReverseFast, c->psFastOver, c->cFastOver);
}

static void correlateFast(SwCtx *c, float *rShift, float *aShift, float *cMax)
{
    /* corrTrackFast.c:482-551 */
    double meanR, sigmaR, maxCorr;
    int iMax = 0, jMax = 0, iMax1 = 0, jMax1 = 0;
    const int nS = 2 * c->eR * OS + 1, N1 = NFAST + 1, NO = N1 * NOVER;
    computeMeanSigma(c, &meanR, &sigmaR);
    ampMatchEdge(c);
    getPeakCorr(c, &iMax, &jMax, meanR, sigmaR, &maxCorr);
    if (maxCorr < 0) return;
    for (int i = 0; i <= NFAST; i++) {
        int i1 = iMax - NFAST / 2 + i, j1 = jMax - NFAST / 2;
        for (int j = 0; j <= NFAST; j++) {
            c->cFast[i * N1 + j].re = (REAL)c->corrResult[i1 * nS + j1];
            c->cFast[i * N1 + j].im = 0.0;
            j1++;
        }
    }
    overSampleW(c);
    double cm = -1.0e30;
    for (int i = (N1 * NOVER) / 2 - NOVER * 2; i < (N1 * NOVER) / 2 + NOVER * 2; i++)
        for (int j = (N1 * NOVER) / 2 - NOVER * 2; j < (N1 * NOVER) / 2 + NOVER * 2; j++) {
            const ocplx *z = &c->cFastOver[i * NO + j];
            double corr = (z->re * z->re + z->im * z->im);
            if (corr > cm) { cm = corr; iMax1 = i; jMax1 = j; }
        }
    *cMax = (float)(sqrt(cm) / ((NFAST + 1) * (NFAST + 1)));
    iMax = (iMax * NOVER) + iMax1 - (NOVER * (NFAST)) / 2;
    jMax = (jMax * NOVER) + jMax1 - (NOVER * (NFAST)) / 2;
    *rShift = ((float)jMax - c->eR * OS * NOVER) / (NOVER * OS);
    *aShift = ((float)iMax - c->eA * OS * NOVER) / (NOVER * OS);
}

int oracle_strackw(const sb_track_params *p, const sb_image *img1, const sb_image *img2, sb_track_result *out,
                   int32_t row0, int32_t row1)
{
    if (!p || !img1 || !img2 || !out) return SB_ERR_ARG;
    if (p->polyShift == 0 && p->initOffsets == NULL) return SB_ERR_ARG;
    SwCtx C, *c = &C;
    memset(c, 0, sizeof(C));
    c->p = p;
    c->src1 = img1;
    c->src2 = img2;
    c->wRa = p->wRa;
    c->wAa = p->wAa;
    c->eR = p->edgePadR + NFAST / 4;
    c->eA = p->edgePadA + NFAST / 4;
    c->wR2 = (c->wRa - 2 * c->eR) * OS;
    c->wA2 = (c->wAa - 2 * c->eA) * OS;
    if (c->wR2 <= 0 || c->wA2 <= 0) return SB_ERR_ARG;
    const int wRa = c->wRa, wAa = c->wAa;
    const size_t n = (size_t)wRa * wAa, n4 = n * OS * OS;
    const int nS = 2 * c->eR * OS + 1, nL = 2 * c->eA * OS + 1;
    const int N1 = NFAST + 1, NO = N1 * NOVER;
    c->in1 = wbuf(n); c->in2 = wbuf(n); c->f1 = wbuf(n); c->f2 = wbuf(n);
    c->f1a = wbuf(n4); c->f2a = wbuf(n4); c->img1 = wbuf(n4); c->img2 = wbuf(n4);
    c->fa1 = wbuf(n4); c->fa2 = wbuf(n4); c->ps = wbuf(n4); c->ca = wbuf(n4);
    c->caMag = (FLT *)calloc(n4, sizeof(FLT));
    c->dataS = (FLT *)calloc(n4, sizeof(FLT));
    c->dataR = (FLT *)calloc((size_t)c->wR2 * c->wA2, sizeof(FLT));
    c->tmpS1 = (double *)calloc(n4, sizeof(double));
    c->tmpS2 = (double *)calloc(n4, sizeof(double));
    c->meanS = (double *)calloc((size_t)nL * nS, sizeof(double));
    c->sigmaS = (double *)calloc((size_t)nL * nS, sizeof(double));
    c->corrResult = (double *)calloc((size_t)nL * nS, sizeof(double));
    c->cFast = wbuf((size_t)N1 * N1); c->psFast = wbuf((size_t)N1 * N1);
    c->psFastOver = wbuf((size_t)NO * NO); c->cFastOver = wbuf((size_t)NO * NO);
    c->aForwardIn = offt2d_plan(wAa, wRa, OFFT_FORWARD);
    c->aForward = offt2d_plan(wAa * OS, wRa * OS, OFFT_FORWARD);
    c->aReverseNoPad = offt2d_plan(wAa * OS, wRa * OS, OFFT_BACKWARD);
    c->cForwardFast = offt2d_plan(N1, N1, OFFT_FORWARD);
    c->cReverseFast = offt2d_plan(NO, NO, OFFT_BACKWARD);

    const int nR = p->nR, nA = p->nA;
    if (row1 <= 0 || row1 > nA) row1 = nA;
    if (row0 < 0) row0 = 0;
    for (int i = row0; i < row1; i++)
        for (int j = 0; j < nR; j++) {
            size_t k = (size_t)i * nR + j;
            out->offR[k] = (float)(-LARGEINT);
            out->offA[k] = (float)(-LARGEINT);
            out->corr[k] = 0;
            out->type[k] = SB_BAD;
        }
    int64_t nAmp = 0, nFail = 0, nTried = 0;
    for (int i = row0; i < row1; i++) {
        int a1 = p->aStart + i * p->deltaA - p->wAa / 2;
        for (int j = 0; j < nR; j++) {
            size_t k = (size_t)i * nR + j;
            int r1 = p->rStart + j * p->deltaR - p->wRa / 2, r2, a2;
            findImage2PosW(c, r1, a1, &r2, &a2);
            float rShift = (float)(r2 - r1), aShift = (float)(a2 - a1), cMax = 0.f;
            int maskVal = maskValueW(c, r1 * p->scaleFactor, a1 * p->scaleFactor);
            if (maskVal == 1) {
                if (r1 > 0 && r1 < img1->nr && a1 > 0 && a1 < img1->na && r2 > 0 && r2 < img2->nr && a2 > 0 &&
                    a2 < img2->na) {
                    float rShift1 = 0, aShift1 = 0;
                    nTried++;
                    getCorrPatchesFast(c, r1, a1, r2, a2);
                    correlateFast(c, &rShift1, &aShift1, &cMax);
                    if (cMax > .00) {
                        rShift -= rShift1;
                        aShift -= aShift1;
                        nAmp++;
                    } else {
                        rShift = (float)-LARGEINT;
                        aShift = (float)-LARGEINT;
                        nFail++;
                    }
                    out->offR[k] = rShift;
                    out->offA[k] = aShift;
                    out->corr[k] = cMax;
                    out->type[k] = SB_AMPMATCH;
                }
            } else {
                out->offR[k] = (float)-LARGEINT;
                out->offA[k] = (float)-LARGEINT;
                out->corr[k] = 0;
                out->type[k] = 0;
            }
        }
    }
    out->nComplex = 0;
    out->nAmp = nAmp;
    out->nAmpL = 0;
    out->nFail = nFail;
    out->nAttempted = nTried;

    free(c->in1); free(c->in2); free(c->f1); free(c->f2); free(c->f1a); free(c->f2a);
    free(c->img1); free(c->img2); free(c->fa1); free(c->fa2); free(c->ps); free(c->ca); free(c->caMag);
    free(c->dataS); free(c->dataR); free(c->tmpS1); free(c->tmpS2); free(c->meanS); free(c->sigmaS);
    free(c->corrResult); free(c->cFast); free(c->psFast); free(c->psFastOver); free(c->cFastOver);
    offt2d_destroy(c->aForwardIn); offt2d_destroy(c->aForward); offt2d_destroy(c->aReverseNoPad);
    offt2d_destroy(c->cForwardFast); offt2d_destroy(c->cReverseFast);
    return SB_OK;
}
