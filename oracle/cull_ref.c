/*
 * cull_ref.c -- TEST INFRASTRUCTURE ONLY (CPU oracle, pinned to the reference build by tests/test_ref_pin.py).
 *
 * Restatement of the cullst pipeline: Cullst/cullst.c:36-121,
 * Cullst/cullSTData.c, cullStats.c, cullSmooth.c, cullIslands.c.  The
 * arithmetic keeps the reference's float/double types (both oracle builds are
 * identical here).  Third-party pieces absent from the reference tree:
 *  - selectForCull (cullSTData.c:132-192, Numerical Recipes' select adapted):
 *    restated as "k-th smallest value, 1-based", which is what it is written
 *    to return.  As compiled, it does not: at :160 the three-statement SWAP
 *    macro follows an unbraced if, so two of its statements always run and
 *    read an uninitialised temporary; the value it returns then depends on
 *    the compiler (tests/test_ref_pin.py).  With nGood = 0 a box with one
 *    valid point makes it return listR[0], which is never written.
 *  - Numerical Recipes svdfit (cullStats.c:91-95): least squares by SVD with
 *    singular values below 1e-5 * max zeroed (the published svdfit TOL);
 *    restated through the eigen-decomposition of the 3x3 normal matrix.
 *  - GrIMP labelRegions (cullIslands.c:78): connected components of the
 *    REGION pixels, labelled 1..K in order of first appearance in a row-major
 *    scan; 8-connectivity unless connectivity == 4.  This is an assumption
 *    (the routine's source is not available); island culling is pinned to
 *    this labelling.
 * cullls (Cullls/cullls.c:23-56, cullLSData.c, cullLSStats.c, cullLSSmooth.c,
 * cullLSIslands.c) shares the stats and islands passes; the landsatSource64
 * values it reads (SLOWVEL, NODATATOUSE, NODATA, NOVER, the lsFit/matchResult
 * fields) come from headers absent from the tree and are inputs here.
 * LARGEINT is 2e9 (clib) except in cullst.c, which redefines it as -2e9, so
 * addSubtractSimOffsets applies to every finite point (cullst.c:11,115).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define LARGEINT 2000000000
#define NARROWREGION 4
#define TRUE 1
#define FALSE 0

static inline int validPt(float r, float a)
{
    /* offR > (1 - LARGEINT) && offA > (1 - LARGEINT), int converted to float */
    const float lim = (float)(1 - LARGEINT);
    return r > lim && a > lim;
}

static void addSubtractSim(const sb_cull_params *p, sb_cull_data *d, float mySign)
{
    /* cullst.c:109-121 with the local LARGEINT = -2e9 */
    const size_t n = (size_t)p->nR * p->nA;
    for (size_t k = 0; k < n; k++) {
        if ((double)d->offA[k] < (2e9 + 1) && (double)d->simA[k] < (2e9 + 1)) {
            d->offA[k] += mySign * d->simA[k];
            d->offR[k] += mySign * d->simR[k];
        }
    }
}

static int cmpf(const void *a, const void *b)
{
    float x = *(const float *)a, y = *(const float *)b;
    return (x > y) - (x < y);
}

int oracle_cull_st_data(const sb_cull_params *p, sb_cull_data *d)
{
    /* cullSTData.c:13-125 */
    const int nR = p->nR, nA = p->nA;
    float *offR = d->offR, *offA = d->offA;
    float *listR = (float *)malloc(sizeof(float) * (size_t)(1000 + (p->bR + 1) * (p->bA + 1)));
    float *listA = (float *)malloc(sizeof(float) * (size_t)(1000 + (p->bR + 1) * (p->bA + 1)));
    int maskFlag = (d->mask != NULL);
    for (int i = 0; i < nA; i++)
        for (int j = 0; j < nR; j++) {
            size_t k = (size_t)i * nR + j;
            if (d->corr[k] < p->corrThresh) {
                offR[k] = (float)-LARGEINT;
                offA[k] = (float)-LARGEINT;
                d->type[k] = 0;
            }
            if (maskFlag) {
                unsigned char maskVal = (unsigned char)d->mask[k] & NARROWREGION;
                if (maskVal > 0 && (signed char)d->type[k] > 2) {
                    offR[k] = (float)-LARGEINT;
                    offA[k] = (float)-LARGEINT;
                    d->type[k] = 0;
                }
                if ((p->singleMT > 0) && ((signed char)d->type[k] != p->singleMT)) {
                    offR[k] = (float)-LARGEINT;
                    offA[k] = (float)-LARGEINT;
                    d->type[k] = 0;
                }
            }
        }
    int64_t nCulled = 0;
    for (int i = 0; i < nA; i++) {
        int i1 = i - p->bA / 2 > 0 ? i - p->bA / 2 : 0;
        int i2 = i + p->bA / 2 < nA - 1 ? i + p->bA / 2 : nA - 1;
        for (int j = 0; j < nR; j++) {
            int j1 = j - p->bR / 2 > 0 ? j - p->bR / 2 : 0;
            int j2 = j + p->bR / 2 < nR - 1 ? j + p->bR / 2 : nR - 1;
            uint32_t ngood = 0;
            for (int ii = i1; ii <= i2; ii++)
                for (int jj = j1; jj <= j2; jj++) {
                    size_t kk = (size_t)ii * nR + jj;
                    if (validPt(offR[kk], offA[kk])) {
                        listR[ngood] = offR[kk];
                        listA[ngood] = offA[kk];
                        ngood++;
                    }
                }
            size_t k = (size_t)i * nR + j;
            if (ngood > (uint32_t)p->nGood) {
                uint32_t midIndex = ngood / 2; /* 1-based rank */
                if (midIndex < 1) midIndex = 1; /* ngood == 1 (nGood 0): the reference reads arr[0], unset */
                qsort(listR, ngood, sizeof(float), cmpf);
                qsort(listA, ngood, sizeof(float), cmpf);
                float medianR = listR[midIndex - 1], medianA = listA[midIndex - 1];
                double diffA = (double)(offA[k] - medianA);
                double diffR = (double)(offR[k] - medianR);
                if (fabs(diffA) > p->maxA || fabs(diffR) > p->maxR) {
                    offR[k] = (float)-LARGEINT;
                    offA[k] = (float)-LARGEINT;
                    nCulled++;
                }
            } else {
                offR[k] = (float)-LARGEINT;
                offA[k] = (float)-LARGEINT;
                nCulled++;
            }
        }
    }
    d->nCulled = nCulled;
    free(listR);
    free(listA);
    return SB_OK;
}

/* Jacobi eigen-decomposition of a symmetric 3x3 matrix: A = V diag(e) V^T. */
static void jacobi3(double A[3][3], double e[3], double V[3][3])
{
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) V[i][j] = (i == j);
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = fabs(A[0][1]) + fabs(A[0][2]) + fabs(A[1][2]);
        if (off == 0.0) break;
        for (int pq = 0; pq < 3; pq++) {
            int P = pq == 2 ? 1 : 0, Q = pq == 0 ? 1 : 2;
            if (A[P][Q] == 0.0) continue;
            double theta = (A[Q][Q] - A[P][P]) / (2.0 * A[P][Q]);
            double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
            for (int k = 0; k < 3; k++) {
                double akp = A[k][P], akq = A[k][Q];
                A[k][P] = cs * akp - sn * akq;
                A[k][Q] = sn * akp + cs * akq;
            }
            for (int k = 0; k < 3; k++) {
                double apk = A[P][k], aqk = A[Q][k];
                A[P][k] = cs * apk - sn * aqk;
                A[Q][k] = sn * apk + cs * aqk;
            }
            for (int k = 0; k < 3; k++) {
                double vkp = V[k][P], vkq = V[k][Q];
                V[k][P] = cs * vkp - sn * vkq;
                V[k][Q] = sn * vkp + cs * vkq;
            }
        }
    }
    for (int i = 0; i < 3; i++) e[i] = A[i][i];
}

/* svdfit with basis (c0, ii, jj), unit sigma; singular values < 1e-5*max are
 * dropped.  Returns the three coefficients. */
static void planeFit(const double *x0, const float *xs, const float *ys, const double *v, int n, double coef[3])
{
    double AtA[3][3] = {{0}}, Atb[3] = {0}, e[3], V[3][3];
    for (int k = 0; k < n; k++) {
        double f[3] = {x0[0], (double)xs[k], (double)ys[k]};
        for (int a = 0; a < 3; a++) {
            Atb[a] += f[a] * v[k];
            for (int b = 0; b < 3; b++) AtA[a][b] += f[a] * f[b];
        }
    }
    jacobi3(AtA, e, V);
    double smax = 0, s[3];
    for (int a = 0; a < 3; a++) {
        s[a] = e[a] > 0 ? sqrt(e[a]) : 0.0;
        smax = s[a] > smax ? s[a] : smax;
    }
    double thresh = 1.0e-5 * smax;
    coef[0] = coef[1] = coef[2] = 0.0;
    for (int a = 0; a < 3; a++) {
        if (s[a] < thresh || s[a] == 0.0) continue;
        double proj = V[0][a] * Atb[0] + V[1][a] * Atb[1] + V[2][a] * Atb[2];
        double w = proj / (s[a] * s[a]);
        for (int b = 0; b < 3; b++) coef[b] += V[b][a] * w;
    }
}

/* cullStats.c:19-144 (box fixed at 9x9, :38-39); cullLSStats.c:19-157 is
 * the same with qvar = (1/NOVER)^2/12 added to the variances before the root
 * (:147-148). */
static void stats_core(int nR, int nA, const float *offR, const float *offA, float *sigmaR, float *sigmaA,
                       double qvar)
{
    const int bR = 9, bA = 9;
    const int cap = 1 + (bR + 1) * (bA + 1);
    double *listR = (double *)malloc(sizeof(double) * cap), *listA = (double *)malloc(sizeof(double) * cap);
    float *xs = (float *)malloc(sizeof(float) * cap), *ys = (float *)malloc(sizeof(float) * cap);
    double aR[4] = {0, 0, 0, 0}, aA[4] = {0, 0, 0, 0};
    for (int i = 0; i < nA; i++) {
        int i1 = i - bA / 2 > 0 ? i - bA / 2 : 0;
        int i2 = i + bA / 2 < nA - 1 ? i + bA / 2 : nA - 1;
        for (int j = 0; j < nR; j++) {
            int j1 = j - bR / 2 > 0 ? j - bR / 2 : 0;
            int j2 = j + bR / 2 < nR - 1 ? j + bR / 2 : nR - 1;
            uint32_t ngood = 0;
            double meanA = 0.0, meanR = 0.0;
            for (int ii = i1; ii <= i2; ii++)
                for (int jj = j1; jj <= j2; jj++) {
                    size_t kk = (size_t)ii * nR + jj;
                    if (validPt(offR[kk], offA[kk])) {
                        listR[ngood] = offR[kk];
                        listA[ngood] = offA[kk];
                        meanA += offA[kk];
                        meanR += offR[kk];
                        xs[ngood] = (float)ii;
                        ys[ngood] = (float)jj;
                        ngood++;
                    }
                }
            meanA /= (double)ngood;
            meanR /= (double)ngood;
            if (ngood > 8) {
                double c[3], x0;
                x0 = (double)(float)meanR; /* data[0].x is a float */
                planeFit(&x0, xs, ys, listR, (int)ngood, c);
                aR[1] = c[0]; aR[2] = c[1]; aR[3] = c[2];
                x0 = (double)(float)meanA;
                planeFit(&x0, xs, ys, listA, (int)ngood, c);
                aA[1] = c[0]; aA[2] = c[1]; aA[3] = c[2];
                aR[1] *= meanR;
                aA[1] *= meanA;
            }
            ngood = 0;
            meanA = meanR = 0.0;
            double varR = 0.0, varA = 0.0;
            for (int ii = i1; ii <= i2; ii++)
                for (int jj = j1; jj <= j2; jj++) {
                    size_t kk = (size_t)ii * nR + jj;
                    if (validPt(offR[kk], offA[kk])) {
                        ngood++;
                        float oR = offR[kk], oA = offA[kk];
                        oR = (float)(oR - (aR[1] + aR[2] * (float)ii + aR[3] * (float)jj));
                        oA = (float)(oA - (aA[1] + aA[2] * (float)ii + aA[3] * (float)jj));
                        meanA += oA;
                        meanR += oR;
                        varA += (float)(oA * oA);
                        varR += (float)(oR * oR);
                    }
                }
            size_t k = (size_t)i * nR + j;
            if (ngood > 8 && offR[k] > (float)(1 - LARGEINT)) {
                float sA = (float)(varA / (float)(ngood - 3));
                float sR = (float)(varR / (float)(ngood - 3));
                sA = (float)(sA - meanA * meanA / (float)((ngood - 3) * ngood));
                sR = (float)(sR - meanR * meanR / (float)((ngood - 3) * ngood));
                sA = (float)(0.00001 > sA ? 0.00001 : sA);
                sR = (float)(0.00001 > sR ? 0.00001 : sR);
                if (qvar != 0.0) {
                    sR += qvar;
                    sA += qvar;
                }
                sigmaA[k] = (float)sqrt((double)sA);
                sigmaR[k] = (float)sqrt((double)sR);
            } else {
                sigmaA[k] = (float)-LARGEINT;
                sigmaR[k] = (float)-LARGEINT;
            }
        }
    }
    free(listR); free(listA); free(xs); free(ys);
}

int oracle_cull_stats(const sb_cull_params *p, sb_cull_data *d)
{
    stats_core(p->nR, p->nA, d->offR, d->offA, d->sigmaR, d->sigmaA, 0.0);
    return SB_OK;
}

static float *sWeights(int s)
{
    /* cullSmooth.c:10-27: 1 inside, 0.5 at the ends for even widths */
    float w2 = (float)((float)s / 2.0 - 0.01);
    float *w = (float *)malloc(sizeof(float) * (size_t)(s + 2));
    float *c = w + s / 2;
    for (int m = -s / 2; m <= s / 2; m++) c[m] = (m < -w2 || m > w2) ? 0.5f : 1.0f;
    return w;
}

int oracle_cull_smooth(const sb_cull_params *p, sb_cull_data *d)
{
    /* cullSmooth.c:29-103 */
    const int nR = p->nR, nA = p->nA;
    const float nlooks[4] = {0.0f, 1.0f, 0.25f, 0.015f};
    float *wAbase = sWeights(p->sA), *wRbase = sWeights(p->sR);
    float *wA = wAbase + p->sA / 2, *wR = wRbase + p->sR / 2;
    for (int i = 0; i < nA; i++) {
        int i1 = i - p->sA / 2 > 0 ? i - p->sA / 2 : 0;
        int iwStart = i1 - i;
        int i2 = i + p->sA / 2 < nA - 1 ? i + p->sA / 2 : nA - 1;
        for (int j = 0; j < nR; j++) {
            int j1 = j - p->sR / 2 > 0 ? j - p->sR / 2 : 0;
            int j2 = j + p->sR / 2 < nR - 1 ? j + p->sR / 2 : nR - 1;
            int jwStart = j1 - j;
            double ngood = 0, meanA = 0.0, meanR = 0.0;
            float nLooksEff = 0.0f;
            int iw = iwStart;
            for (int ii = i1; ii <= i2; ii++, iw++) {
                int jw = jwStart;
                for (int jj = j1; jj <= j2; jj++, jw++) {
                    size_t kk = (size_t)ii * nR + jj;
                    if (validPt(d->offR[kk], d->offA[kk])) {
                        double w = wA[iw] * wR[jw];
                        ngood += w;
                        nLooksEff = (float)(nLooksEff + w * nlooks[(int)(signed char)d->type[kk] & 3]);
                        meanA += w * d->offA[kk];
                        meanR += w * d->offR[kk];
                    }
                }
            }
            size_t k = (size_t)i * nR + j;
            if (((ngood > 1) || (p->sA == 1) || (p->sR == 1)) && d->offR[k] > (float)(1 - LARGEINT) &&
                d->sigmaA[k] > (float)(1 - LARGEINT)) {
                nLooksEff = (float)(nLooksEff > 1. ? nLooksEff : 1.);
                d->sigmaA[k] = (float)(d->sigmaA[k] / sqrt((double)nLooksEff));
                d->sigmaR[k] = (float)(d->sigmaR[k] / sqrt((double)nLooksEff));
                d->offRS[k] = (float)(meanR / (float)ngood);
                d->offAS[k] = (float)(meanA / (float)ngood);
            } else {
                d->offRS[k] = (float)-LARGEINT;
                d->offAS[k] = (float)-LARGEINT;
            }
        }
    }
    free(wAbase);
    free(wRbase);
    return SB_OK;
}

/* union-find with path halving */
static int32_t uf_find(int32_t *par, int32_t x)
{
    while (par[x] != x) {
        par[x] = par[par[x]];
        x = par[x];
    }
    return x;
}

/* cullIslands.c:13-168 + screenIslands :173-198 (cullLSIslands.c:15-204 is
 * the same on XS/YS) */
static void islands_core(int nR, int nA, int connectivity, int islandThresh, float *offRS, float *offAS,
                         int64_t *nIslands, int64_t *nIslandPoints)
{
    const size_t n = (size_t)nR * nA;
    const float regionMin = (float)(-LARGEINT + 1000);
    int32_t *par = (int32_t *)malloc(sizeof(int32_t) * n);
    for (size_t k = 0; k < n; k++) par[k] = offRS[k] >= regionMin ? (int32_t)k : -1;
    const int conn8 = (connectivity != 4);
    for (int i = 0; i < nA; i++)
        for (int j = 0; j < nR; j++) {
            size_t k = (size_t)i * nR + j;
            if (par[k] < 0) continue;
            int nb[4][2] = {{0, -1}, {-1, 0}, {-1, -1}, {-1, 1}};
            int nnb = conn8 ? 4 : 2;
            for (int q = 0; q < nnb; q++) {
                int ii = i + nb[q][0], jj = j + nb[q][1];
                if (ii < 0 || jj < 0 || jj >= nR) continue;
                size_t kk = (size_t)ii * nR + jj;
                if (par[kk] < 0) continue;
                int32_t ra = uf_find(par, (int32_t)k), rb = uf_find(par, (int32_t)kk);
                if (ra != rb) {
                    if (ra < rb) par[rb] = ra; else par[ra] = rb;
                }
            }
        }
    /* labels 1..K by first appearance (the root is the smallest raster index) */
    int32_t *label = (int32_t *)malloc(sizeof(int32_t) * n);
    int32_t K = 0;
    for (size_t k = 0; k < n; k++) {
        if (par[k] < 0) { label[k] = 0; continue; }
        int32_t r = uf_find(par, (int32_t)k);
        if (r == (int32_t)k) label[k] = ++K;
        else label[k] = label[r];
    }
    int32_t *minX = (int32_t *)malloc(sizeof(int32_t) * (size_t)(K + 1));
    int32_t *maxX = (int32_t *)malloc(sizeof(int32_t) * (size_t)(K + 1));
    int32_t *minY = (int32_t *)malloc(sizeof(int32_t) * (size_t)(K + 1));
    int32_t *maxY = (int32_t *)malloc(sizeof(int32_t) * (size_t)(K + 1));
    for (int32_t l = 0; l <= K; l++) { minX[l] = minY[l] = LARGEINT; maxX[l] = maxY[l] = -LARGEINT; }
    for (int i = 0; i < nA; i++)
        for (int j = 0; j < nR; j++) {
            int32_t l = label[(size_t)i * nR + j];
            if (l <= 0) continue;
            if (j < minX[l]) minX[l] = j;
            if (j > maxX[l]) maxX[l] = j;
            if (i < minY[l]) minY[l] = i;
            if (i > maxY[l]) maxY[l] = i;
        }
    int64_t nIsl = 0, nPts = 0;
    char *cull = (char *)calloc((size_t)K + 1, 1);
    for (int32_t l = 1; l < K; l++) { /* label K is skipped, as in the reference */
        if ((maxX[l] - minX[l]) > islandThresh || (maxY[l] - minY[l]) > islandThresh) continue;
        cull[l] = 1;
        nIsl++;
    }
    for (size_t k = 0; k < n; k++)
        if (label[k] > 0 && cull[label[k]]) {
            offRS[k] = (float)-LARGEINT;
            if (offAS) offAS[k] = (float)-LARGEINT;
            nPts++;
        }
    *nIslands = nIsl;
    *nIslandPoints = nPts;
    free(par); free(label); free(minX); free(maxX); free(minY); free(maxY); free(cull);
}

int oracle_cull_islands(const sb_cull_params *p, sb_cull_data *d)
{
    islands_core(p->nR, p->nA, p->connectivity, p->islandThresh, d->offRS, d->offAS, &d->nIslands,
                 &d->nIslandPoints);
    return SB_OK;
}

int oracle_cull(const sb_cull_params *p, sb_cull_data *d)
{
    /* cullst.c:36-107 */
    if (p->useSim) addSubtractSim(p, d, -1.0f);
    int passes = p->nCullPasses > 0 ? p->nCullPasses : 3;
    for (int k = 0; k < passes; k++) oracle_cull_st_data(p, d);
    oracle_cull_stats(p, d);
    if (p->useSim) addSubtractSim(p, d, 1.0f);
    oracle_cull_smooth(p, d);
    if (p->islandThresh > 0) oracle_cull_islands(p, d);
    return SB_OK;
}

/* ---------------------------------------------------------------- cullls */

/* cullLSData.c:13-138: the cullSTData median test on X (columns) and Y
 * (rows) without the corr/mask pre-pass.  A point is kept when more than
 * nGood box points are valid, Y > NODATA + 1, and both deviations from the
 * box medians are within the limits; the limits are 40 m/yr * deltaT / pixel
 * size (at least 0.2) when every valid box point carries the SLOWVEL bit,
 * else maxX/maxY.  The first pass also counts the valid points (nMatch) and
 * the points with data (nAttempt). */
static void cullls_data(const sb_cullls_params *p, sb_cullls_data *d, int first)
{
    const int nx = p->nx, ny = p->ny;
    float *X = d->X, *Y = d->Y;
    const int bR = p->boxSize, bA = p->boxSize;
    float *listX = (float *)malloc(sizeof(float) * (size_t)(1000 + (bR + 1) * (bA + 1)));
    float *listY = (float *)malloc(sizeof(float) * (size_t)(1000 + (bR + 1) * (bA + 1)));
    if (first) {
        int64_t nGoodPts = 0, nWithData = 0;
        for (size_t k = 0; k < (size_t)nx * ny; k++) {
            if (validPt(X[k], Y[k])) nGoodPts++;
            if ((d->type[k] & p->noDataMask) == 0) nWithData++;
        }
        d->nAttempt = nWithData;
        d->nMatch = nGoodPts;
    }
    double slowX = 40.0 / 365. * p->deltaT, slowY = slowX;
    slowX /= p->dx;
    slowY /= p->dy;
    slowX = slowX > 0.2 ? slowX : 0.2;
    slowY = slowY > 0.2 ? slowY : 0.2;
    int64_t nCulled = 0;
    for (int i = 0; i < ny; i++) {
        int i1 = i - bA / 2 > 0 ? i - bA / 2 : 0;
        int i2 = i + bA / 2 < ny - 1 ? i + bA / 2 : ny - 1;
        for (int j = 0; j < nx; j++) {
            int j1 = j - bR / 2 > 0 ? j - bR / 2 : 0;
            int j2 = j + bR / 2 < nx - 1 ? j + bR / 2 : nx - 1;
            int slowFlag = TRUE;
            uint32_t ngood = 0;
            for (int ii = i1; ii <= i2; ii++)
                for (int jj = j1; jj <= j2; jj++) {
                    size_t kk = (size_t)ii * nx + jj;
                    if (validPt(X[kk], Y[kk])) {
                        listX[ngood] = X[kk];
                        listY[ngood] = Y[kk];
                        ngood++;
                        if (!(d->type[kk] & p->slowVelMask)) slowFlag = FALSE;
                    }
                }
            size_t k = (size_t)i * nx + j;
            if (ngood > (uint32_t)p->nGood && (double)Y[k] > p->noDataLimit) {
                uint32_t midIndex = ngood / 2;
                if (midIndex < 1) midIndex = 1;
                qsort(listX, ngood, sizeof(float), cmpf);
                qsort(listY, ngood, sizeof(float), cmpf);
                float medianX = listX[midIndex - 1], medianY = listY[midIndex - 1];
                double diffY = (double)(Y[k] - medianY);
                double diffX = (double)(X[k] - medianX);
                double maxX = slowFlag ? slowX : (double)p->maxX;
                double maxY = slowFlag ? slowY : (double)p->maxY;
                if (fabs(diffY) > maxY || fabs(diffX) > maxX) {
                    X[k] = (float)-LARGEINT;
                    Y[k] = (float)-LARGEINT;
                    nCulled++;
                }
            } else {
                X[k] = (float)-LARGEINT;
                Y[k] = (float)-LARGEINT;
                nCulled++;
            }
        }
    }
    d->nCulled = nCulled;
    free(listX);
    free(listY);
}

/* cullLSSmooth.c:29-70: unweighted box mean, one look per valid point. */
static void cullls_smooth(const sb_cullls_params *p, sb_cullls_data *d)
{
    const int nx = p->nx, ny = p->ny;
    for (int i = 0; i < ny; i++) {
        int i1 = i - p->sY / 2 > 0 ? i - p->sY / 2 : 0;
        int i2 = i + p->sY / 2 < ny - 1 ? i + p->sY / 2 : ny - 1;
        for (int j = 0; j < nx; j++) {
            int j1 = j - p->sX / 2 > 0 ? j - p->sX / 2 : 0;
            int j2 = j + p->sX / 2 < nx - 1 ? j + p->sX / 2 : nx - 1;
            uint32_t ngood = 0;
            float nLooksEff = 0.0f;
            double meanY = 0.0, meanX = 0.0;
            for (int ii = i1; ii <= i2; ii++)
                for (int jj = j1; jj <= j2; jj++) {
                    size_t kk = (size_t)ii * nx + jj;
                    if (validPt(d->X[kk], d->Y[kk])) {
                        ngood++;
                        nLooksEff++;
                        meanY += d->Y[kk];
                        meanX += d->X[kk];
                    }
                }
            size_t k = (size_t)i * nx + j;
            if (((ngood > 1) || (p->sY == 1) || (p->sX == 1)) && d->X[k] > (float)(1 - LARGEINT) &&
                d->sigmaY[k] > (float)(1 - LARGEINT)) {
                nLooksEff = (float)((double)nLooksEff > 1. ? (double)nLooksEff : 1.);
                d->sigmaY[k] = (float)(d->sigmaY[k] / sqrt((double)nLooksEff));
                d->sigmaX[k] = (float)(d->sigmaX[k] / sqrt((double)nLooksEff));
                d->XS[k] = (float)(meanX / (float)ngood);
                d->YS[k] = (float)(meanY / (float)ngood);
            } else {
                d->XS[k] = (float)-LARGEINT;
                d->YS[k] = (float)-LARGEINT;
            }
        }
    }
}

int oracle_cullls(const sb_cullls_params *p, sb_cullls_data *d)
{
    /* cullls.c:23-56 */
    int passes = p->nCullPasses > 0 ? p->nCullPasses : 3;
    for (int k = 0; k < passes; k++) cullls_data(p, d, k == 0);
    stats_core(p->nx, p->ny, d->X, d->Y, d->sigmaX, d->sigmaY, ((1.0 / p->nOver) * (1.0 / p->nOver)) / 12.);
    cullls_smooth(p, d);
    d->nIslands = d->nIslandPoints = 0;
    if (p->islandThresh > 0)
        islands_core(p->nx, p->ny, p->connectivity, p->islandThresh, d->XS, d->YS, &d->nIslands, &d->nIslandPoints);
    return SB_OK;
}
