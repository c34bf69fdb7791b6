/*
 * shim_clib.c -- TEST INFRASTRUCTURE ONLY.  Stand-ins for the GrIMP library
 * routines (clib, mosaicSource, unwrapSource, gdalIO) that the reference's
 * hot-path sources call but that are not part of the reference tree, so those
 * sources can be compiled and run unmodified as a parity reference.  Written
 * from what each routine is used for at its call sites.
 *
 * error() and nrerror() do not exit the process: they print the message and
 * return to the harness through refshim_fail (longjmp), which then exits with
 * a non-zero status, as the reference's tools would.
 */
#include <math.h>
#include <setjmp.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "clib/standard.h"
#include "gdalIO/gdalIO/grimpgdal.h"
#include "mosaicSource/common/common.h"
#include "unwrapSource/unWrap/unwrapInclude.h"

jmp_buf refshim_fail;
int refshim_fail_armed = 0;

void refshim_abort(void)
{
    if (refshim_fail_armed) longjmp(refshim_fail, 1);
    exit(2);
}

void error(char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vfprintf(stderr, fmt, ap);
    va_end(ap);
    fputc('\n', stderr);
    refshim_abort();
}

FILE *openInputFile(char *file)
{
    FILE *fp = fopen(file, "rb");
    if (!fp) error("openInputFile: cannot open %s", file);
    return fp;
}

FILE *openOutputFile(char *file)
{
    FILE *fp = fopen(file, "wb");
    if (!fp) error("openOutputFile: cannot open %s", file);
    return fp;
}

/* word size of an element kind: the swap is per word, so an 8-byte complex
 * float read with FLOAT32FLAG swaps its two 4-byte halves */
static size_t word_of(int32_t flags)
{
    switch (flags) {
    case INT16FLAG: return 2;
    case INT32FLAG: case FLOAT32FLAG: return 4;
    case FLOAT64FLAG: return 8;
    default: return 1;
    }
}

static void swap_words(unsigned char *p, size_t bytes, size_t w)
{
    if (w <= 1) return;
    for (size_t k = 0; k + w <= bytes; k += w)
        for (size_t a = 0, b = w - 1; a < b; a++, b--) {
            unsigned char t = p[k + a];
            p[k + a] = p[k + b];
            p[k + b] = t;
        }
}

size_t freadBS(void *ptr, size_t size, size_t nitems, FILE *fp, int32_t flags)
{
    size_t n = fread(ptr, size, nitems, fp);
    swap_words((unsigned char *)ptr, n * size, word_of(flags));
    return n;
}

size_t fwriteBS(void *ptr, size_t size, size_t nitems, FILE *fp, int32_t flags)
{
    size_t bytes = size * nitems;
    unsigned char *tmp = (unsigned char *)malloc(bytes ? bytes : 1);
    memcpy(tmp, ptr, bytes);
    swap_words(tmp, bytes, word_of(flags));
    size_t n = fwrite(tmp, size, nitems, fp);
    free(tmp);
    return n;
}

char *appendSuff(char *file, char *suffix, char *buf)
{
    strcpy(buf, file);
    strcat(buf, suffix);
    return buf;
}

/* geocentric radius (km) of the ellipsoid with semi-axes eMajor, eMinor at
 * latitude lat (rad) */
double earthRadius(double lat, double eMinor, double eMajor)
{
    const double a = eMajor, b = eMinor, c = cos(lat), s = sin(lat);
    return sqrt((pow(a * a * c, 2) + pow(b * b * s, 2)) / (pow(a * c, 2) + pow(b * s, 2)));
}

/* bilinear interpolation of image[row][col] at column x, row y; a position
 * outside the grid, or any corner at or below minvalue, gives noData (the
 * same assumption as the oracle's restatement) */
float bilinearInterp(float **image, double x, double y, int32_t nx, int32_t ny, float minvalue, float noData)
{
    if (nx < 2 || ny < 2) return noData;
    if (x < 0 || y < 0 || x > (double)(nx - 1) || y > (double)(ny - 1)) return noData;
    int j = (int)x, i = (int)y;
    if (j >= nx - 1) j = nx - 2;
    if (i >= ny - 1) i = ny - 2;
    double t = x - j, u = y - i;
    float p1 = image[i][j], p2 = image[i][j + 1], p3 = image[i + 1][j + 1], p4 = image[i + 1][j];
    if (p1 <= minvalue || p2 <= minvalue || p3 <= minvalue || p4 <= minvalue) return noData;
    return (float)((1.0 - t) * (1.0 - u) * p1 + t * (1.0 - u) * p2 + t * u * p3 + (1.0 - t) * u * p4);
}

CPLErr GDALRasterIO(GDALRasterBandH hBand, GDALRWFlag eRWFlag, int nXOff, int nYOff, int nXSize, int nYSize,
                    void *pData, int nBufXSize, int nBufYSize, GDALDataType eBufType, int nPixelSpace, int nLineSpace)
{
    (void)hBand; (void)eRWFlag; (void)nXOff; (void)nYOff; (void)nXSize; (void)nYSize; (void)pData;
    (void)nBufXSize; (void)nBufYSize; (void)eBufType; (void)nPixelSpace; (void)nLineSpace;
    error("GDALRasterIO: GDAL is not available; the parity harness reads raw files");
    return CE_Failure;
}

/* connected components of the REGION pixels (see unwrapInclude.h) */
int refshim_label_connectivity = 8;

static int32_t uf_root(int32_t *par, int32_t k)
{
    while (par[k] != k) {
        par[k] = par[par[k]];
        k = par[k];
    }
    return k;
}

void labelRegions(unwrapImageStructure *uw)
{
    const int nr = uw->rangeSize, na = uw->azimuthSize;
    const size_t n = (size_t)nr * na;
    int32_t *par = (int32_t *)malloc(sizeof(int32_t) * (n ? n : 1));
    for (int i = 0; i < na; i++)
        for (int j = 0; j < nr; j++) {
            size_t k = (size_t)i * nr + j;
            par[k] = (uw->bCuts[i][j] & REGION) ? (int32_t)k : -1;
        }
    const int nb8[4][2] = {{0, -1}, {-1, 0}, {-1, -1}, {-1, 1}};
    const int nnb = refshim_label_connectivity == 4 ? 2 : 4;
    for (int i = 0; i < na; i++)
        for (int j = 0; j < nr; j++) {
            size_t k = (size_t)i * nr + j;
            if (par[k] < 0) continue;
            for (int q = 0; q < nnb; q++) {
                int ii = i + nb8[q][0], jj = j + nb8[q][1];
                if (ii < 0 || jj < 0 || jj >= nr) continue;
                size_t kk = (size_t)ii * nr + jj;
                if (par[kk] < 0) continue;
                int32_t ra = uf_root(par, (int32_t)k), rb = uf_root(par, (int32_t)kk);
                if (ra < rb) par[rb] = ra;
                else if (rb < ra) par[ra] = rb;
            }
        }
    int32_t next = 0;
    int32_t *lab = (int32_t *)malloc(sizeof(int32_t) * (n ? n : 1));
    for (size_t k = 0; k < n; k++) {
        if (par[k] < 0) { lab[k] = LARGEINT; continue; }
        int32_t r = uf_root(par, (int32_t)k);
        lab[k] = (r == (int32_t)k) ? ++next : lab[r];
    }
    for (int i = 0; i < na; i++)
        for (int j = 0; j < nr; j++) uw->labels[i][j] = lab[(size_t)i * nr + j];
    free(par);
    free(lab);
}
