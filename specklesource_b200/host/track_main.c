/*
 * track_main.c -- the drop-in `strack` and `strackw` command lines (built
 * twice; -DSTRACKW selects strackw).  Same flags, parameter-file keys and
 * output files as Strack/strack.c + Strack/parseTrack.c (strack) and
 * Strackw/strackw.c (strackw); the per-point work runs on the GPU through
 * sb_strack / sb_strackw.
 *
 *   strack  [-noComplex -singleAmp -gauss -integerComplex -noHanning -checkAzFocus -LSB] parFile
 *   strackw [-integerComplex -LSB] parFile
 *
 * Images are raw SLC files described by a GDAL VRT sidecar (<image>.vrt).
 * GrIMP .par/geodat readers (readOldPar, parseInputFile) are not part of the
 * reference tree, so `image1par` files, geodat masks and a non-zero baseline
 * are refused with a message, and an interferogram (intfile, strack only)
 * takes its size and looks from <intfile>.vrt.
 */
#define _GNU_SOURCE
#include <libgen.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "../../include/speckle_b200.h"
#include "sbio.h"

extern const char *sbio_tool;

#ifdef STRACKW
#define TOOL "strackw"
#else
#define TOOL "strack"
#endif

static void usage(void)
{
#ifdef STRACKW
    sbio_die("sTrack -integerComplex -LSB parFile \n\tLSB  use LSB for both output and floating point input");
#else
    sbio_die("sTrack -noComplex -singleAmp -gauss -integerComplex -noHanning -checkAzFocus -LSB parFile \n"
             "\tLSB  use LSB for both output and floating point input");
#endif
}

typedef struct {
    int noComplex, floatFlag, hanningFlag, gaussFlag, maxTries, byteOrder, checkAzFocus;
    const char *parFile;
} Args;

static void read_args(int argc, char **argv, Args *a)
{
    /* Strack/strack.c:137-178, Strackw/strackw.c:129-150 */
    a->floatFlag = 1;
    a->noComplex = 0;
    a->hanningFlag = 1;
    a->gaussFlag = 0;
    a->byteOrder = SB_MSB;
    a->maxTries = 2;
    a->checkAzFocus = 0;
#ifdef STRACKW
    if (argc < 2 || argc > 4) usage();
    a->noComplex = 1;
#else
    if (argc < 2 || argc > 6) usage();
#endif
    a->parFile = argv[argc - 1];
    for (int i = 1; i <= argc - 2; i++) {
        const char *s = strchr(argv[i], '-');
        if (!s) usage();
#ifndef STRACKW
        if (strstr(s, "noComplex")) a->noComplex = 1;
        else
#endif
        if (strstr(s, "integerComplex")) a->floatFlag = 0;
#ifndef STRACKW
        else if (strstr(s, "-noHanning")) a->hanningFlag = 0;
        else if (strstr(s, "-gauss")) a->gaussFlag = 1;
        else if (strstr(s, "-singleAmp")) a->maxTries = 1;
        else if (strstr(s, "-checkAzFocus")) a->checkAzFocus = 1;
#endif
        else if (strstr(s, "-LSB")) a->byteOrder = SB_LSB;
        else usage();
    }
}

static int ival(const sbio_rdf *r, const char *key, int required, int dflt)
{
    const char *v = sbio_rdf_get(r, key);
    int x;
    if (!v) {
        if (required) sbio_die("%s not specified", key);
        return dflt;
    }
    if (sscanf(v, "%i", &x) != 1) {
        if (required) sbio_die("Invalid %s", key);
        return dflt;
    }
    return x;
}

static char *suffixed(const char *base, const char *suf)
{
    char *s = malloc(strlen(base) + strlen(suf) + 1);
    strcpy(s, base);
    strcat(s, suf);
    return s;
}

/* An SLC image through its VRT sidecar (checkForVrt + parseSLCVrtNew). */
/* The interferogram for getInt (Strack/getInt.c:11-77): complex int16 samples,
 * big-endian unless its VRT says LSB, with the size and looks that the
 * reference takes from the intgeodat file.  GrIMP's geodat reader
 * (parseInputFile) is not part of the reference tree, so the same facts come
 * from <intfile>.vrt: rasterXSize/rasterYSize, dataType CInt16, ByteOrder and
 * the metadata keys nRangeLooks / nAzimuthLooks.  As in getInt, a file with
 * fewer lines than the raster is read as far as it goes and the missing lines
 * hold (1, 1). */
static void load_interferogram(const char *intFile, sb_interferogram *f)
{
    char vrt[4200];
    snprintf(vrt, sizeof vrt, "%s.vrt", intFile);
    sbio_vrt v;
    if (!sbio_exists(vrt) || !sbio_vrt_read(vrt, &v))
        sbio_die("getInt: %s needs a VRT sidecar %s (size, CInt16, ByteOrder, nRangeLooks, nAzimuthLooks): "
                 "GrIMP's geodat reader is not part of the reference tree", intFile, vrt);
    if (v.sampleType != SB_CINT16) sbio_die("getInt: %s must describe CInt16 samples", vrt);
    const char *nrl = sbio_vrt_meta(&v, "nRangeLooks"), *nal = sbio_vrt_meta(&v, "nAzimuthLooks");
    if (!nrl || !nal) sbio_die("getInt: %s lacks nRangeLooks / nAzimuthLooks", vrt);
    f->nr = v.nr;
    f->na = v.na;
    f->nrl = atoi(nrl);
    f->nal = atoi(nal);
    if (f->nr <= 0 || f->na <= 0 || f->nrl <= 0 || f->nal <= 0) sbio_die("getInt: invalid size or looks in %s", vrt);
    f->byteOrder = v.byteOrder == SB_LSB ? SB_LSB : SB_MSB;
    f->onDevice = 0;
    const size_t row = (size_t)f->nr * 4;
    unsigned char *buf = malloc(row * f->na);
    if (!buf) sbio_die("getInt: cannot allocate the interferogram buffer");
    /* fill value (1, 1) in the file's byte order */
    const unsigned char one[4] = {f->byteOrder == SB_MSB ? 0 : 1, f->byteOrder == SB_MSB ? 1 : 0,
                                  f->byteOrder == SB_MSB ? 0 : 1, f->byteOrder == SB_MSB ? 1 : 0};
    for (size_t k = 0; k < (size_t)f->nr * f->na; k++) memcpy(buf + 4 * k, one, 4);
    const char *src = v.nbands > 0 ? v.source : intFile;
    FILE *fp = fopen(src, "rb");
    if (!fp) sbio_die("getInt: cannot open %s", src);
    fseeko(fp, 0, SEEK_END);
    off_t size = ftello(fp);
    fseeko(fp, 0, SEEK_SET);
    size_t nLines = (size_t)size / row;
    if (nLines > (size_t)f->na) nLines = f->na;
    if (nLines && fread(buf, row, nLines, fp) != nLines) sbio_die("getInt: short read on %s", src);
    fclose(fp);
    f->data = buf;
}

static void *load_image(const char *image, const char *parKey, const sbio_rdf *r, const Args *a, sb_image *im,
                        int *vrtByteOrder)
{
    char *vrt = NULL;
    size_t L = strlen(image);
    if (L > 4 && strcmp(image + L - 4, ".vrt") == 0) vrt = strdup(image);
    else if (sbio_exists(suffixed(image, ".vrt"))) vrt = suffixed(image, ".vrt");
    if (!vrt) {
        if (sbio_rdf_get(r, parKey))
            sbio_die("%s: GrIMP .par image descriptions are not supported (the readOldPar reader is not part of the "
                     "reference tree); describe %s with a VRT sidecar", parKey, image);
        sbio_die("parseTrack: Missing %s and no vrt", parKey);
    }
    sbio_vrt v;
    if (!sbio_vrt_read(vrt, &v)) sbio_die("cannot parse VRT %s", vrt);
    const char *src = v.source[0] ? v.source : image;
    size_t sz;
    void *data = sbio_read_all(src, &sz);
    const size_t elem = a->floatFlag ? 8 : 4;
    if (sz < (size_t)v.nr * v.na * elem)
        sbio_die("%s holds %zu bytes, %d x %d samples need %zu", src, sz, v.na, v.nr, (size_t)v.nr * v.na * elem);
    im->data = data;
    im->nr = v.nr;
    im->na = v.na;
    im->sampleType = a->floatFlag ? SB_CFLOAT32 : SB_CINT16;
    im->onDevice = 0;
    if (v.byteOrder >= 0) *vrtByteOrder = v.byteOrder;
    free(vrt);
    return data;
}

int main(int argc, char **argv)
{
    sbio_tool = TOOL;
    Args a;
    read_args(argc, argv, &a);
    fprintf(stderr, "Using: %s\n", a.parFile);
    sbio_rdf *r = sbio_rdf_read(a.parFile);

    /* ---- parseTrack (Strack/parseTrack.c:13-212) */
    const char *image1 = sbio_rdf_get(r, "image1");
    const char *image2 = sbio_rdf_get(r, "image2");
    if (!image1) sbio_die("parseTrack: Missing image1");
    if (!image2) sbio_die("parseTrack: Missing image2");
    const char *outputfile = sbio_rdf_get(r, "outputfile");
    if (!outputfile) sbio_die("parseTrack: missing ouput file");
    sb_track_params p;
    memset(&p, 0, sizeof p);
    p.rStart = ival(r, "rstart", 1, 0);
    p.aStart = ival(r, "astart", 1, 0);
    p.deltaR = ival(r, "deltar", 1, 0);
    p.deltaA = ival(r, "deltaa", 1, 0);
    p.nR = ival(r, "nR", 1, 0);
    p.nA = ival(r, "nA", 1, 0);
    p.wR = ival(r, "wr", 1, 0);
    p.wA = ival(r, "wa", 1, 0);
    p.wRa = ival(r, "wra", 1, 0);
    p.wAa = ival(r, "waa", 1, 0);
    const int edgePad = ival(r, "edgepad", 0, 0);
    p.scaleFactor = ival(r, "scalefactor", 0, 1);
    p.edgePadR = ival(r, "edgeR", 0, edgePad);
    p.edgePadA = ival(r, "edgeA", 0, edgePad);
    p.navgR = ival(r, "navgR", 1, 0);
    p.navgA = ival(r, "navgA", 1, 0);
    p.rStart /= p.scaleFactor;
    p.aStart /= p.scaleFactor;
    p.deltaR /= p.scaleFactor;
    p.deltaA /= p.scaleFactor;
    p.noComplex = a.noComplex;
    p.hanningFlag = a.hanningFlag;
    p.maxTries = a.maxTries;
    p.checkAzFocus = a.checkAzFocus;
    p.gaussFlag = a.gaussFlag;
    p.azDefocusThresh = 1.8f;  /* Strack/strack.c:45 */

    /* ---- images */
    sb_image im1, im2;
    int vrtOrder = -1;
    void *d1 = load_image(image1, "image1par", r, &a, &im1, &vrtOrder);
    void *d2 = load_image(image2, "image2par", r, &a, &im2, &vrtOrder);
    int byteOrder = a.byteOrder;
    if (vrtOrder >= 0) byteOrder = vrtOrder;  /* the VRT overrides (strack.c:87) */
    im1.byteOrder = im2.byteOrder = a.floatFlag ? byteOrder : SB_MSB;

    /* ---- interferogram, geodat, baseline (strack.c:92-126) */
    sb_interferogram intf;
    memset(&intf, 0, sizeof intf);
#ifndef STRACKW
    const char *intFile = sbio_rdf_get(r, "intfile");
    if (intFile && !a.noComplex) {
        load_interferogram(intFile, &intf);
        p.intf = &intf;
    }
#endif
    const char *intGeodat = sbio_rdf_get(r, "intgeodat");
#ifndef STRACKW
    if (!intGeodat) sbio_die("getInt: Missing geodat filename");
#endif
    sb_baseline bl;
    memset(&bl, 0, sizeof bl);
    const char *baseParams = sbio_rdf_get(r, "baseparams");
    if (baseParams && !a.noComplex) {
        FILE *f = fopen(baseParams, "r");
        if (!f) sbio_die("parseBase: cannot open %s", baseParams);
        if (fscanf(f, "%lf%lf%lf%lf", &bl.Bn, &bl.Bp, &bl.dBn, &bl.dBp) != 4)
            sbio_die("parseBase -- Missing baseline at line: 1");
        fclose(f);
        if (bl.Bn != 0 || bl.Bp != 0 || bl.dBn != 0 || bl.dBp != 0)
            sbio_die("parseBase: a non-zero baseline needs the image geometry of GrIMP's geodat/par readers, "
                     "which are not part of the reference tree");
    }
    p.baseline = NULL;

    /* ---- initial offsets (parseInitialOffsets.c, readBothOffsetsStrack.c) */
    sb_offset_grid grid;
    const char *initShift = sbio_rdf_get(r, "initShift");
    char *initVrt = initShift ? suffixed(initShift, ".vrt") : NULL;
    if (initShift && sbio_exists(initVrt)) {
        /* readBothOffsetsStrackVrt (Strack/readBothOffsetsStrack.c:46-77): band 1
           the range offsets, band 2 the azimuth offsets, r0/a0/deltaR/deltaA metadata */
        p.polyShift = 0;
        sbio_vrt v;
        if (!sbio_vrt_read(initVrt, &v) || v.nbands < 2) sbio_die("Problem reading offsets from %s", initVrt);
        const char *m0 = sbio_vrt_meta(&v, "r0"), *m1 = sbio_vrt_meta(&v, "a0");
        const char *m2 = sbio_vrt_meta(&v, "deltaR"), *m3 = sbio_vrt_meta(&v, "deltaA");
        if (!m0 || !m1 || !m2 || !m3) sbio_die("%s lacks r0/a0/deltaR/deltaA", initVrt);
        if (!strstr(v.desc[0], "Range")) sbio_die("Problem reading range offsets from %s", initVrt);
        if (!strstr(v.desc[1], "Azimuth")) sbio_die("Problem reading azimuth offsets from %s", initVrt);
        grid.nr = v.nr;
        grid.na = v.na;
        grid.r0 = atoi(m0);
        grid.a0 = atoi(m1);
        grid.deltaR = (float)atof(m2);
        grid.deltaA = (float)atof(m3);
        grid.dr = sbio_vrt_read_float_band(&v, 0, (size_t)grid.nr * grid.na);
        grid.da = sbio_vrt_read_float_band(&v, 1, (size_t)grid.nr * grid.na);
        p.initOffsets = &grid;
    } else if (initShift) {
        p.polyShift = 0;
        double h[6];
        char *daFile = suffixed(initShift, ".da"), *drFile = suffixed(initShift, ".dr");
        char *datFile = suffixed(daFile, ".dat");
        if (!sbio_dat_read(datFile, h))
            sbio_die("readBothOffsetsStrack -- Missing image params at line: 1 of %s", datFile);
        grid.r0 = (int)h[0];
        grid.a0 = (int)h[1];
        grid.nr = (int)h[2];
        grid.na = (int)h[3];
        grid.deltaR = (float)h[4];
        grid.deltaA = (float)h[5];
        grid.da = sbio_read_floats(daFile, (size_t)grid.nr * grid.na, 1);
        grid.dr = sbio_read_floats(drFile, (size_t)grid.nr * grid.na, 1);
        p.initOffsets = &grid;
        /* polynomial coefficients stay zero (parseInitialOffsets.c:19-27) */
    } else {
        const char *polyFile = sbio_rdf_get(r, "initialoffsetfile");
        if (!polyFile) sbio_die("parseTrack: Missing initialoffsetfile");
        p.polyShift = 1;
        sbio_read_poly(polyFile, p.rShiftPoly, p.aShiftPoly);
    }

    /* ---- mask (getMask.c) */
    sb_mask mask;
    const char *maskFile = sbio_rdf_get(r, "maskfile");
    if (maskFile)
        sbio_die("maskfile: geodat masks need GrIMP's parseInputFile, which is not part of the reference tree; "
                 "use offsetmaskfile + offsetmaskdat");
    maskFile = sbio_rdf_get(r, "offsetmaskfile");
    const char *maskVrt = sbio_rdf_get(r, "offsetmaskvrt");
    if (maskFile || maskVrt) {
        double h[6];
        if (maskVrt) {
            sbio_vrt v;
            if (!sbio_vrt_read(maskVrt, &v)) sbio_die("getMaskVRT: Cannot open vrt %s", maskVrt);
            const char *m0 = sbio_vrt_meta(&v, "r0"), *m1 = sbio_vrt_meta(&v, "a0");
            const char *m2 = sbio_vrt_meta(&v, "deltaR"), *m3 = sbio_vrt_meta(&v, "deltaA");
            if (!m0 || !m1 || !m2 || !m3) sbio_die("getMaskVRT: %s lacks r0/a0/deltaR/deltaA", maskVrt);
            mask.r0 = atoi(m0);
            mask.a0 = atoi(m1);
            mask.nrl = atoi(m2);
            mask.nal = atoi(m3);
            mask.nr = v.nr;
            mask.na = v.na;
            maskFile = v.source;
        } else {
            const char *dat = sbio_rdf_get(r, "offsetmaskdat");
            if (!dat) sbio_die("getMask: Missing geodat filename");
            if (!sbio_dat_read(dat, h)) sbio_die("readOffsets -- Missing image parameters at line: 1 of %s", dat);
            mask.r0 = (int)h[0];
            mask.a0 = (int)h[1];
            mask.nr = (int)h[2];
            mask.na = (int)h[3];
            mask.nrl = (int)h[4];
            mask.nal = (int)h[5];
        }
        size_t sz;
        mask.mask = sbio_read_all(maskFile, &sz);
        if (sz < (size_t)mask.nr * mask.na) sbio_die("mask %s is shorter than %d x %d", maskFile, mask.na, mask.nr);
        p.mask = &mask;
    }

    /* ---- track */
    sb_context *ctx;
    int rc = sb_context_create(0, &ctx);
    if (rc != SB_OK) sbio_die("no usable CUDA device (status %d)", rc);
    const size_t n = (size_t)p.nR * p.nA;
    float *offR = malloc(n * 4), *offA = malloc(n * 4), *corr = malloc(n * 4), *azd = malloc(n * 4);
    uint8_t *type = malloc(n);
    sb_track_result res;
    memset(&res, 0, sizeof res);
    res.offR = offR;
    res.offA = offA;
    res.corr = corr;
    res.type = type;
#ifdef STRACKW
    res.azd = NULL;
    fprintf(stderr, "\nSPECKLE TRACKING\n");
    rc = sb_strackw(ctx, &p, &im1, &im2, &res);
#else
    res.azd = azd;
    fprintf(stderr, "\nSPECKLE TRACKING\n");
    rc = sb_strack(ctx, &p, &im1, &im2, &res);
#endif
    if (rc != SB_OK) sbio_die("%s", sb_last_error(ctx));
    float ms[4];
    sb_last_timing(ctx, ms);

    /* ---- outputs (sTrackOut.c:44-60, writeDatFile, writeVrt.c) */
    const int msb = byteOrder == SB_MSB;
    char *fR = suffixed(outputfile, ".dr"), *fA = suffixed(outputfile, ".da"), *fC = suffixed(outputfile, ".cc");
    char *fT = suffixed(outputfile, ".mt"), *fD = suffixed(outputfile, ".dat"), *fZ = suffixed(outputfile, ".azd");
    sbio_write_items(fR, offR, 4, n, msb);
    sbio_write_items(fA, offA, 4, n, msb);
    sbio_write_items(fC, corr, 4, n, msb);
#ifndef STRACKW
    sbio_write_items(fZ, azd, 4, n, msb);
#endif
    sbio_write_items(fT, type, 1, n, 0);
    FILE *fd = fopen(fD, "w");
    if (!fd) sbio_die("cannot create %s", fD);
    fprintf(fd, "%i %i %i %i %i %i\n", p.rStart * p.scaleFactor, p.aStart * p.scaleFactor, p.nR, p.nA,
            p.deltaR * p.scaleFactor, p.deltaA * p.scaleFactor);
#ifndef STRACKW
    {
        char *copy = strdup(image2);
        fprintf(fd, "%s %s/%s\n", intGeodat, dirname(copy), intGeodat);
        free(copy);
    }
#endif
    fclose(fd);
    char m[16][2][256];
    int nm = 0;
#define META(k, ...) (snprintf(m[nm][0], 256, "%s", k), snprintf(m[nm][1], 256, __VA_ARGS__), nm++)
    META("r0", "%i", p.rStart * p.scaleFactor);
    META("a0", "%i", p.aStart * p.scaleFactor);
    META("deltaA", "%i", p.deltaA * p.scaleFactor);
    META("deltaR", "%i", p.deltaR * p.scaleFactor);
    META("sigmaStreaks", "%f", 0.);
    META("sigmaRange", "%f", 0.);
    if (intGeodat) META("geo1", "%s", intGeodat);
    META("Image1", "%s", image1);
    META("Image2", "%s", image2);
    META("wR", "%i", p.wR);
    META("wA", "%i", p.wA);
    META("wRa", "%i", p.wRa);
    META("wAa", "%i", p.wAa);
    META("scaleFactor", "%i", p.scaleFactor);
    META("ByteOrder", "%s", msb ? "MSB" : "LSB");
    const char *meta[16][2];
    for (int k = 0; k < nm; k++) {
        meta[k][0] = m[k][0];
        meta[k][1] = m[k][1];
    }
    sbio_band bands[3] = {{fR, "RangeOffsets", "Float32", 4}, {fA, "AzimuthOffsets", "Float32", 4},
                          {fC, "Correlation", "Float32", 4}};
    sbio_band mt = {fT, "MatchType", "Byte", 1};
    char *fV = suffixed(outputfile, ".vrt"), *fMV = suffixed(outputfile, ".mt.vrt");
    sbio_vrt_write(fV, p.nR, p.nA, meta, nm, bands, 3, msb, 1);
    sbio_vrt_write(fMV, p.nR, p.nA, meta, nm - 1, &mt, 1, msb, 0);

    const double tot = (double)(res.nAttempted > 0 ? res.nAttempted : 1);
    fprintf(stderr,
            "Tot %lld, nMtch %lld %4.1f nCmpx %lld %4.1f nAmp %lld %4.1f (%lld - %lld) nFl %lld %4.1f "
            "GPU %.1f ms (h2d %.1f, kernels %.1f, d2h %.1f)\n",
            (long long)res.nAttempted, (long long)(res.nComplex + res.nAmp + res.nAmpL),
            100. * (res.nComplex + res.nAmp + res.nAmpL) / tot, (long long)res.nComplex, 100. * res.nComplex / tot,
            (long long)(res.nAmp + res.nAmpL), 100. * (res.nAmp + res.nAmpL) / tot, (long long)res.nAmp,
            (long long)res.nAmpL, (long long)res.nFail, 100. * res.nFail / tot, ms[0], ms[1], ms[2], ms[3]);
    sb_context_destroy(ctx);
    free(d1);
    free(d2);
    sbio_rdf_free(r);
    return 0;
}
