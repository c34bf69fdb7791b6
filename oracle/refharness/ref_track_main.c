/*
 * ref_track_main.c -- TEST INFRASTRUCTURE ONLY.  Runs the reference's own
 * speckleTrack() (Strack/speckleTrack.c:159-346), or corrTrackFast()
 * (Strackw/corrTrackFast.c:89-231) when built with -DREF_STRACKW, compiled
 * unmodified from the reference tree against the stand-ins in
 * oracle/refshim/, so the oracle can be checked against the reference's own
 * code.  It fills TrackParams the way strack.c/strackw.c and parseTrack.c do
 * (raw image files, no GDAL), runs the tracker, which writes its .dr .da .cc
 * .mt (.azd) files, and writes the baseline tables initPhaseCorrect computed
 * (<out>.tables: sinThetaD, cosThetaD, overRange as float64).
 *
 *   ref_strack|ref_strackw <parameter file>
 *
 * The parameter file holds "key value" lines (see oracle/refpin.py).
 */
#include <setjmp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef REF_STRACKW
#include "strackt.h"
void corrTrackFast(TrackParams *trackPar);
#else
#include "strack.h"
#endif

extern jmp_buf refshim_fail;
extern int refshim_fail_armed;
extern int refshim_label_connectivity;
#ifndef REF_STRACKW
extern double *sinThetaD, *cosThetaD, *overRange;
#endif

/* The VRT sidecar needs GDAL's metadata writer; the harness reads the raw
 * outputs, so the VRT is not written. */
void writeVrtFile(TrackParams *trackPar) { (void)trackPar; }

/* initial offset grid given in the parameter file (offsets file: dr then da,
 * float32 native, ona x onr each) */
static Offsets gOffsets;
static int gHaveOffsets = 0;

int readBothOffsetsStrackVrt(Offsets *offsets, char *vrtFile)
{
    (void)vrtFile;
    if (!gHaveOffsets) return FALSE;
    *offsets = gOffsets;
    return TRUE;
}

void readBothOffsetsStrack(Offsets *offsets)
{
    (void)offsets;
    error("readBothOffsetsStrack: the harness passes offsets through readBothOffsetsStrackVrt");
}

static float **rows_of(float *block, int na, int nr)
{
    float **r = (float **)malloc(sizeof(float *) * (size_t)na);
    for (int i = 0; i < na; i++) r[i] = block + (size_t)i * nr;
    return r;
}

static void *read_file(const char *path, size_t bytes)
{
    FILE *fp = fopen(path, "rb");
    if (!fp) { fprintf(stderr, "cannot open %s\n", path); exit(3); }
    void *buf = malloc(bytes ? bytes : 1);
    if (fread(buf, 1, bytes, fp) != bytes) { fprintf(stderr, "short read %s\n", path); exit(3); }
    fclose(fp);
    return buf;
}

static char *cat2(const char *a, const char *b)
{
    char *s = (char *)malloc(strlen(a) + strlen(b) + 1);
    strcpy(s, a);
    strcat(s, b);
    return s;
}

int main(int argc, char **argv)
{
    if (argc != 2) { fprintf(stderr, "usage: %s <parameter file>\n", argv[0]); return 1; }
    FILE *pf = fopen(argv[1], "r");
    if (!pf) { fprintf(stderr, "cannot open %s\n", argv[1]); return 1; }
    static TrackParams t; /* zero-initialised, as the reference's static defaults */
    char key[256], val[4096];
    char out[4096] = "", ofile[4096] = "", mfile[4096] = "";
    int onr = 0, ona = 0, mnr = 0, mna = 0;
    double or0 = 0, oa0 = 0, odr = 1, oda = 1;
    t.scaleFactor = 1;
    t.hanningFlag = TRUE;
    t.maxTries = 2;
    t.azDefocusThresh = 1.8f;
    t.floatFlag = TRUE;
    t.polyShift = TRUE;
    t.byteOrder = LSB;
    t.lambda = 0.0555;
    t.imageP1.H = 700000.0;
    t.imageP1.rn = 850000.0;
    t.imageP1.slpR = 2.33;
    t.latc = 70.0;
    t.intGeodat = "none";
    t.navgR = t.navgA = 1;
    while (fscanf(pf, "%255s %4095s", key, val) == 2) {
#define I(name) else if (!strcmp(key, #name)) t.name = atoi(val)
#define D(name) else if (!strcmp(key, #name)) t.name = atof(val)
        if (!strcmp(key, "image1")) t.imageFile1 = strdup(val);
        else if (!strcmp(key, "image2")) t.imageFile2 = strdup(val);
        else if (!strcmp(key, "out")) strcpy(out, val);
        else if (!strcmp(key, "na1")) t.imageP1.nSlpA = atoi(val);
        else if (!strcmp(key, "nr1")) t.imageP1.nSlpR = atoi(val);
        else if (!strcmp(key, "na2")) t.imageP2.nSlpA = atoi(val);
        else if (!strcmp(key, "nr2")) t.imageP2.nSlpR = atoi(val);
        else if (!strcmp(key, "H")) t.imageP1.H = atof(val);
        else if (!strcmp(key, "rn")) t.imageP1.rn = atof(val);
        else if (!strcmp(key, "slpR")) t.imageP1.slpR = atof(val);
        else if (!strcmp(key, "rpoly0")) t.rShiftPoly[0] = atof(val);
        else if (!strcmp(key, "rpoly1")) t.rShiftPoly[1] = atof(val);
        else if (!strcmp(key, "rpoly2")) t.rShiftPoly[2] = atof(val);
        else if (!strcmp(key, "apoly0")) t.aShiftPoly[0] = atof(val);
        else if (!strcmp(key, "apoly1")) t.aShiftPoly[1] = atof(val);
        else if (!strcmp(key, "apoly2")) t.aShiftPoly[2] = atof(val);
        else if (!strcmp(key, "ofile")) strcpy(ofile, val);
        else if (!strcmp(key, "onr")) onr = atoi(val);
        else if (!strcmp(key, "ona")) ona = atoi(val);
        else if (!strcmp(key, "or0")) or0 = atof(val);
        else if (!strcmp(key, "oa0")) oa0 = atof(val);
        else if (!strcmp(key, "odeltaR")) odr = atof(val);
        else if (!strcmp(key, "odeltaA")) oda = atof(val);
        else if (!strcmp(key, "mfile")) strcpy(mfile, val);
        else if (!strcmp(key, "mnr")) mnr = atoi(val);
        else if (!strcmp(key, "mna")) mna = atoi(val);
        else if (!strcmp(key, "mr0")) t.maskDat.r0 = atoi(val);
        else if (!strcmp(key, "ma0")) t.maskDat.a0 = atoi(val);
        else if (!strcmp(key, "mnrl")) t.maskDat.nrl = atoi(val);
        else if (!strcmp(key, "mnal")) t.maskDat.nal = atoi(val);
        else if (!strcmp(key, "azDefocusThresh")) t.azDefocusThresh = (float)atof(val);
        I(rStart); I(aStart); I(deltaR); I(deltaA); I(nR); I(nA); I(wR); I(wA); I(wRa); I(wAa);
        I(scaleFactor); I(noComplex); I(hanningFlag); I(maxTries); I(checkAzFocus); I(gaussFlag);
        I(floatFlag); I(byteOrder); I(polyShift); I(edgePadR); I(edgePadA); I(navgR); I(navgA);
        D(Bn); D(Bp); D(dBn); D(dBp); D(dBnQ); D(dBpQ); D(lambda); D(latc);
        else { fprintf(stderr, "unknown key %s\n", key); return 1; }
#undef I
#undef D
    }
    fclose(pf);
    t.outFileR = cat2(out, ".dr");
    t.outFileA = cat2(out, ".da");
    t.outFileC = cat2(out, ".cc");
    t.outFileT = cat2(out, ".mt");
    t.outFileD = cat2(out, ".dat");
    t.outFileAzDefocus = cat2(out, ".azd");
    t.vrtFile = cat2(out, ".vrt");
    t.MTvrtFile = cat2(out, ".mt.vrt");
    t.initOffsetsFile = cat2(out, ".init");
    if (ofile[0]) {
        float *blk = (float *)read_file(ofile, sizeof(float) * 2 * (size_t)ona * onr);
        gOffsets.nr = onr;
        gOffsets.na = ona;
        gOffsets.rO = or0;
        gOffsets.aO = oa0;
        gOffsets.deltaR = odr;
        gOffsets.deltaA = oda;
        gOffsets.dr = (void **)rows_of(blk, ona, onr);
        gOffsets.da = (void **)rows_of(blk + (size_t)ona * onr, ona, onr);
        gHaveOffsets = 1;
    }
    if (mfile[0]) {
        char *m = (char *)read_file(mfile, (size_t)mna * mnr);
        t.maskDat.nr = mnr;
        t.maskDat.na = mna;
        t.maskDat.mask = (char **)malloc(sizeof(char *) * (size_t)mna);
        for (int i = 0; i < mna; i++) t.maskDat.mask[i] = m + (size_t)i * mnr;
        t.maskFlag = TRUE;
    }
    /* the output grids (TrackParams results), as the tools' mains allocate them */
    float *g = (float *)calloc((size_t)4 * t.nA * t.nR, sizeof(float));
    t.offR = rows_of(g, t.nA, t.nR);
    t.offA = rows_of(g + (size_t)t.nA * t.nR, t.nA, t.nR);
    t.corr = rows_of(g + (size_t)2 * t.nA * t.nR, t.nA, t.nR);
    t.aZDefocus = rows_of(g + (size_t)3 * t.nA * t.nR, t.nA, t.nR);
    char *ty = (char *)calloc((size_t)t.nA * t.nR, 1);
    t.type = (char **)malloc(sizeof(char *) * (size_t)t.nA);
    for (int i = 0; i < t.nA; i++) t.type[i] = ty + (size_t)i * t.nR;
    refshim_fail_armed = 1;
    if (setjmp(refshim_fail)) return 2;
#ifdef REF_STRACKW
    corrTrackFast(&t);
#else
    speckleTrack(&t);
    if (sinThetaD && cosThetaD && overRange) {
        char *tp = cat2(out, ".tables");
        FILE *fp = fopen(tp, "wb");
        fwrite(sinThetaD, sizeof(double), (size_t)t.imageP1.nSlpR, fp);
        fwrite(cosThetaD, sizeof(double), (size_t)t.imageP1.nSlpR, fp);
        fwrite(overRange, sizeof(double), (size_t)t.imageP1.nSlpR, fp);
        fclose(fp);
    }
#endif
    printf("nComplex %d nAmp %d nAmpL %d nFail %d\n", t.nComplex, t.nAmp, t.nAmpL, t.nFail);
    return 0;
}
