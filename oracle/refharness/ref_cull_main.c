/*
 * ref_cull_main.c -- TEST INFRASTRUCTURE ONLY.  Runs the reference's own cull
 * passes (Cullst/cullSTData.c, cullStats.c, cullSmooth.c, cullIslands.c),
 * compiled unmodified against oracle/refshim/, in the order of cullst's main
 * (Cullst/cullst.c:36-101).  The main itself is compiled in this translation
 * unit under another name so that its addSubtractSimOffsets (static, with the
 * file's own LARGEINT of -2e9) is the one applied; the file loaders and the
 * writer it calls are not used (the harness reads and writes raw arrays).
 *
 *   ref_cull <parameter file>
 *
 * Inputs: <in>.offR .offA .corr (float32) .type (uint8) [.mask (uint8)]
 * [.simR .simA (float32)], native order, nA x nR.  Outputs: <out>.offR .offA
 * .type .offRS .offAS .sigmaR .sigmaA.
 */
#include <setjmp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define main reference_cullst_main
#include "speckleSource/Cullst/cullst.c"
#undef main

extern jmp_buf refshim_fail;
extern int refshim_fail_armed;
extern int refshim_label_connectivity;

/* cullst.c's main refers to these; the harness never calls that main */
void GDALAllRegister(void) {}
void loadCullData(CullParams *cullPar) { (void)cullPar; }
void loadSimData(CullParams *cullPar) { (void)cullPar; }
int32_t loadCullMask(CullParams *cullPar) { (void)cullPar; return FALSE; }
void writeCullData(CullParams *cullPar) { (void)cullPar; }

static float **fmat(float *blk, int na, int nr)
{
    float **r = (float **)malloc(sizeof(float *) * (size_t)na);
    for (int i = 0; i < na; i++) r[i] = blk + (size_t)i * nr;
    return r;
}

static void *slurp(const char *base, const char *ext, size_t bytes)
{
    char path[4200];
    snprintf(path, sizeof path, "%s%s", base, ext);
    FILE *fp = fopen(path, "rb");
    if (!fp) return NULL;
    void *b = malloc(bytes);
    if (fread(b, 1, bytes, fp) != bytes) { fprintf(stderr, "short read %s\n", path); exit(3); }
    fclose(fp);
    return b;
}

static void spill(const char *base, const char *ext, const void *p, size_t bytes)
{
    char path[4200];
    snprintf(path, sizeof path, "%s%s", base, ext);
    FILE *fp = fopen(path, "wb");
    fwrite(p, 1, bytes, fp);
    fclose(fp);
}

int main(int argc, char **argv)
{
    if (argc != 2) { fprintf(stderr, "usage: %s <parameter file>\n", argv[0]); return 1; }
    FILE *pf = fopen(argv[1], "r");
    if (!pf) return 1;
    static CullParams c;
    char key[256], val[4096], in[4096] = "", out[4096] = "";
    int passes = 3;
    while (fscanf(pf, "%255s %4095s", key, val) == 2) {
        if (!strcmp(key, "in")) strcpy(in, val);
        else if (!strcmp(key, "out")) strcpy(out, val);
        else if (!strcmp(key, "nR")) c.nR = atoi(val);
        else if (!strcmp(key, "nA")) c.nA = atoi(val);
        else if (!strcmp(key, "bR")) c.bR = atoi(val);
        else if (!strcmp(key, "bA")) c.bA = atoi(val);
        else if (!strcmp(key, "nGood")) c.nGood = atoi(val);
        else if (!strcmp(key, "maxA")) c.maxA = (float)atof(val);
        else if (!strcmp(key, "maxR")) c.maxR = (float)atof(val);
        else if (!strcmp(key, "sR")) c.sR = atoi(val);
        else if (!strcmp(key, "sA")) c.sA = atoi(val);
        else if (!strcmp(key, "islandThresh")) c.islandThresh = atoi(val);
        else if (!strcmp(key, "corrThresh")) c.corrThresh = (float)atof(val);
        else if (!strcmp(key, "singleMT")) c.singleMT = atoi(val);
        else if (!strcmp(key, "useSim")) c.useSim = atoi(val);
        else if (!strcmp(key, "connectivity")) refshim_label_connectivity = atoi(val);
        else if (!strcmp(key, "passes")) passes = atoi(val);
        else { fprintf(stderr, "unknown key %s\n", key); return 1; }
    }
    fclose(pf);
    const size_t n = (size_t)c.nA * c.nR;
    c.offR = fmat((float *)slurp(in, ".offR", 4 * n), c.nA, c.nR);
    c.offA = fmat((float *)slurp(in, ".offA", 4 * n), c.nA, c.nR);
    c.corr = fmat((float *)slurp(in, ".corr", 4 * n), c.nA, c.nR);
    char *ty = (char *)slurp(in, ".type", n);
    c.type = (char **)malloc(sizeof(char *) * (size_t)c.nA);
    for (int i = 0; i < c.nA; i++) c.type[i] = ty + (size_t)i * c.nR;
    char *mk = (char *)slurp(in, ".mask", n);
    c.maskFlag = mk != NULL;
    if (mk) {
        c.mask = (char **)malloc(sizeof(char *) * (size_t)c.nA);
        for (int i = 0; i < c.nA; i++) c.mask[i] = mk + (size_t)i * c.nR;
    }
    if (c.useSim) {
        c.offSimR = fmat((float *)slurp(in, ".simR", 4 * n), c.nA, c.nR);
        c.offSimA = fmat((float *)slurp(in, ".simA", 4 * n), c.nA, c.nR);
    }
    c.offRS = fmat((float *)calloc(n, 4), c.nA, c.nR);
    c.offAS = fmat((float *)calloc(n, 4), c.nA, c.nR);
    c.sigmaR = fmat((float *)calloc(n, 4), c.nA, c.nR);
    c.sigmaA = fmat((float *)calloc(n, 4), c.nA, c.nR);
    refshim_fail_armed = 1;
    if (setjmp(refshim_fail)) return 2;
    /* cullst.c:55-101 */
    if (c.useSim == TRUE) addSubtractSimOffsets(&c, -1.0);
    for (int k = 0; k < passes; k++) cullSTData(&c);
    cullStats(&c);
    if (c.useSim == TRUE) addSubtractSimOffsets(&c, 1.0);
    cullSmooth(&c);
    if (c.islandThresh > 0) cullIslands(&c);
    spill(out, ".offR", c.offR[0], 4 * n);
    spill(out, ".offA", c.offA[0], 4 * n);
    spill(out, ".type", c.type[0], n);
    spill(out, ".offRS", c.offRS[0], 4 * n);
    spill(out, ".offAS", c.offAS[0], 4 * n);
    spill(out, ".sigmaR", c.sigmaR[0], 4 * n);
    spill(out, ".sigmaA", c.sigmaA[0], 4 * n);
    return 0;
}
