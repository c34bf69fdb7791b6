/*
 * cullst_main.c -- the drop-in `cullst` command line (Cullst/cullst.c): same
 * flags, inputs <inbase>.{dat,dr,da,cc,mt} (or <inbase>.vrt + .mt.vrt),
 * optional ./offsets.mask, and outputs <outbase>.{dr,da,cc,mt,vrt,mt.vrt}
 * plus the sigmas <inbase>.{sr,sa}; the passes run on the GPU through sb_cull.
 *
 *   cullst [-useSim offsets -ignoreOffsets -islandThresh n -singleMT n -maxR r -maxA a -nGood n
 *           -boxSize n -sr n -sa n -corrThresh c] inbase outbase
 */
#define _GNU_SOURCE
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/speckle_b200.h"
#include "sbio.h"

extern const char *sbio_tool;

static void usage(void)
{
    sbio_die("cullst -useSim offsets -ignoreOffsets -islandThresh islandThresh -singleMT singleMT -maxR maxR -maxA "
             "maxA -nGood nGood -boxSize boxSize -sr sr -sa sa inbase outbase");
}

static char *suffixed(const char *base, const char *suf)
{
    char *s = malloc(strlen(base) + strlen(suf) + 1);
    strcpy(s, base);
    strcat(s, suf);
    return s;
}

int main(int argc, char **argv)
{
    sbio_tool = "cullst";
    /* ---- readArgs (cullst.c:123-358) */
    if (argc < 3 || argc > 21) usage();
    sb_cull_params p;
    memset(&p, 0, sizeof p);
    int sr = 2, sa = 8, boxSize = 9, nGood = 17, singleMT = -1, islandThresh = -1, ignoreOffsets = 0, useSim = 0;
    float maxA = 1.0f, maxR = .75f, corrThresh = 0.0f;
    const char *simBase = NULL;
    for (int i = 1; i <= argc - 3; i++) {
        const char *s = strchr(argv[i], '-');
        if (!s) usage();
        const char *nx = (i + 1 < argc) ? argv[i + 1] : "";
        if (strstr(s, "sr")) { sscanf(nx, "%i", &sr); i++; }
        else if (strstr(s, "sa")) { sscanf(nx, "%i", &sa); i++; }
        else if (strstr(s, "corrThresh")) {
            sscanf(nx, "%f", &corrThresh);
            if (corrThresh < 0 || corrThresh >= 1) { fprintf(stderr, "\n\ncoorThresh must be in interval (0,1)\n\n"); usage(); }
            i++;
        }
        else if (strstr(s, "boxSize")) { sscanf(nx, "%i", &boxSize); i++; }
        else if (strstr(s, "nGood")) { sscanf(nx, "%i", &nGood); i++; }
        else if (strstr(s, "singleMT")) {
            sscanf(nx, "%i", &singleMT);
            if (singleMT < 1 || singleMT > 3) { fprintf(stderr, "singleMT should be in range 0 to 3\n"); usage(); }
            i++;
        }
        else if (strstr(s, "maxA")) { sscanf(nx, "%f", &maxA); i++; }
        else if (strstr(s, "maxR")) { sscanf(nx, "%f", &maxR); i++; }
        else if (strstr(s, "islandThresh")) { sscanf(nx, "%i", &islandThresh); i++; }
        else if (strstr(s, "useSim")) { useSim = 1; simBase = nx; i++; }
        else if (strstr(s, "ignoreOffsets")) ignoreOffsets = 1;
        else usage();
    }
    const char *inBase = argv[argc - 2], *outBase = argv[argc - 1];

    /* ---- loadCullData (loadCullData.c:136-198) */
    int nr, na, r0, a0, deltaR, deltaA;
    float *offR, *offA, *corr;
    uint8_t *type;
    char *geo1 = NULL, *geo2 = NULL;
    const char *inVrt = suffixed(inBase, ".vrt");
    if (sbio_exists(inVrt)) {
        sbio_vrt v;
        if (!sbio_vrt_read(inVrt, &v) || v.nbands < 3) sbio_die("loadFromVRT: cannot read %s", inVrt);
        nr = v.nr;
        na = v.na;
        const char *m;
        r0 = (m = sbio_vrt_meta(&v, "r0")) ? atoi(m) : 0;
        a0 = (m = sbio_vrt_meta(&v, "a0")) ? atoi(m) : 0;
        deltaR = (m = sbio_vrt_meta(&v, "deltaR")) ? (int)atof(m) : 1;
        deltaA = (m = sbio_vrt_meta(&v, "deltaA")) ? (int)atof(m) : 1;
        const int msb = v.byteOrder != SB_LSB;
        offR = sbio_read_floats(v.sources[0], (size_t)nr * na, msb);
        offA = sbio_read_floats(v.sources[1], (size_t)nr * na, msb);
        corr = sbio_read_floats(v.sources[2], (size_t)nr * na, msb);
        sbio_vrt mv;
        const char *mtVrt = suffixed(inBase, ".mt.vrt");
        if (!sbio_vrt_read(mtVrt, &mv)) sbio_die("loadFromVRT: cannot read %s", mtVrt);
        size_t sz;
        type = sbio_read_all(mv.source, &sz);
    } else {
        double h[6];
        const char *dat = suffixed(inBase, ".dat");
        if (!sbio_dat_read(dat, h)) sbio_die("readOffsets -- Missing image parameters at line: 1 of %s", dat);
        r0 = (int)h[0]; a0 = (int)h[1]; nr = (int)h[2]; na = (int)h[3]; deltaR = (int)h[4]; deltaA = (int)h[5];
        FILE *f = fopen(dat, "r");
        char line[4096];
        if (fgets(line, sizeof line, f) && fgets(line, sizeof line, f) && strstr(line, "geodat")) {
            char g1[2048], g2[2048];
            if (sscanf(line, "%2047s %2047s", g1, g2) == 2) { geo1 = strdup(g1); geo2 = strdup(g2); }
        }
        fclose(f);
        const size_t n = (size_t)nr * na;
        offR = sbio_read_floats(suffixed(inBase, ".dr"), n, 1);
        offA = sbio_read_floats(suffixed(inBase, ".da"), n, 1);
        corr = sbio_read_floats(suffixed(inBase, ".cc"), n, 1);
        size_t sz;
        type = sbio_read_all(suffixed(inBase, ".mt"), &sz);
        if (sz < n) sbio_die("%s.mt is shorter than %d x %d", inBase, na, nr);
    }
    const size_t n = (size_t)nr * na;
    for (size_t k = 0; k < n; k++)  /* loadCullData.c:193-196, int compared as float */
        if (offA[k] < (float)(-SB_LARGEINT + 1)) type[k] = 0;

    /* ---- sim offsets (loadSimData reads the input's .dat for the size check) */
    float *simR = NULL, *simA = NULL;
    if (useSim) {
        simR = sbio_read_floats(suffixed(simBase, ".dr"), n, 1);
        simA = sbio_read_floats(suffixed(simBase, ".da"), n, 1);
    }
    /* ---- offsets.mask in the working directory (cullst.c:63-69) */
    uint8_t *mask = NULL;
    if (sbio_exists("offsets.mask") && !ignoreOffsets) {
        double h[6];
        if (!sbio_dat_read("offsets.dat", h)) sbio_die("readOffsets -- Missing image parameters in offsets.dat");
        if ((int)h[3] == na && (int)h[2] == nr) {
            size_t sz;
            mask = sbio_read_all("offsets.mask", &sz);
            if (sz < n) sbio_die("offsets.mask is shorter than the grid");
        } else {
            fprintf(stderr, "Ignoring mask because it is not the same size: regoffsets ?\n");
        }
    }
    p.nR = nr; p.nA = na; p.bR = boxSize; p.bA = boxSize; p.nGood = nGood; p.maxA = maxA; p.maxR = maxR;
    p.sR = sr; p.sA = sa; p.islandThresh = islandThresh; p.corrThresh = corrThresh; p.singleMT = singleMT;
    p.useSim = useSim; p.connectivity = 8; p.nCullPasses = 3;
    sb_cull_data d;
    memset(&d, 0, sizeof d);
    d.offR = offR; d.offA = offA; d.corr = corr; d.type = type; d.mask = mask; d.simR = simR; d.simA = simA;
    d.offRS = malloc(n * 4); d.offAS = malloc(n * 4); d.sigmaR = malloc(n * 4); d.sigmaA = malloc(n * 4);
    sb_context *ctx;
    int rc = sb_context_create(0, &ctx);
    if (rc != SB_OK) sbio_die("no usable CUDA device (status %d)", rc);
    rc = sb_cull(ctx, &p, &d);
    if (rc != SB_OK) sbio_die("%s", sb_last_error(ctx));
    float ms[4];
    sb_last_timing(ctx, ms);
    fprintf(stderr, "nCulled (last pass) %lld; killed %lld islands with a total of %lld pixels; GPU %.1f ms\n",
            (long long)d.nCulled, (long long)d.nIslands, (long long)d.nIslandPoints, ms[0]);

    /* ---- writeCullData (writeCullData.c:55-81): MSB, sigmas next to the input */
    sbio_write_items(suffixed(outBase, ".dr"), d.offRS, 4, n, 1);
    sbio_write_items(suffixed(outBase, ".da"), d.offAS, 4, n, 1);
    sbio_write_items(suffixed(inBase, ".sr"), d.sigmaR, 4, n, 1);
    sbio_write_items(suffixed(inBase, ".sa"), d.sigmaA, 4, n, 1);
    sbio_write_items(suffixed(outBase, ".cc"), corr, 4, n, 1);
    sbio_write_items(suffixed(outBase, ".mt"), type, 1, n, 0);
    char m[20][2][256];
    int nm = 0;
#define META(k, ...) (snprintf(m[nm][0], 256, "%s", k), snprintf(m[nm][1], 256, __VA_ARGS__), nm++)
    META("r0", "%i", r0);
    META("a0", "%i", a0);
    META("deltaA", "%i", deltaA);
    META("deltaR", "%i", deltaR);
    META("sigmaStreaks", "%f", 0.);
    META("sigmaRange", "%f", 0.);
    META("sR", "%i", sr);
    META("sA", "%i", sa);
    META("boxSize", "%i", boxSize);
    META("nGood", "%i", nGood);
    META("maxR", "%f", maxR);
    META("maxA", "%f", maxA);
    META("corrThresh", "%f", corrThresh);
    META("singleMT", "%i", singleMT);
    if (geo1 && geo2) { META("geo1", "%s", geo1); META("geo2", "%s", geo2); }
    META("ByteOrder", "%s", "MSB");
    const char *meta[20][2];
    for (int k = 0; k < nm; k++) { meta[k][0] = m[k][0]; meta[k][1] = m[k][1]; }
    char *fR = suffixed(outBase, ".dr"), *fA = suffixed(outBase, ".da"), *fSR = suffixed(inBase, ".sr");
    char *fSA = suffixed(inBase, ".sa"), *fC = suffixed(outBase, ".cc"), *fT = suffixed(outBase, ".mt");
    sbio_band bands[5] = {{fR, "RangeOffsets", "Float32", 4}, {fA, "AzimuthOffsets", "Float32", 4},
                          {fSR, "RangeSigma", "Float32", 4}, {fSA, "AzimuthSigma", "Float32", 4},
                          {fC, "Correlation", "Float32", 4}};
    sbio_vrt_write(suffixed(outBase, ".vrt"), nr, na, meta, nm, bands, 5, 1, 1);
    sbio_band mt = {fT, "MatchType", "Byte", 1};
    sbio_vrt_write(suffixed(fT, ".vrt"), nr, na, meta, nm - 1, &mt, 1, 1, 0);
    sb_context_destroy(ctx);
    return 0;
}
