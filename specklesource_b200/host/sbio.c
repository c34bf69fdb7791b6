/*
 * sbio.c -- host-side file formats of the drop-in tools (see sbio.h).
 * The RDF reader follows the keys of Strack/parseTrack.c (the rdfSource
 * grammar itself is not in the reference tree; this reader accepts
 * "key [(unit)] = value" with '!' or '#' comments, keys case-insensitive).
 */
#define _GNU_SOURCE
#include "sbio.h"

#include <ctype.h>
#include <libgen.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>
#include <unistd.h>

const char *sbio_tool = "speckle";

void sbio_die(const char *fmt, ...)
{
    va_list ap;
    fprintf(stderr, "%s: ", sbio_tool);
    va_start(ap, fmt);
    vfprintf(stderr, fmt, ap);
    va_end(ap);
    fprintf(stderr, "\n");
    exit(1);
}

/* ------------------------------------------------------------------ RDF */

struct sbio_rdf {
    int n;
    char **key;
    char **val;
};

static char *trim(char *s)
{
    while (*s && isspace((unsigned char)*s)) s++;
    char *e = s + strlen(s);
    while (e > s && isspace((unsigned char)e[-1])) *--e = '\0';
    return s;
}

sbio_rdf *sbio_rdf_read(const char *path)
{
    FILE *f = fopen(path, "r");
    if (!f) sbio_die("cannot open parameter file %s", path);
    sbio_rdf *r = calloc(1, sizeof(*r));
    char line[8192];
    while (fgets(line, sizeof line, f)) {
        char *c = strpbrk(line, "!#");
        if (c) *c = '\0';
        char *eq = strchr(line, '=');
        if (!eq) continue;
        *eq = '\0';
        char *k = line, *v = trim(eq + 1);
        char *paren = strchr(k, '(');
        if (paren) *paren = '\0';
        k = trim(k);
        if (!*k) continue;
        r->key = realloc(r->key, sizeof(char *) * (r->n + 1));
        r->val = realloc(r->val, sizeof(char *) * (r->n + 1));
        r->key[r->n] = strdup(k);
        r->val[r->n] = strdup(v);
        r->n++;
    }
    fclose(f);
    return r;
}

const char *sbio_rdf_get(const sbio_rdf *r, const char *key)
{
    for (int i = r->n - 1; i >= 0; i--)
        if (strcasecmp(r->key[i], key) == 0) return r->val[i];
    return NULL;
}

void sbio_rdf_free(sbio_rdf *r)
{
    if (!r) return;
    for (int i = 0; i < r->n; i++) {
        free(r->key[i]);
        free(r->val[i]);
    }
    free(r->key);
    free(r->val);
    free(r);
}

/* ------------------------------------------------------------------ files */

int sbio_exists(const char *path) { return path && access(path, F_OK) == 0; }

void *sbio_read_all(const char *path, size_t *size)
{
    FILE *f = fopen(path, "rb");
    if (!f) sbio_die("cannot open %s", path);
    fseeko(f, 0, SEEK_END);
    off_t n = ftello(f);
    fseeko(f, 0, SEEK_SET);
    void *buf = malloc(n > 0 ? (size_t)n : 1);
    if (!buf) sbio_die("out of memory reading %s", path);
    if (n > 0 && fread(buf, 1, (size_t)n, f) != (size_t)n) sbio_die("short read on %s", path);
    fclose(f);
    *size = (size_t)n;
    return buf;
}

static void swap_items(unsigned char *p, size_t size, size_t n)
{
    if (size == 1) return;
    for (size_t k = 0; k < n; k++, p += size)
        for (size_t b = 0; b < size / 2; b++) {
            unsigned char t = p[b];
            p[b] = p[size - 1 - b];
            p[size - 1 - b] = t;
        }
}

void sbio_write_items(const char *path, const void *data, size_t size, size_t n, int msb)
{
    FILE *f = fopen(path, "wb");
    if (!f) sbio_die("cannot create %s", path);
    const size_t chunk = 1 << 20;
    unsigned char *tmp = malloc(chunk * size);
    for (size_t k = 0; k < n; k += chunk) {
        size_t m = n - k < chunk ? n - k : chunk;
        memcpy(tmp, (const unsigned char *)data + k * size, m * size);
        if (msb) swap_items(tmp, size, m);
        if (fwrite(tmp, size, m, f) != m) sbio_die("write error on %s", path);
    }
    free(tmp);
    fclose(f);
}

float *sbio_read_floats(const char *path, size_t n, int msb)
{
    size_t sz;
    float *v = sbio_read_all(path, &sz);
    if (sz < n * sizeof(float)) sbio_die("%s holds %zu bytes, expected %zu", path, sz, n * sizeof(float));
    if (msb) swap_items((unsigned char *)v, 4, n);
    return v;
}

/* ------------------------------------------------------------------ VRT */

static const char *attr(const char *tag, const char *name, char *out, size_t cap)
{
    char pat[64];
    snprintf(pat, sizeof pat, "%s=\"", name);
    const char *p = strcasestr(tag, pat);
    if (!p) return NULL;
    p += strlen(pat);
    size_t k = 0;
    while (*p && *p != '"' && k + 1 < cap) out[k++] = *p++;
    out[k] = '\0';
    return out;
}

static const char *element(const char *txt, const char *name, char *out, size_t cap)
{
    char open[64];
    snprintf(open, sizeof open, "<%s", name);
    const char *p = strcasestr(txt, open);
    if (!p) return NULL;
    p = strchr(p, '>');
    if (!p) return NULL;
    p++;
    size_t k = 0;
    while (*p && *p != '<' && k + 1 < cap) out[k++] = *p++;
    out[k] = '\0';
    char *t = trim(out);
    memmove(out, t, strlen(t) + 1);
    return out;
}

int sbio_vrt_read(const char *path, sbio_vrt *v)
{
    memset(v, 0, sizeof(*v));
    v->byteOrder = -1;
    v->sampleType = -1;
    size_t sz;
    char *txt = sbio_read_all(path, &sz);
    txt = realloc(txt, sz + 1);
    txt[sz] = '\0';
    char buf[4096];
    const char *ds = strcasestr(txt, "<VRTDataset");
    if (!ds) {
        free(txt);
        return 0;
    }
    if (!attr(ds, "rasterXSize", buf, sizeof buf)) {
        free(txt);
        return 0;
    }
    v->nr = atoi(buf);
    attr(ds, "rasterYSize", buf, sizeof buf);
    v->na = atoi(buf);
    const char *band = strcasestr(txt, "<VRTRasterBand");
    if (band && attr(band, "dataType", buf, sizeof buf)) {
        if (strcasecmp(buf, "CFloat32") == 0) v->sampleType = SB_CFLOAT32;
        else if (strcasecmp(buf, "CInt16") == 0) v->sampleType = SB_CINT16;
    }
    if (band && element(band, "ByteOrder", buf, sizeof buf))
        v->byteOrder = strcasecmp(buf, "MSB") == 0 ? SB_MSB : SB_LSB;
    for (const char *b = band; b && v->nbands < 8; b = strcasestr(b + 1, "<VRTRasterBand")) {
        if (!element(b, "SourceFilename", buf, sizeof buf)) continue;
        /* per-band facts, looked up only inside this band's element */
        const char *end = strcasestr(b, "</VRTRasterBand>");
        size_t blen = end ? (size_t)(end - b) : strlen(b);
        char *bb = strndup(b, blen);
        char tmp[256];
        const int k = v->nbands;
        v->desc[k][0] = '\0';
        if (element(bb, "Description", tmp, sizeof tmp)) snprintf(v->desc[k], 256, "%s", tmp);
        v->bandMSB[k] = element(bb, "ByteOrder", tmp, sizeof tmp) && strcasecmp(tmp, "MSB") == 0;
        v->offset[k] = element(bb, "ImageOffset", tmp, sizeof tmp) ? atoll(tmp) : 0;
        free(bb);
        const char *tag = strcasestr(b, "<SourceFilename");
        char rel[16] = "";
        attr(tag, "relativeToVRT", rel, sizeof rel);
        char *dst = v->sources[v->nbands++];
        if (buf[0] != '/' && strcmp(rel, "0") != 0) {
            char *copy = strdup(path);
            snprintf(dst, 4096, "%s/%s", dirname(copy), buf);
            free(copy);
        } else {
            snprintf(dst, 4096, "%s", buf);
        }
    }
    if (v->nbands > 0) snprintf(v->source, sizeof v->source, "%s", v->sources[0]);
    /* <MDI key="...">value</MDI> */
    const char *p = txt;
    while (v->nmeta < 64 && (p = strcasestr(p, "<MDI"))) {
        char key[256], val[256];
        if (attr(p, "key", key, sizeof key) && element(p, "MDI", val, sizeof val)) {
            snprintf(v->meta[v->nmeta][0], 256, "%s", key);
            snprintf(v->meta[v->nmeta][1], 256, "%s", val);
            v->nmeta++;
        }
        p += 4;
    }
    free(txt);
    return 1;
}

float *sbio_vrt_read_float_band(const sbio_vrt *v, int b, size_t n)
{
    if (b < 0 || b >= v->nbands) sbio_die("VRT has no band %d", b + 1);
    size_t sz;
    unsigned char *all = sbio_read_all(v->sources[b], &sz);
    const size_t off = (size_t)v->offset[b];
    if (sz < off + n * 4) sbio_die("%s holds %zu bytes, band needs %zu", v->sources[b], sz, off + n * 4);
    float *out = malloc(n * sizeof(float));
    memcpy(out, all + off, n * sizeof(float));
    free(all);
    if (v->bandMSB[b]) swap_items((unsigned char *)out, 4, n);
    return out;
}

const char *sbio_vrt_meta(const sbio_vrt *v, const char *key)
{
    for (int i = 0; i < v->nmeta; i++)
        if (strcmp(v->meta[i][0], key) == 0) return v->meta[i][1];
    return NULL;
}

void sbio_vrt_write(const char *path, int nr, int na, const char *const meta[][2], int nmeta,
                    const sbio_band *bands, int nbands, int msb, int withNoData)
{
    FILE *f = fopen(path, "w");
    if (!f) sbio_die("cannot create %s", path);
    fprintf(f, "<VRTDataset rasterXSize=\"%d\" rasterYSize=\"%d\">\n", nr, na);
    if (nmeta > 0) {
        fprintf(f, "  <Metadata>\n");
        for (int i = 0; i < nmeta; i++) fprintf(f, "    <MDI key=\"%s\">%s</MDI>\n", meta[i][0], meta[i][1]);
        fprintf(f, "  </Metadata>\n");
    }
    for (int b = 0; b < nbands; b++) {
        char *copy = strdup(bands[b].file);
        fprintf(f, "  <VRTRasterBand dataType=\"%s\" band=\"%d\" subClass=\"VRTRawRasterBand\">\n", bands[b].type,
                b + 1);
        fprintf(f, "    <Description>%s</Description>\n", bands[b].name);
        if (withNoData) fprintf(f, "    <NoDataValue>-2e9</NoDataValue>\n");
        fprintf(f, "    <SourceFilename relativeToVRT=\"1\">%s</SourceFilename>\n", basename(copy));
        fprintf(f, "    <ImageOffset>0</ImageOffset>\n    <PixelOffset>%d</PixelOffset>\n", bands[b].size);
        fprintf(f, "    <LineOffset>%lld</LineOffset>\n", (long long)nr * bands[b].size);
        if (bands[b].size > 1) fprintf(f, "    <ByteOrder>%s</ByteOrder>\n", msb ? "MSB" : "LSB");
        fprintf(f, "  </VRTRasterBand>\n");
        free(copy);
    }
    fprintf(f, "</VRTDataset>\n");
    fclose(f);
}

/* ------------------------------------------------------------------ .dat */

int sbio_dat_read(const char *path, double v[6])
{
    FILE *f = fopen(path, "r");
    if (!f) return 0;
    char line[4096];
    int ok = 0;
    while (fgets(line, sizeof line, f)) {
        char *t = trim(line);
        if (!*t || *t == ';' || *t == '#') continue;
        ok = sscanf(t, "%lf %lf %lf %lf %lf %lf", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5]) == 6;
        break;
    }
    fclose(f);
    return ok;
}

/* ------------------------------------------------------------------ polynomial */

void sbio_read_poly(const char *path, double r[3], double a[3])
{
    FILE *f = fopen(path, "r");
    if (!f) sbio_die("parseInitialOffsets: cannot open %s", path);
    char line[4096];
    int rd = 0, ad = 0;
    while (fgets(line, sizeof line, f)) {
        char *p;
        if ((p = strstr(line, "range_offset_polynomial:"))) {
            if (sscanf(strchr(p, ':') + 1, "%lf%lf%lf", &r[0], &r[1], &r[2]) != 3)
                sbio_die("parseInitialOffsets: missing range parameter %s", p);
            rd = 1;
        } else if ((p = strstr(line, "azimuth_offset_polynomial:"))) {
            if (sscanf(strchr(p, ':') + 1, "%lf%lf%lf", &a[0], &a[1], &a[2]) != 3)
                sbio_die("parseInitialOffsets: missing azimuth parameter %s", p);
            ad = 1;
        }
    }
    fclose(f);
    if (!rd || !ad) sbio_die("parseInitialOffsets: missing polynomial in %s", path);
}
