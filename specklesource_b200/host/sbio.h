/*
 * sbio.h -- host-side file formats of the drop-in command-line tools:
 * RDF parameter files, raw big-endian rasters, .dat headers, minimal GDAL
 * VRT sidecars, initial-offset polynomials and offset grids.
 */
#ifndef SBIO_H
#define SBIO_H

#include <stddef.h>
#include <stdint.h>

#include "../../include/speckle_b200.h"

/* Prints "tool: message" to stderr and exits with status 1 (the reference's
 * clib error() also ends the process). */
void sbio_die(const char *fmt, ...);

/* ---- RDF parameter files: "key [(unit)] = value [! comment]" per line. */
typedef struct sbio_rdf sbio_rdf;
sbio_rdf *sbio_rdf_read(const char *path);
/* Value of key (case-insensitive), or NULL. */
const char *sbio_rdf_get(const sbio_rdf *r, const char *key);
void sbio_rdf_free(sbio_rdf *r);

/* ---- files */
int sbio_exists(const char *path);
/* Whole file into memory; *size gets the byte count. */
void *sbio_read_all(const char *path, size_t *size);
/* Writes n items of `size` bytes, swapping each item's bytes when msb != 0. */
void sbio_write_items(const char *path, const void *data, size_t size, size_t n, int msb);
/* Reads n float32 values, swapping when msb != 0. */
float *sbio_read_floats(const char *path, size_t n, int msb);

/* ---- minimal GDAL VRT: raster size, byte order, data type, source file of band 1 */
typedef struct {
    int nr, na;
    int byteOrder;      /* SB_MSB, SB_LSB, or -1 when not stated */
    int sampleType;     /* SB_CFLOAT32, SB_CINT16, or -1 (Float32/Byte bands) */
    char source[4096];  /* path of band 1's raw file (resolved relative to the VRT) */
    char sources[8][4096]; /* every band's raw file, resolved the same way */
    char desc[8][256];     /* every band's <Description> ("" when absent) */
    int bandMSB[8];        /* every band's ByteOrder (1: MSB; 0: LSB or not stated) */
    long long offset[8];   /* every band's ImageOffset in bytes */
    int nbands;
    char meta[64][2][256];
    int nmeta;
} sbio_vrt;
int sbio_vrt_read(const char *path, sbio_vrt *v);
/* Reads band b (float32) of a VRT into n floats, honouring its byte order and
 * image offset. */
float *sbio_vrt_read_float_band(const sbio_vrt *v, int b, size_t n);
const char *sbio_vrt_meta(const sbio_vrt *v, const char *key);

typedef struct {
    const char *file;   /* raw file name (written relative to the VRT) */
    const char *name;   /* band description */
    const char *type;   /* "Float32" or "Byte" */
    int size;           /* bytes per pixel */
} sbio_band;
/* Writes a VRT of raw bands; nodata < 0 adds <NoDataValue>-2e9</NoDataValue>. */
void sbio_vrt_write(const char *path, int nr, int na, const char *const meta[][2], int nmeta,
                    const sbio_band *bands, int nbands, int msb, int withNoData);

/* ---- .dat header "r0 a0 nr na deltaR deltaA" */
int sbio_dat_read(const char *path, double v[6]);

/* ---- initial offset polynomials (parseInitialOffsets.c:11-64) */
void sbio_read_poly(const char *path, double r[3], double a[3]);

#endif
