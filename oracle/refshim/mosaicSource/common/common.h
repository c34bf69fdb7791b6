/*
 * mosaicSource/common/common.h -- TEST INFRASTRUCTURE ONLY.  Stand-in for
 * GrIMP's mosaicSource common header (not part of the reference tree): the
 * fields of SARData and Offsets that the reference's hot-path sources read,
 * plus the helpers they call.  Field names follow their uses in
 * Strack/speckleTrack.c and Strackw/corrTrackFast.c.
 */
#ifndef REFSHIM_COMMON_H
#define REFSHIM_COMMON_H
#include <stdint.h>
#include <stdio.h>

#include "clib/standard.h"

/* SLC image parameters (the fields the tracking code reads) */
typedef struct {
    int32_t nSlpR, nSlpA; /* image size in range / azimuth samples */
    double H;             /* platform altitude (m) */
    double rn;            /* near range (m) */
    double slpR;          /* range sample spacing (m) */
    double slpA;
} SARData;

/* Offset grid of a prior match (readBothOffsetsStrack) */
typedef struct {
    char *file, *rFile;
    char *vrtFile;
    int32_t nr, na;
    double rO, aO;
    double deltaR, deltaA;
    void **dr;
    void **da;
    void **sr;
    void **sa;
} Offsets;

/* dictionary node of GrIMP's VRT metadata (only passed around) */
typedef struct dictNodeType dictNode;

#define EMINOR 6356.7523
#define EMAJOR 6378.137
/* radius (km) of the ellipsoid at geodetic latitude lat (rad) */
double earthRadius(double lat, double eMinor, double eMajor);
/* bilinear interpolation of a float grid at (x, y) with no-data handling
 * (mosaicSource, absent): values <= minvalue are no data, noData is returned
 * outside the grid or where every neighbour is no data */
float bilinearInterp(float **image, double x, double y, int32_t nx, int32_t ny, float minvalue, float noData);
char *appendSuff(char *file, char *suffix, char *buf);

#endif
