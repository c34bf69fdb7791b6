/*
 * unwrapSource/unWrap/unwrapInclude.h -- TEST INFRASTRUCTURE ONLY.  The types
 * and mask bits of GrIMP's unwrapper that Cullst/cullIslands.c uses, and its
 * connected-component labeller labelRegions (not part of the reference tree).
 * Assumed semantics (the same assumption as the oracle's restatement): pixels
 * whose mask has REGION set are labelled 1..K in order of first appearance in
 * a row-major scan, 8-connected (4 with refshim_label_connectivity = 4); every
 * other pixel gets LARGEINT.
 */
#ifndef REFSHIM_UNWRAPINCLUDE_H
#define REFSHIM_UNWRAPINCLUDE_H
#include <stdint.h>

#define VALIDPIXEL 0x1
#define REGION 0x2
#define validPixel(a) (((a) & VALIDPIXEL) ? TRUE : FALSE)

typedef struct {
    float **phase;
    int32_t rangeSize, azimuthSize;
    char **bCuts;
    int32_t **labels;
} unwrapImageStructure;

typedef struct {
    int32_t nH, nB;      /* hole and border pixel counts */
    int32_t cH, cB;      /* fill counters */
    int32_t *xb, *yb;    /* border pixels */
    int32_t *xh, *yh;    /* hole pixels */
} hole;

extern int refshim_label_connectivity;
void labelRegions(unwrapImageStructure *uw);
#endif
