/*
 * clib/standard.h -- TEST INFRASTRUCTURE ONLY.  Stand-in for GrIMP's clib
 * header, which is not part of the reference tree, so that the reference's
 * own hot-path sources compile here as a parity reference (oracle/_ref).
 * Only what those sources use is declared; the values are the ones their
 * outputs imply (LARGEINT from the -2e9 no-data of Strack/writeVrt.c:69).
 */
#ifndef REFSHIM_CLIB_STANDARD_H
#define REFSHIM_CLIB_STANDARD_H
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <sys/types.h>

#define TRUE 1
#define FALSE 0
#define LARGEINT 2000000000
#ifndef PI
#define PI 3.14159265358979323846
#endif
#define DTOR (PI / 180.0)
#define RTOD (180.0 / PI)
#ifndef min
#define min(a, b) (((a) < (b)) ? (a) : (b))
#endif
#ifndef max
#define max(a, b) (((a) > (b)) ? (a) : (b))
#endif

/* element kinds for the byte-swapping readers and writers */
#define BYTEFLAG 1
#define INT16FLAG 2
#define INT32FLAG 3
#define FLOAT32FLAG 4
#define FLOAT64FLAG 5

/* Prints the message and exits, as clib's error() does. */
void error(char *fmt, ...);
FILE *openInputFile(char *file);
FILE *openOutputFile(char *file);
/* fread/fwrite of big-endian files: elements of `size` bytes are byte-swapped */
size_t freadBS(void *ptr, size_t size, size_t nitems, FILE *fp, int32_t flags);
size_t fwriteBS(void *ptr, size_t size, size_t nitems, FILE *fp, int32_t flags);

#endif
