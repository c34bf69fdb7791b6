/*
 * speckle_b200.h -- C ABI of the B200 (sm_100a) speckle-tracking library.
 *
 * The library re-implements the hot path of GrIMP's speckleSource:
 *   strack  (Strack/speckleTrack.c)  -> sb_strack()
 *   strackw (Strackw/corrTrackFast.c) -> sb_strackw()
 *   cullst  (Cullst/cull*.c)          -> sb_cull() and the four per-pass calls
 * Every entry point takes plain pointers, sizes and structs of plain values.
 * Nothing here depends on PyTorch or on any C++ type.
 *
 * Conventions
 *   - Return value: SB_OK (0) or a negative SB_ERR_* code.  The library never
 *     exits the process; sb_last_error() gives a one-line reason.
 *   - Grids are row-major nA rows (azimuth) x nR columns (range).
 *   - Per-point failures stay in-band exactly as in the reference:
 *     offsets = -SB_LARGEINT (-2e9), corr = 0 or the last correlation tried,
 *     type = SB_BAD (0).
 *   - A context is bound to one CUDA device and is not thread-safe; use one
 *     context per host thread.  Work is issued on the context's own stream.
 */
#ifndef SPECKLE_B200_H
#define SPECKLE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SB_ABI_VERSION 2

/* Status codes. */
#define SB_OK 0
#define SB_ERR_ARG (-1)         /* invalid argument or parameter combination */
#define SB_ERR_CUDA (-2)        /* a CUDA call failed */
#define SB_ERR_NOMEM (-3)       /* device or host allocation failed */
#define SB_ERR_UNSUPPORTED (-4) /* option the reference has but this build does not */
#define SB_ERR_NODEVICE (-5)    /* no CUDA device / kernels not loadable */
#define SB_ERR_TIMEOUT (-6)     /* a bounded device-side wait gave up */

/* Sentinel used by every output file of the reference (clib LARGEINT). */
#define SB_LARGEINT 2000000000

/* Match types written to the .mt files (Strack/speckleTrack.c:19-22). */
#define SB_BAD 0
#define SB_CMATCH 1
#define SB_AMPMATCH 2
#define SB_AMPMATCHLARGE 3

/* Byte orders (Strack/strack.h:9-10). */
#define SB_LSB 0
#define SB_MSB 1

/* Sample types of the SLC images. */
#define SB_CFLOAT32 0 /* complex float32 (default; "floatFlag == TRUE") */
#define SB_CINT16 1   /* complex int16 ("-integerComplex") */

typedef struct sb_context sb_context;

/* ------------------------------------------------------------------------ */
/* Context                                                                   */
/* ------------------------------------------------------------------------ */

/* Create a context on CUDA device `device`.  No reference counterpart: the
 * reference keeps its state in module globals (Strack/speckleTrack.c:89-134). */
int sb_context_create(int device, sb_context **out);
void sb_context_destroy(sb_context *ctx);
/* Last error message of this context (never NULL). */
const char *sb_last_error(const sb_context *ctx);
/* ABI version compiled into the library. */
int sb_abi_version(void);
/* Device-side time (ms) of the last sb_strack/sb_strackw/sb_cull call, measured
 * with CUDA events on the context stream, split into: [0] whole call,
 * [1] host->device copies, [2] kernels, [3] device->host copies. */
int sb_last_timing(const sb_context *ctx, float ms[4]);
/* Number of kernels launched by the last call. */
int64_t sb_last_launch_count(const sb_context *ctx);
/* Device time (ms, CUDA events on the context stream) of the main kernels of
 * the last sb_strack call: [0] complex stage, [1] small amplitude try,
 * [2] large amplitude try, [3] Gaussian fits, [4] bookkeeping (select, fill,
 * finalize); and the number of points each of [0..2] processed in [5..7]. */
int sb_last_stage_timing(const sb_context *ctx, float ms[8]);
/* Bound of every device-side wait of this context's kernels (the cullSTData
 * wavefront kernel waits for the previous grid row): a wait gives up after
 * `naps` naps of 64 ns, the kernel returns early and the call fails with
 * SB_ERR_TIMEOUT; the context stays usable.  Default 2^26 (~4 s); 0 gives
 * up at the first unmet check.  No reference counterpart (the reference's
 * raster loop, Cullst/cullSTData.c:75-123, never waits). */
int sb_set_wait_limit(sb_context *ctx, int64_t naps);

/* Transform form of strack's complex stage (cmpPSWithPad + the IFFT of
 * cmpTrackFast, Strack/speckleTrack.c:604-709).  No reference counterpart:
 * the reference has one form, FFTW in float.
 *   SB_FORM_FP32       FP32 FFTs on the CUDA cores (default).
 *   SB_FORM_SPLIT_BF16 the patch DFTs as GEMMs on the tensor cores with
 *                      operands split into hi + lo bfloat16 (three products,
 *                      FP32 accumulation); the oversampling, the peak search
 *                      and every decision stay FP32/FP64 as in the FP32 form.
 *                      Used where supported -- complex window 64, no
 *                      baseline, no interferogram, no -gauss -- and the FP32
 *                      form otherwise; sb_last_form() tells which one ran. */
#define SB_FORM_FP32 0
#define SB_FORM_SPLIT_BF16 1
int sb_set_form(sb_context *ctx, int form);
/* Form the complex stage of the last sb_strack call ran (SB_FORM_*). */
int sb_last_form(const sb_context *ctx);

/* Launch shape of one kernel for one window size, as an autotuner measured it
 * (specklesource_b200/autotune.py writes the table the Python runtime
 * applies).  No reference counterpart.  threads: a compiled thread count
 * (0: the default); ctasPerSm: CTAs per SM of the persistent grid, at most
 * the resident maximum (0: that maximum).  Kernels and windows:
 *   SB_TUNE_COMPLEX     FP32 complex stage, window 16, 24, 32, 48 or 64
 *   SB_TUNE_COMPLEX_TC  split-BF16 complex stage, window 64 (threads 0)
 *   SB_TUNE_AMPLITUDE   shared-memory amplitude try, window 16, 24, 32, 48 or 64
 *                       (threads 0)
 * Results do not depend on ctasPerSm; a different thread count changes the
 * order of the float partial sums of the patch powers (not the transforms).
 * Unknown kernels, windows or thread counts: SB_ERR_UNSUPPORTED; a CTA count
 * above the resident maximum: SB_ERR_ARG. */
#define SB_TUNE_COMPLEX 0
#define SB_TUNE_COMPLEX_TC 1
#define SB_TUNE_AMPLITUDE 2
int sb_set_tuning(sb_context *ctx, int kernel, int window, int threads, int ctasPerSm);

/* Device memory the context holds (bytes): the buffers its calls grew, kept
 * for reuse by later calls, and its constant tables.  No reference
 * counterpart (the reference mallocs per run and never frees). */
int64_t sb_context_device_bytes(const sb_context *ctx);
/* Frees the context's grown buffers (after its stream is idle); later calls
 * grow them again.  The constant tables are kept.  For a server that admits
 * jobs against a device-memory budget.  No reference counterpart. */
int sb_context_release(sb_context *ctx);

/* ------------------------------------------------------------------------ */
/* Inputs                                                                    */
/* ------------------------------------------------------------------------ */

/* One SLC image: na rows (azimuth) of nr complex samples (range).  The bytes
 * are those of the image file (raw, as read by loadBuffer,
 * Strack/speckleTrack.c:1369-1399); byteOrder says whether they must be
 * swapped (MSB = big-endian file, the reference default). */
typedef struct {
    const void *data;
    int32_t nr;
    int32_t na;
    int32_t sampleType; /* SB_CFLOAT32 or SB_CINT16 */
    int32_t byteOrder;  /* SB_LSB: native little-endian; SB_MSB: swap */
    int32_t onDevice;   /* 0: host pointer; 1: device pointer (already resident) */
} sb_image;

/* Prior offset grid used for the initial shift when polyShift == 0
 * (Offsets read by readBothOffsetsStrack, Strack/readBothOffsetsStrack.c:79-120).
 * Values are native floats; <= -0.9*LARGEINT means "no value". */
typedef struct {
    int32_t nr;
    int32_t na;
    double r0;
    double a0;
    double deltaR;
    double deltaA;
    const float *dr; /* na x nr, host */
    const float *da; /* na x nr, host */
} sb_offset_grid;

/* Byte mask gating each grid point (maskData, Strack/strack.h:42-51). */
typedef struct {
    int32_t r0;
    int32_t a0;
    int32_t nr;
    int32_t na;
    int32_t nrl; /* range looks (sample spacing of the mask) */
    int32_t nal; /* azimuth looks */
    const uint8_t *mask; /* na x nr, host; values are read as signed char */
} sb_mask;

/* Baseline phase flattening (phaseCorrectBaseline, speckleTrack.c:868-907).
 * All-zero baseline terms make the correction an exact identity, which is
 * also what the reference computes when no baseparams file is given (the
 * fields are then pinned to zero). */
typedef struct {
    double Bn, Bp, dBn, dBp, dBnQ, dBpQ;
    double lambda;
    /* Per range sample of image 1 (length nSlpR): sin/cos of the look-angle
     * offset and 1/range, as tabulated by initPhaseCorrect
     * (speckleTrack.c:1556-1625).  May be NULL when all terms are zero. */
    const double *sinThetaD;
    const double *cosThetaD;
    const double *overRange;
} sb_baseline;

/* Multi-looked interferogram used to flatten the fringe phase of patch 1
 * before complex matching (the intfile / intgeodat inputs; read by getInt,
 * Strack/getInt.c:11-77, applied by phaseCorrectInt,
 * Strack/speckleTrack.c:909-1000).  Samples are complex int16 (re, im pairs),
 * na x nr, each covering nrl x nal SLC pixels.  Lines the reference finds
 * missing from a short file hold (1, 1); pass them that way. */
typedef struct {
    const void *data;  /* na * nr (re, im) int16 pairs */
    int32_t nr, na;    /* size (the geodat's rangeSize / azimuthSize) */
    int32_t nrl, nal;  /* range / azimuth looks */
    int32_t byteOrder; /* SB_MSB as in the file (freadBS), or SB_LSB */
    int32_t onDevice;  /* data is a device pointer */
} sb_interferogram;

/* Parameters shared by strack and strackw (TrackParams, Strack/strack.h:56-165). */
typedef struct {
    int32_t rStart, aStart; /* first estimate (already divided by scaleFactor) */
    int32_t deltaR, deltaA; /* grid step */
    int32_t nR, nA;         /* grid size */
    int32_t wR, wA;         /* complex window */
    int32_t wRa, wAa;       /* amplitude window (strackw: search window) */
    int32_t scaleFactor;    /* output offsets are multiplied by this */
    /* strack flags (Strack/strack.c:137-178) */
    int32_t noComplex;      /* -noComplex */
    int32_t hanningFlag;    /* 1 unless -noHanning */
    int32_t maxTries;       /* 2, or 1 with -singleAmp */
    int32_t checkAzFocus;   /* -checkAzFocus */
    int32_t gaussFlag;      /* -gauss: 2-D Gaussian peak fit (cmpTrackGauss) */
    float azDefocusThresh;  /* 1.8 in the reference CLI */
    /* strackw parameters (parseTrack.c:222-253) */
    int32_t edgePadR, edgePadA; /* search radius, before the internal +NFAST/4 */
    int32_t navgR, navgA;       /* box pre-smoothing half widths (>1 enables) */
    /* initial shift (parseInitialOffsets.c, findImage2Pos) */
    int32_t polyShift;          /* 1: polynomial; 0: initOffsets grid */
    double rShiftPoly[3];       /* Rshift = p0 + p1*range + p2*azimuth */
    double aShiftPoly[3];
    const sb_offset_grid *initOffsets; /* required when polyShift == 0 */
    const sb_mask *mask;               /* NULL: every point is tried */
    const sb_baseline *baseline;       /* NULL: zero baseline */
    const sb_interferogram *intf;      /* NULL: no interferogram (strack complex stage only) */
} sb_track_params;

/* ------------------------------------------------------------------------ */
/* Outputs                                                                   */
/* ------------------------------------------------------------------------ */

/* Grids written row by row to <outputfile>.{dr,da,cc,azd,mt} by writeOffsets
 * (Strack/sTrackOut.c:44-60).  Pointers are host memory unless onDevice. */
typedef struct {
    float *offR;
    float *offA;
    float *corr;
    float *azd;     /* strack only; may be NULL for strackw */
    uint8_t *type;
    int32_t onDevice;
    /* statistics printed by printLineSummary (speckleTrack.c:1426-1447) */
    int64_t nComplex, nAmp, nAmpL, nFail, nAttempted;
} sb_track_result;

/* ------------------------------------------------------------------------ */
/* Tracking                                                                  */
/* ------------------------------------------------------------------------ */

/* Replaces void speckleTrack(TrackParams *) (Strack/strack.h:170,
 * body Strack/speckleTrack.c:159-346): complex match first, then the small
 * and large amplitude tries, for every point of the nA x nR grid. */
int sb_strack(sb_context *ctx, const sb_track_params *p, const sb_image *img1,
              const sb_image *img2, sb_track_result *out);

/* Many pairs in one call: speckleTrack (as sb_strack) for nPairs image pairs,
 * params[k], img1[k], img2[k] -> out[k].  No reference counterpart (the
 * reference tracks one pair per run); each pair's grids and statistics equal
 * its own sb_strack result.  The pairs are grouped by window size and every
 * stage runs once per group over the points of all its pairs (one persistent
 * complex-stage launch per group), which pays off for many small pairs.
 * Pairs may differ in image size, grid, windows, initial shift and mask; the
 * images share sample type and byte order, and the flags noComplex,
 * hanningFlag, maxTries, checkAzFocus, gaussFlag, azDefocusThresh and
 * scaleFactor are the same for every pair.  Baseline and interferogram
 * flattening are refused (SB_ERR_UNSUPPORTED): use sb_strack.  The device
 * holds both images of every pair at once (copied into two atlases). */
int sb_strack_batch(sb_context *ctx, int32_t nPairs, const sb_track_params *params, const sb_image *img1,
                    const sb_image *img2, sb_track_result *out);

/* Replaces void corrTrackFast(TrackParams *) (Strackw/strackt.h:31,
 * body Strackw/corrTrackFast.c:89-231): normalised amplitude correlation of a
 * chip of image 2 inside a search window of image 1. */
int sb_strackw(sb_context *ctx, const sb_track_params *p, const sb_image *img1,
               const sb_image *img2, sb_track_result *out);

/* Batched Doppler-carrier estimate: replaces estDopCarrier1 (Strack/strack.h:180,
 * Strack/dopplerEstimation.c:25-40) for nPatch pairs of nAz x nRg complex
 * patches stored contiguously (interleaved re,im float32, device pointers).
 * azShift[k] receives the roll rescaled to wA. */
int sb_est_dop_carrier(sb_context *ctx, const float *patches1, const float *patches2,
                       int32_t nPatch, int32_t nAz, int32_t nRg, int32_t wA,
                       int32_t *azShift);

/* ------------------------------------------------------------------------ */
/* Culling                                                                   */
/* ------------------------------------------------------------------------ */

/* CullParams (Cullst/cullst.h:4-59) restricted to the values the passes read. */
typedef struct {
    int32_t nR, nA;
    int32_t bR, bA;        /* -boxSize (cullSTData); cullStats always uses 9 */
    int32_t nGood;         /* -nGood */
    float maxA, maxR;      /* -maxA -maxR */
    int32_t sR, sA;        /* -sr -sa */
    int32_t islandThresh;  /* -islandThresh (<=0: no island pass) */
    float corrThresh;      /* -corrThresh */
    int32_t singleMT;      /* -singleMT (only honoured with a mask, as in the reference) */
    int32_t useSim;        /* -useSim */
    int32_t connectivity;  /* island labelling: 8 (default) or 4 */
    int32_t nCullPasses;   /* cullSTData repetitions; cullst runs 3 */
} sb_cull_params;

/* Buffers of one cull job (host memory unless onDevice).  offR/offA/type are
 * modified in place like the reference's CullParams arrays. */
typedef struct {
    float *offR, *offA;   /* in/out (cullSTData edits them in place) */
    const float *corr;    /* in */
    uint8_t *type;        /* in/out */
    const uint8_t *mask;  /* offsets.mask (NULL: maskFlag FALSE) */
    const float *simR, *simA; /* -useSim offsets (NULL unless useSim) */
    float *offRS, *offAS; /* out: smoothed offsets (.dr/.da of outbase) */
    float *sigmaR, *sigmaA; /* out: sigmas (.sr/.sa next to inbase) */
    int32_t onDevice;
    int64_t nCulled;      /* out: points culled by the last cullSTData pass */
    int64_t nIslands, nIslandPoints; /* out */
} sb_cull_data;

/* Whole cullst pipeline of Cullst/cullst.c:71-101: sim subtract, cullSTData
 * x nCullPasses, cullStats, sim add, cullSmooth, cullIslands. */
int sb_cull(sb_context *ctx, const sb_cull_params *p, sb_cull_data *d);

/* Single passes, same buffers.  Replace cullSTData/cullStats/cullSmooth/
 * cullIslands(CullParams *) (Cullst/cullst.h:60-66). */
int sb_cull_st_data(sb_context *ctx, const sb_cull_params *p, sb_cull_data *d);
int sb_cull_stats(sb_context *ctx, const sb_cull_params *p, sb_cull_data *d);
int sb_cull_smooth(sb_context *ctx, const sb_cull_params *p, sb_cull_data *d);
int sb_cull_islands(sb_context *ctx, const sb_cull_params *p, sb_cull_data *d);

/* ------------------------------------------------------------------------ */
/* Culling Landsat offsets (cullls)                                          */
/* ------------------------------------------------------------------------ */

/* CullLSParams (Cullls/cullls.h:2-35) restricted to the values the passes
 * read, plus the values cullls takes from landsatSource64 headers that are
 * not part of the reference tree (lstrack.h, lsfit.h, common.h): the caller
 * supplies them.  X is the column (range-like) offset, Y the row offset. */
typedef struct {
    int32_t nx, ny;        /* matches.nx, matches.ny: grid columns and rows */
    int32_t boxSize;       /* -boxSize (bR = bA; cullls default 9) */
    int32_t nGood;         /* -nGood (default 17) */
    float maxX, maxY;      /* -maxX (.75) -maxY (1.0): median deviation limits */
    int32_t sX, sY;        /* -sx -sy (3): smoothing box */
    int32_t islandThresh;  /* -islandThresh (<=0: no island pass; default -1) */
    int32_t nCullPasses;   /* cullLSData repetitions; cullls runs 3 */
    int32_t connectivity;  /* island labelling: 8 (default) or 4 */
    double deltaT;         /* fitDat.deltaT, days between the images */
    double dx, dy;         /* matches.dx, matches.dy: pixel size (m) */
    double noDataLimit;    /* NODATA + 1 as the Y > NODATA + 1 test sees it */
    double nOver;          /* lstrack's NOVER (quantisation 1/nOver px), > 0 */
    uint8_t slowVelMask;   /* SLOWVEL bit(s) of matches.type */
    uint8_t noDataMask;    /* NODATATOUSE bit(s) of matches.type */
    uint8_t reserved[6];
} sb_cullls_params;

/* Buffers of one cullls job (host memory unless onDevice). */
typedef struct {
    float *X, *Y;          /* in/out: cullLSData culls them in place */
    const uint8_t *type;   /* in: matches.type */
    float *XS, *YS;        /* out: smoothed offsets (.cull.dx/.cull.dy) */
    float *sigmaX, *sigmaY; /* out: sigmas (.cull.sx/.cull.sy) */
    int32_t onDevice;
    int64_t nAttempt;      /* out: points with (type & noDataMask) == 0, before culling */
    int64_t nMatch;        /* out: valid points before culling */
    int64_t nCulled;       /* out: points culled by the last cullLSData pass */
    int64_t nIslands, nIslandPoints; /* out */
} sb_cullls_data;

/* Whole cullls pipeline of Cullls/cullls.c:23-56: cullLSData x nCullPasses,
 * cullLSStats, cullLSSmooth, cullLSIslands (cullLSData.c:13-138,
 * cullLSStats.c:19-157, cullLSSmooth.c:11-73, cullLSIslands.c:15-174). */
int sb_cullls(sb_context *ctx, const sb_cullls_params *p, sb_cullls_data *d);

/* ------------------------------------------------------------------------ */
/* Allocation-free amplitude correlation                                     */
/* ------------------------------------------------------------------------ */

/* No counterpart in the reference: an extra entry point of this library.
 *
 * For callers that must not allocate device memory while they run -- a host
 * application that has reserved the GPU's memory up front for its own pool,
 * or a latency-critical loop in which cudaMalloc/cudaFree would add an
 * implicit device synchronisation.  It computes the amplitude try of strack
 * (getAmpPatches + ampMatch + ampTrackFast, Strack/speckleTrack.c:398-597,
 * 1006-1189, without the Gaussian-width fit) for nPatch pairs of wa x wa
 * patches that the caller has already cut out, and allocates nothing: its
 * workspace is a fixed SB_NOALLOC_SCRATCH_BYTES array in the library's device
 * memory, which every GPU that loads the library holds until the process
 * exits.
 *
 * All pointers are device pointers.  patches1/patches2: nPatch patches of
 * wa x wa complex float32 (re, im interleaved, native byte order), patch k at
 * offset k*wa*wa*2 floats.  azShift: per-patch spectral roll in rows (any
 * integer; it is reduced modulo wa, as a roll is periodic in wa), or NULL to
 * estimate it from each pair as estDopCarrier1 does.  Outputs per patch:
 * haveData (1 when the zero-count and empty-patch tests pass), cMax
 * (normalised correlation; -1 when the peak is too close to the edge),
 * iMax/jMax (peak in 1/NOVER-sample units, or -1000).
 * wa must be 16, 24, 32, 48 or 64 (SB_NOALLOC_MAX_WA); larger windows are
 * rejected with SB_ERR_ARG.
 * Set-up: sb_context_create loads this entry point's kernels and its
 * workspace on the context's device (CUDA loads modules lazily; the
 * workspace is allocated when its module loads), once per device and
 * process.  A caller that reserves the GPU's memory for its own pool creates
 * its context first; the calls themselves load no code and allocate nothing.
 * Every call looks the workspace's device address up in the current CUDA
 * context.  Every call shares the one workspace: calls that overlap on the
 * GPU (other threads, other contexts on the same device) race and must be
 * serialised by the caller.  The workspace keeps the last call's contents;
 * every element is written before it is read, so nothing needs clearing. */
#define SB_NOALLOC_MAX_WA 64
#define SB_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)
int sb_amp_match_noalloc(sb_context *ctx, const float *patches1, const float *patches2, int32_t nPatch,
                         int32_t wa, const int32_t *azShift, double *cMax, int32_t *iMax, int32_t *jMax,
                         int32_t *haveData);

#ifdef __cplusplus
}
#endif

#endif /* SPECKLE_B200_H */
