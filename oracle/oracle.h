/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the speckleSource
 * hot path, used by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg as the checker.  Nothing in the product links it.
 *
 * Parity pinned to the reference's own code: the reference's hot-path
 * sources (Strack/speckleTrack.c, Strackw/corrTrackFast.c, Cullst/cull*.c)
 * compile unmodified against stand-ins for the libraries its tree lacks
 * (oracle/refshim/; `make ref` -> oracle/_ref/), and tests/test_ref_pin.py
 * checks this restatement against them (offsets and match types identical)
 * live and through committed fixtures of their outputs
 * (tests/golden/ref_small.npz).  Known-answer tests of its own are in
 * tests/test_oracle_kat.py.
 * Built twice from the same sources:
 *   liboracle_f64.so  REAL=double, FLT=double  -- the FP64 oracle
 *   liboracle_f32.so  REAL=float,  FLT=float   -- reference-like precision,
 *                                                 the timed CPU baseline
 * The entry points take the same structs as the product's C ABI.
 */
#ifndef ORACLE_H
#define ORACLE_H

#include "../include/speckle_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* speckleTrack (Strack/speckleTrack.c:159-346) over grid rows [row0, row1);
 * row1 <= 0 means nA. Images must be host, native-order or MSB. */
int oracle_strack(const sb_track_params *p, const sb_image *img1, const sb_image *img2,
                  sb_track_result *out, int32_t row0, int32_t row1);

/* corrTrackFast (Strackw/corrTrackFast.c:89-231) over grid rows [row0,row1). */
int oracle_strackw(const sb_track_params *p, const sb_image *img1, const sb_image *img2,
                   sb_track_result *out, int32_t row0, int32_t row1);

/* cullst pipeline (Cullst/cullst.c:36-107) and its passes. */
int oracle_cull(const sb_cull_params *p, sb_cull_data *d);
int oracle_cull_st_data(const sb_cull_params *p, sb_cull_data *d);
int oracle_cull_stats(const sb_cull_params *p, sb_cull_data *d);
int oracle_cull_smooth(const sb_cull_params *p, sb_cull_data *d);
int oracle_cull_islands(const sb_cull_params *p, sb_cull_data *d);

/* cullls pipeline (Cullls/cullls.c:23-56). */
int oracle_cullls(const sb_cullls_params *p, sb_cullls_data *d);

/* estDopCarrier1 (Strack/dopplerEstimation.c:25-40) on one pair of
 * interleaved complex patches (float32 re,im), returning the roll scaled to wA. */
int oracle_est_dop_carrier(const float *p1, const float *p2, int32_t nAz, int32_t nRg,
                           int32_t wA);

/* 2-D DFT helper exposed for FFT tests: in-place on interleaved REAL data
 * passed as double (converted internally). */
int oracle_fft2d(double *data, int32_t na, int32_t nr, int32_t sign);
int oracle_fft2d_time(int32_t na, int32_t nr, int32_t reps, double *secs);

/* sizeof(REAL): 4 or 8 */
int oracle_real_size(void);

#ifdef __cplusplus
}
#endif

#endif
