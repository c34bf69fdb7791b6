// strack_common.cuh -- data layout and scalar rules shared by the strack
// stage kernels (complex, small amplitude, large amplitude) and the finalize
// kernel.  The control flow of the reference's per-point loop
// (Strack/speckleTrack.c:194-323) is replayed by strack_walk() from the
// per-stage records, so every stage kernel and the finalize kernel take the
// same decisions the serial loop takes.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/speckle_b200.h"

namespace sbk {

constexpr int NOVER = 12;  // speckleTrack.c:15
constexpr int NFAST = 8;   // speckleTrack.c:16
constexpr int OS = 2;      // speckleTrack.c:25-26
constexpr int LA = 2;      // speckleTrack.c:18
constexpr int NGAUSS = 18; // speckleTrack.c:29

// Host-computed plan of one grid point (findImage2Pos, maskValue, boundsCheck).
struct PointPlan {
    int32_t r1, a1, r2, a2;  // complex window corners in image 1 / image 2
    uint32_t flags;
};
enum : uint32_t {
    PF_MASK = 1u,      // maskVal > 0
    PF_CBOUND = 2u,    // complex window in bounds
    PF_SBOUND = 4u,    // small amplitude window in bounds
    PF_LBOUND = 8u,    // large amplitude window in bounds
};

// Per-point results of the stage kernels.
struct PointRec {
    double cMax[3];   // complex, small amp, large amp
    int32_t iMax[3];  // oversampled peak index (NOVER units), or -1000
    int32_t jMax[3];
    float azd;        // running aZDefocus value
    int32_t azset;    // azShift set at this point by a Doppler estimate (-1: none)
    uint32_t flags;
    int32_t azUsed;   // azShift the amplitude tries used
    double cRaw;      // amplitude try: findCPeak value before oversampling
    int32_t iC, jC;   // amplitude try: coarse peak (or -1000)
};

// Samples handed from a stage kernel to the Gaussian-width fit kernel
// (gaussPeak1D, speckleTrack.c:2137-2202): one entry per list position.
struct FitJob {
    int32_t point;
    int32_t gate;            // 0: the NGAUSS gate failed, no fit
    int32_t x0[2];           // first sample position: [0] range fit, [1] azimuth fit
    float samp[2][NGAUSS];   // |c| samples through the coarse peak
};
enum : uint32_t {
    RF_HD_C = 1u,      // getPatches returned TRUE
    RF_GOOD_C = 2u,
    RF_HD_S = 4u,      // getAmpPatches (small) returned TRUE
    RF_GOOD_S = 8u,
    RF_HD_L = 16u,
    RF_GOOD_L = 32u,
    RF_DONE_C = 64u,   // stage kernels have written their part
    RF_DONE_S = 128u,
    RF_DONE_L = 256u,
    RF_GATE_C = 512u,  // Gaussian gate passed (fit pending / done)
};

struct WalkParams {
    int32_t wR, wA, wRa, wAa;
    int32_t noComplex, maxTries;
};

// Shift of a complex match (finalizeCmpxMatch, speckleTrack.c:714-739).
__host__ __device__ inline void cmpx_shifts(int iMax, int jMax, int wR, int wA, float* rShift1, float* aShift1)
{
    const double invNOVER = 1.0 / (float)NOVER;
    const double wRover2exp = wR / 2. * NOVER * OS;
    const double wAover2exp = wA / 2. * NOVER * OS;
    *rShift1 = (float)(((float)jMax - wRover2exp) * invNOVER / OS);
    *aShift1 = (float)(((float)iMax - wAover2exp) * invNOVER / OS);
}

__host__ __device__ inline bool cmpx_good(double cMax, int iMax, int jMax, int wR, int wA, int noComplex)
{
    if (!(cMax > .185 && noComplex == 0)) return false;
    float r, a;
    cmpx_shifts(iMax, jMax, wR, wA, &r, &a);
    return fabs((double)r) < 0.125 * wR * OS && fabs((double)a) < 0.125 * wA * OS;
}

// Shift of an amplitude match (speckleTrack.c:275-276).
__host__ __device__ inline void amp_shifts(int iMax, int jMax, int wRa, int wAa, int s, float* rShift1, float* aShift1)
{
    const double invNOVER = 1.0 / (float)NOVER;
    *rShift1 = (float)(((float)jMax - wRa * 0.5 * OS * NOVER * s) * invNOVER / OS);
    *aShift1 = (float)(((float)iMax - wAa * 0.5 * OS * NOVER * s) * invNOVER / OS);
}

__host__ __device__ inline bool amp_good(double cMax, int iMax, int jMax, int wRa, int wAa, int s)
{
    const double cThresh = (s == 1) ? 0.07 : 0.028;
    float r, a;
    amp_shifts(iMax, jMax, wRa, wAa, s, &r, &a);
    return fabs((double)r) < 0.15 * wRa * OS * s && fabs((double)a) < 0.15 * wAa * OS * s && cMax > cThresh;
}

// Result of replaying the per-point loop.
struct WalkOut {
    int stage_next;   // 1: small amp needs computing, 2: large amp needs computing, 0: done
    int good;
    int type;
    int haveData;
    double cMax;      // value written to the .cc grid
    float rShift1, aShift1;
    int nSkip;
};

// Replays speckleTrack.c:221-299 for one point using the records available.
// Stops at the first try whose record is missing and reports it.
__host__ __device__ inline WalkOut strack_walk(const PointPlan& pl, const PointRec& rc, const WalkParams& w)
{
    WalkOut o;
    o.stage_next = 0;
    o.good = 0;
    o.type = SB_BAD;
    o.haveData = 1;
    o.cMax = 0.0;
    o.rShift1 = 0.f;
    o.aShift1 = 0.f;
    o.nSkip = 0;
    const int mask = (pl.flags & PF_MASK) != 0;
    if ((pl.flags & PF_CBOUND) && mask && w.noComplex == 0) {
        o.haveData = (rc.flags & RF_HD_C) != 0;
        if (o.haveData) {
            o.cMax = rc.cMax[0];
            if (rc.flags & RF_GOOD_C) {
                o.good = 1;
                o.type = SB_CMATCH;
                cmpx_shifts(rc.iMax[0], rc.jMax[0], w.wR, w.wA, &o.rShift1, &o.aShift1);
            }
        } else {
            o.nSkip++;
        }
    }
    int nTries = 0;
    while (!o.good && o.haveData && mask && nTries < w.maxTries) {
        const int st = nTries == 0 ? 1 : 2;
        const uint32_t bound = st == 1 ? PF_SBOUND : PF_LBOUND;
        const uint32_t done = st == 1 ? RF_DONE_S : RF_DONE_L;
        const uint32_t hd = st == 1 ? RF_HD_S : RF_HD_L;
        const uint32_t gd = st == 1 ? RF_GOOD_S : RF_GOOD_L;
        if (pl.flags & bound) {
            if (!(rc.flags & done)) {
                o.stage_next = st;
                return o;
            }
            if (rc.flags & hd) {
                o.cMax = rc.cMax[st];
                if (rc.flags & gd) {
                    o.good = 1;
                    o.type = st == 1 ? SB_AMPMATCH : SB_AMPMATCHLARGE;
                    amp_shifts(rc.iMax[st], rc.jMax[st], w.wRa, w.wAa, st == 1 ? 1 : LA, &o.rShift1,
                               &o.aShift1);
                }
            } else {
                o.cMax = 0.0;
                o.nSkip++;
                o.haveData = 0;
            }
        } else {
            o.cMax = 0.0;
        }
        nTries++;
    }
    return o;
}

// Byte swap helpers for big-endian SLC files.
__device__ __forceinline__ uint32_t bswap32(uint32_t v) { return __byte_perm(v, 0, 0x0123); }
__device__ __forceinline__ uint32_t bswap16x2(uint32_t v) { return __byte_perm(v, 0, 0x2301); }

// One complex sample of an SLC image (loadBuffer, speckleTrack.c:1369-1399).
__device__ __forceinline__ float2 load_sample(const void* __restrict__ img, int nr, int row, int col, int sampleType,
                                              int byteOrder)
{
    const size_t k = (size_t)row * (size_t)nr + (size_t)col;
    if (sampleType == SB_CFLOAT32) {
        uint2 w = __ldg(reinterpret_cast<const uint2*>(img) + k);
        if (byteOrder == SB_MSB) {
            w.x = bswap32(w.x);
            w.y = bswap32(w.y);
        }
        return make_float2(__uint_as_float(w.x), __uint_as_float(w.y));
    } else {
        uint32_t w = __ldg(reinterpret_cast<const uint32_t*>(img) + k);
        if (byteOrder == SB_MSB) w = bswap16x2(w);
        return make_float2((float)(int16_t)(w & 0xffffu), (float)(int16_t)(w >> 16));
    }
}

}  // namespace sbk
