// strack_finalize.h -- launchers of the strack bookkeeping kernels.
#pragma once
#include <cuda_runtime.h>

#include "strack_common.cuh"

namespace sbk {

struct PlanArgs {
    int rStart, aStart, deltaR, deltaA, nR, nA;
    int wR, wA, wRa, wAa;
    int scaleFactor, noComplex;
    double rPoly[3], aPoly[3];
    int nr1, na1, nr2, na2;
    const uint8_t* mask;  // device copy of the mask, or nullptr
    int mR0, mA0, mNr, mNa, mNrl, mNal;
    // batched calls (zero otherwise): the pair's first image rows in the
    // atlases, the key its complex candidates get, and the pair index to
    // record per point (pairOf, when non-null)
    int a1Off, a2Off;
    int keyValue;
    int* pairOf;
    int pairId;
    // > 0: complex candidates are keyed by their range strip of image 1,
    // min(r1 / stripPx, SB_BANDS_MAX - 1), instead of keyValue
    int stripPx;
};

// Writes the plan of every point and key[p] = keyValue for complex candidates, else -1.
cudaError_t launch_plan_poly(const PlanArgs& a, PointPlan* plan, int* key, cudaStream_t st);

cudaError_t launch_rec_init(PointRec* rec, int n, cudaStream_t st);

// Band of every complex-list entry for the overlapped upload (at most
// SB_BANDS_MAX bands): the key of the ordered partition by band.
constexpr int SB_BANDS_MAX = 32;
cudaError_t launch_band_key(const PointPlan* plan, const int* list, int n, int W, int rows1, int rows2, int nb,
                            int* bandOf, cudaStream_t st);
// key[p] = 0 for the points whose next missing try is `stage`, else -1.
cudaError_t launch_select(const PointPlan* plan, const PointRec* rec, int n, const WalkParams& w, int stage,
                          int* key, cudaStream_t st);
cudaError_t launch_az_fill(const PointRec* rec, int n, int* azEff, cudaStream_t st);
// pairOf (batched calls): pair of each point; statistics go to stats[8 * pair]
cudaError_t launch_finalize(const PointPlan* plan, const PointRec* rec, int n, const WalkParams& w, int scaleFactor,
                            float* offR, float* offA, float* corr, float* azd, uint8_t* type,
                            unsigned long long* stats, cudaStream_t st, const int* pairOf = nullptr);

}  // namespace sbk
