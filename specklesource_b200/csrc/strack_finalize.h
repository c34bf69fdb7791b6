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
};

cudaError_t launch_plan_poly(const PlanArgs& a, PointPlan* plan, int* clist, int* ccount, cudaStream_t st);

cudaError_t launch_rec_init(PointRec* rec, int n, cudaStream_t st);

// Band bucketing of the complex list for the overlapped upload (at most
// SB_BANDS_MAX bands): counts per band, then a scatter into band order.
constexpr int SB_BANDS_MAX = 16;
cudaError_t launch_band_count(const PointPlan* plan, const int* list, int n, int W, int rows1, int rows2, int nb,
                              int* bandOf, int* counts, cudaStream_t st);
cudaError_t launch_band_scatter(const int* list, const int* bandOf, int n, int nb, int* cursor, int* out,
                                cudaStream_t st);
cudaError_t launch_select(const PointPlan* plan, const PointRec* rec, int n, const WalkParams& w, int stage,
                          int* list, int* count, cudaStream_t st);
cudaError_t launch_az_fill(const PointRec* rec, int n, int* azEff, cudaStream_t st);
cudaError_t launch_finalize(const PointPlan* plan, const PointRec* rec, int n, const WalkParams& w, int scaleFactor,
                            float* offR, float* offA, float* corr, float* azd, uint8_t* type,
                            unsigned long long* stats, cudaStream_t st);

}  // namespace sbk
