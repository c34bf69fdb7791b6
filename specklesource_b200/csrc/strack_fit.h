// strack_fit.h -- launcher of the Gaussian-width fit kernel.
#pragma once
#include <cuda_runtime.h>

#include "strack_common.cuh"

namespace sbk {

struct FitArgs {
    const FitJob* fit;
    int nList;            // number of fit jobs, or its upper bound when nListDev is set
    const int* nListDev;  // non-null: the number of jobs, read on the device
    int stage;  // 0 complex, 1 small amplitude, 2 large amplitude
    int wR, wA, wRa, wAa;
    int noComplex;
    float azThresh;
    int checkAzFocus;
    PointRec* rec;
};

cudaError_t launch_strack_fit(const FitArgs& a, cudaStream_t st);

}  // namespace sbk
