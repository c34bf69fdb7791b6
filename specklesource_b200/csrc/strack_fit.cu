// strack_fit.cu -- Gaussian peak-width fits of a strack stage and the
// decisions that depend on them.  One CTA (two warps) per list entry: warp 0
// fits the range profile, warp 1 the azimuth profile, both in double precision
// (gaussPeak1D + mrqminMod, Strack/speckleTrack.c:2137-2202, 2309-2416).
//   complex stage:   aZDefocus = sigmaAz/sigmaRg when the NGAUSS gate passed;
//                    finalizeCmpxMatch only inside the gate and, with
//                    -checkAzFocus, only when |aZDefocus| < threshold
//                    (complexMatch, :380-392);
//   amplitude tries: aZDefocus updated when the gate passed; the early return
//                    of ampTrackFast (:551-553) keeps the coarse peak.
#include <cuda_runtime.h>

#include "strack_device.cuh"
#include "strack_fit.h"

namespace sbk {

__global__ void __launch_bounds__(64) strack_fit_kernel(FitArgs a)
{
    __shared__ double sig[2];
    const int job = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const FitJob* fj = &a.fit[job];
    const int gate = fj->gate;
    if (gate > 0) {
        const float smp = lane < NGAUSS ? fj->samp[warp][lane] : 0.f;
        const int xp = fj->x0[warp] + lane;
        const double s = gauss_peak_1d(smp, xp, lane);
        if (lane == 0) sig[warp] = s;
    }
    __syncthreads();
    if (threadIdx.x != 0 || gate < 0) return;
    const int p = fj->point;
    PointRec* r = &a.rec[p];
    if (a.stage == 0) {
        bool good = false;
        if (gate > 0) {
            const float azd = (float)(sig[1] / sig[0]);
            r->azd = azd;
            if (fabsf(azd) < a.azThresh || a.checkAzFocus == 0)
                good = cmpx_good(r->cMax[0], r->iMax[0], r->jMax[0], a.wR, a.wA, a.noComplex);
        }
        if (good) r->flags |= RF_GOOD_C;
    } else {
        const int st = a.stage;
        float azd = r->azd;
        if (gate > 0) {
            azd = (float)(sig[1] / sig[0]);
            r->azd = azd;
        }
        const bool early = r->iC < -999 || (fabsf(azd) >= a.azThresh && a.checkAzFocus != 0);
        if (early) {
            r->cMax[st] = r->cRaw;
            r->iMax[st] = r->iC;
            r->jMax[st] = r->jC;
        }
        const int s = st == 1 ? 1 : LA;
        if (amp_good(r->cMax[st], r->iMax[st], r->jMax[st], a.wRa, a.wAa, s))
            r->flags |= (st == 1 ? RF_GOOD_S : RF_GOOD_L);
    }
}

cudaError_t launch_strack_fit(const FitArgs& a, cudaStream_t st)
{
    if (a.nList <= 0) return cudaSuccess;
    strack_fit_kernel<<<a.nList, 64, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace sbk
