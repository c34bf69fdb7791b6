// strack_peak.cu -- the end of cmpTrackFast (Strack/speckleTrack.c:648-709)
// and the sample gathering of complexMatch's Gaussian-width fits (:372-385),
// one warp per patch.
//
// The complex kernel leaves, for every patch, findCPeak's coarse peak, the
// patch powers and |c|^2 of the 2x surface around the peak (PeakJob).  Here a
// warp oversamples the 8 x 8 block by 12 (overSampleC: |D Y D^T| over the
// 48 x 48 search window, first maximum in raster order), normalises the
// correlation, places the peak in 1/NOVER units and copies the 2 x 18 samples
// through the oversampled peak's coarse cell for the fit kernel.  Taking this
// tail out of the complex kernel removes five block barriers and a phase in
// which a quarter of its threads idle; a warp does it without block barriers.
#include <cuda_runtime.h>
#include <stdint.h>

#include "strack_device.cuh"
#include "strack_kernels.h"

namespace sbk {

constexpr int kPeakWarps = 8;  // warps per CTA

__global__ void __launch_bounds__(32 * kPeakWarps) strack_peak_kernel(PeakArgs a)
{
    __shared__ __align__(16) float osD[OSW * NFAST + 2 * 16];
    __shared__ __align__(16) float2 Yb[kPeakWarps][NFAST * NFAST];
    __shared__ __align__(16) float2 T[kPeakWarps][NFAST * OSW];
    __shared__ float blk[kPeakWarps][NFAST * NFAST];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int e = threadIdx.x; e < OSW * NFAST + 2 * 16; e += blockDim.x) osD[e] = reinterpret_cast<const float*>(a.osD)[e];
    __syncthreads();
    const int W2 = 2 * a.W;
    const int nWarps = gridDim.x * kPeakWarps;
    for (int it = blockIdx.x * kPeakWarps + w; it < a.nList; it += nWarps) {
        const PeakJob* pj = a.peak + it;
        const int iC = pj->iC, jC = pj->jC;
        if (iC == PJ_NODATA) continue;  // getPatches failed: the complex kernel wrote the record
        const int p = pj->point;
        double cMax = -1.0;
        int iMax = -1000, jMax = -1000, gate = 0;
        if (iC >= -999) {
            for (int t = lane; t < NFAST * NFAST; t += 32) blk[w][t] = sqrtf((&pj->blk[0][0])[t]);
            __syncwarp();
            const ArgMax ob = oversample_peak_warp(blk[w], osD, Yb[w], T[w]);
            const int iMax1 = ob.pos / OSW + (NFAST * NOVER) / 2 - 2 * NOVER;
            const int jMax1 = ob.pos % OSW + (NFAST * NOVER) / 2 - 2 * NOVER;
            cMax = (double)ob.v / (NFAST * NFAST);
            cMax = a.hanCorr * cMax / (sqrt(pj->p1 * pj->p2) * pow((double)(a.W * a.W), 2));
            iMax = (iC * NOVER) + iMax1 - (NOVER * NFAST) / 2;
            jMax = (jC * NOVER) + jMax1 - (NOVER * NFAST) / 2;
            // samples for gaussPeak1D x 2 through the coarse cell of the peak:
            // iM in [iC - 2, iC + 1] (iMax1 in [24, 72), iMax > 0), so the
            // strips hold them
            const int iM = iMax / NOVER, jM = jMax / NOVER;
            gate = (iM - NGAUSS / 2) >= 0 && (iM + NGAUSS / 2) < W2 && (jM - NGAUSS / 2) >= 0 &&
                   (jM + NGAUSS / 2) < W2;
            if (gate) {
                FitJob* fj = &a.fit[it];
                for (int t = lane; t < 2 * NGAUSS; t += 32) {
                    const int f = t / NGAUSS, k = t % NGAUSS;
                    if (f == 0)
                        fj->samp[0][k] = sqrtf(pj->hs[iM - (iC - 2)][jM - NGAUSS / 2 + k - (jC - NGAUSS / 2 - 2)]);
                    else
                        fj->samp[1][k] = sqrtf(pj->vs[iM - NGAUSS / 2 + k - (iC - NGAUSS / 2 - 2)][jM - (jC - 2)]);
                }
                if (lane == 0) {
                    fj->x0[0] = jM - NGAUSS / 2;
                    fj->x0[1] = iM - NGAUSS / 2;
                }
            }
        }
        if (lane == 0) {
            PointRec* r = &a.rec[p];
            r->cMax[0] = cMax;
            r->iMax[0] = iMax;
            r->jMax[0] = jMax;
            if (gate) r->flags |= RF_GATE_C;
            a.fit[it].point = p;
            a.fit[it].gate = gate;
        }
        __syncwarp();  // blk[w] is rewritten by the next patch
    }
}

cudaError_t launch_strack_peak(const PeakArgs& a, int numSM, cudaStream_t st)
{
    if (a.nList <= 0) return cudaSuccess;
    long long blocks = ((long long)a.nList + kPeakWarps - 1) / kPeakWarps;
    const long long cap = (long long)numSM * 8;
    if (blocks > cap) blocks = cap;
    strack_peak_kernel<<<(unsigned)blocks, 32 * kPeakWarps, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace sbk
