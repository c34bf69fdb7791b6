// dop.cu -- sb_est_dop_carrier: estDopCarrier1 (Strack/dopplerEstimation.c:25-88)
// for a batch of patch pairs, one CTA per pair: complex means, lag-1 azimuth
// products in double, atan2, the integer roll, rescaled to wA.
#include <cuda_runtime.h>

#include "capi_internal.h"
#include "strack_device.cuh"

namespace sbk {

__global__ void __launch_bounds__(256) dop_kernel(const float2* p1, const float2* p2, int nAz, int nRg, int wA,
                                                  int* out)
{
    __shared__ double red[(256 / 32 + 1) * 8];
    const size_t n = (size_t)nAz * nRg;
    const float2* a = p1 + (size_t)blockIdx.x * n;
    const float2* b = p2 + (size_t)blockIdx.x * n;
    double m[4] = {0, 0, 0, 0};
    for (size_t e = threadIdx.x; e < n; e += blockDim.x) {
        m[0] += a[e].x; m[1] += a[e].y; m[2] += b[e].x; m[3] += b[e].y;
    }
    block_allsum<4, 256>(m, red);
    const double nn = (double)n;
    const double m1r = m[0] / nn, m1i = m[1] / nn, m2r = m[2] / nn, m2i = m[3] / nn;
    double d[4] = {0, 0, 0, 0};
    for (size_t e = threadIdx.x; e < (size_t)(nAz - 1) * nRg; e += blockDim.x) {
        const float2 x0 = a[e], x1 = a[e + nRg], y0 = b[e], y1 = b[e + nRg];
        double ar = (double)x1.x - m1r, ai = (double)x1.y - m1i, br = (double)x0.x - m1r, bi = (double)x0.y - m1i;
        d[0] += ar * br + ai * bi;
        d[1] += ai * br - ar * bi;
        ar = (double)y1.x - m2r; ai = (double)y1.y - m2i; br = (double)y0.x - m2r; bi = (double)y0.y - m2i;
        d[2] += ar * br + ai * bi;
        d[3] += ai * br - ar * bi;
    }
    block_allsum<4, 256>(d, red);
    if (threadIdx.x == 0) out[blockIdx.x] = dop_shift(d[0], d[1], d[2], d[3], nAz, wA);
}

}  // namespace sbk

extern "C" int sb_est_dop_carrier(sb_context* c, const float* patches1, const float* patches2, int32_t nPatch,
                                  int32_t nAz, int32_t nRg, int32_t wA, int32_t* azShift)
{
    if (!c) return SB_ERR_ARG;
    c->err.clear();
    c->launches = 0;
    if (!patches1 || !patches2 || !azShift) return sb_ctx_fail(c, SB_ERR_ARG, "null pointer argument");
    if (nPatch <= 0 || nAz < 2 || nRg < 1 || wA <= 0) return sb_ctx_fail(c, SB_ERR_ARG, "invalid sizes");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return sb_ctx_cuda(c, e, "cudaSetDevice");
    sbk::dop_kernel<<<nPatch, 256, 0, c->stream>>>(reinterpret_cast<const float2*>(patches1),
                                                   reinterpret_cast<const float2*>(patches2), nAz, nRg, wA, azShift);
    e = cudaGetLastError();
    if (e != cudaSuccess) return sb_ctx_cuda(c, e, "dop_kernel");
    c->launches = 1;
    e = cudaStreamSynchronize(c->stream);
    return sb_ctx_cuda(c, e, "sb_est_dop_carrier");
}
