// strack_fit.cu -- Gaussian peak-width fits of a strack stage and the
// decisions that depend on them.  One thread per fit (two per list entry:
// even lane = range profile, odd lane = azimuth profile), all in registers,
// double precision (gaussPeak1D + mrqminMod, Strack/speckleTrack.c:2137-2202,
// 2309-2416).
//   complex stage:   aZDefocus = sigmaAz/sigmaRg when the NGAUSS gate passed;
//                    finalizeCmpxMatch only inside the gate and, with
//                    -checkAzFocus, only when |aZDefocus| < threshold
//                    (complexMatch, :380-392);
//   amplitude tries: aZDefocus updated when the gate passed; the early return
//                    of ampTrackFast (:551-553) keeps the coarse peak.
// The 3x3 normal equations of each Levenberg-Marquardt step are solved by
// Cramer's rule (Numerical Recipes uses Gauss-Jordan; both give the exact
// solution up to double rounding); a zero determinant ends the fit, as a
// singular matrix does in the reference's solver.
#include <cuda_runtime.h>

#include "strack_device.cuh"
#include "strack_fit.h"

namespace sbk {

struct Cof {
    double a11, a21, a22, a31, a32, a33;
    double b1, b2, b3;
    double chisq;
};

__device__ __forceinline__ Cof cof18(const double (&x)[NGAUSS], const double (&y)[NGAUSS], double A, double mu,
                                     double sig)
{
    Cof c = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double sig2i = 1.0 / (0.1 * 0.1);
    const double s2 = sig * sig, s3 = s2 * sig;
#pragma unroll
    for (int k = 0; k < NGAUSS; ++k) {
        const double t = x[k] - mu;
        const double ex = exp(-(0.5 * t * t / s2));
        const double ymod = A * ex;
        const double d1 = ex, d2 = ymod * t / s2, d3 = ymod * t * t / s3;
        const double dy = y[k] - ymod;
        const double w1 = d1 * sig2i, w2 = d2 * sig2i, w3 = d3 * sig2i;
        c.a11 += w1 * d1;
        c.a21 += w2 * d1;
        c.a22 += w2 * d2;
        c.a31 += w3 * d1;
        c.a32 += w3 * d2;
        c.a33 += w3 * d3;
        c.b1 += dy * w1;
        c.b2 += dy * w2;
        c.b3 += dy * w3;
        c.chisq += dy * dy * sig2i;
    }
    return c;
}

// sigma = a[3]/2 of the fit to 18 samples at x0, x0+1, ...
__device__ double fit_sigma(const float* samp, int x0)
{
    double x[NGAUSS], y[NGAUSS];
    float mx = 0.f;
#pragma unroll
    for (int k = 0; k < NGAUSS; ++k) mx = fmaxf(mx, samp[k]);
#pragma unroll
    for (int k = 0; k < NGAUSS; ++k) {
        x[k] = (double)(x0 + k);
        y[k] = (double)samp[k] / (double)mx;
    }
    double A = 1.0, mu = (double)(x0 + NGAUSS / 2), sg = 2.0;
    double alamda = 0.001;
    Cof al = cof18(x, y, A, mu, sg);
    double ochisq = al.chisq;
    double lasti = 2e9;
    for (int it = 0; it < 5; ++it) {
        const double f = 1.0 + alamda;
        const double m11 = al.a11 * f, m22 = al.a22 * f, m33 = al.a33 * f;
        const double m21 = al.a21, m31 = al.a31, m32 = al.a32;
        const double det = m11 * (m22 * m33 - m32 * m32) - m21 * (m21 * m33 - m32 * m31) + m31 * (m21 * m32 - m22 * m31);
        if (det == 0.0 || det != det) break;
        const double d1 = (al.b1 * (m22 * m33 - m32 * m32) - m21 * (al.b2 * m33 - m32 * al.b3) +
                           m31 * (al.b2 * m32 - m22 * al.b3)) / det;
        const double d2 = (m11 * (al.b2 * m33 - al.b3 * m32) - al.b1 * (m21 * m33 - m32 * m31) +
                           m31 * (m21 * al.b3 - al.b2 * m31)) / det;
        const double d3 = (m11 * (m22 * al.b3 - m32 * al.b2) - m21 * (m21 * al.b3 - al.b2 * m31) +
                           al.b1 * (m21 * m32 - m22 * m31)) / det;
        const double At = A + d1, mt = mu + d2, st = sg + d3;
        const Cof tr = cof18(x, y, At, mt, st);
        if (tr.chisq < ochisq) {
            alamda *= 0.1;
            ochisq = tr.chisq;
            al = tr;
            A = At;
            mu = mt;
            sg = st;
        } else {
            alamda *= 10.0;
        }
        if (fabs(mu - lasti) < 0.001) break;
        lasti = mu;
    }
    return sg * .5;
}

__global__ void __launch_bounds__(128) strack_fit_kernel(FitArgs a)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int job = t >> 1, f = t & 1;
    const int nList = a.nListDev ? min(a.nList, *a.nListDev) : a.nList;
    const bool live = job < nList;
    int gate = 0;
    double s = 0.0;
    if (live) {
        const FitJob* fj = &a.fit[job];
        gate = fj->gate;
        if (gate > 0) s = fit_sigma(fj->samp[f], fj->x0[f]);
    }
    const double sAz = __shfl_down_sync(0xffffffffu, s, 1);
    if (!live || f != 0 || gate < 0) return;
    const int p = a.fit[job].point;
    PointRec* r = &a.rec[p];
    if (a.stage == 0) {
        bool good = false;
        if (gate > 0) {
            const float azd = (float)(sAz / s);
            r->azd = azd;
            if (fabsf(azd) < a.azThresh || a.checkAzFocus == 0)
                good = cmpx_good(r->cMax[0], r->iMax[0], r->jMax[0], a.wR, a.wA, a.noComplex);
        }
        if (good) r->flags |= RF_GOOD_C;
    } else {
        const int st = a.stage;
        float azd = r->azd;
        if (gate > 0) {
            azd = (float)(sAz / s);
            r->azd = azd;
        }
        const bool early = r->iC < -999 || (fabsf(azd) >= a.azThresh && a.checkAzFocus != 0);
        if (early) {
            r->cMax[st] = r->cRaw;
            r->iMax[st] = r->iC;
            r->jMax[st] = r->jC;
        }
        const int sc = st == 1 ? 1 : LA;
        if (amp_good(r->cMax[st], r->iMax[st], r->jMax[st], a.wRa, a.wAa, sc))
            r->flags |= (st == 1 ? RF_GOOD_S : RF_GOOD_L);
    }
}

cudaError_t launch_strack_fit(const FitArgs& a, cudaStream_t st)
{
    if (a.nList <= 0) return cudaSuccess;
    const long long threads = 2LL * a.nList;
    strack_fit_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace sbk
