// strack_cmplx.cu -- complex (speckle) matching stage of strack, one CTA per
// grid point, everything resident in shared memory.
//
// Follows getPatches (Strack/speckleTrack.c:1194-1330), estDopCarrier1
// (Strack/dopplerEstimation.c:25-88), phaseCorrectBaseline (:868-907),
// cmpPSWithPad (:604-643), cmpTrackFast (:648-709), findCPeak (:744-805),
// overSampleC (:852-863), gaussPeak1D (:2137-2202), complexMatch (:349-394)
// and finalizeCmpxMatch (:714-739).
//
// The 2W x 2W inverse transform of the zero-padded cross spectrum is computed
// as four W x W inverse transforms, one per output parity (e1, e2): with the
// non-zero quadrants folded to X'[k1'][k2'] = S[(k1'+azShift) % W][k2'],
//   c[2 m1 + e1][2 m2 + e2] = IDFT_W(X' tau_e1[k1'] tau_e2[k2'])[m1][m2],
//   tau_0 = 1, tau_1[k'] = +-exp(+2 pi i k' / 2W) (minus for k' >= W/2),
// which is the same sum regrouped.  Only |c| is kept (four W x W float planes).
#include <cuda_runtime.h>

#include "strack_device.cuh"
#include "strack_kernels.h"

namespace sbk {

template <int W, int NT>
struct CmplxSmem {
    static constexpr int RS = W + 1;
    static constexpr int IMG = W * RS;  // float2
    static constexpr size_t bytes =
        sizeof(float2) * (2 * IMG) + sizeof(float) * (2 * W * W) + sizeof(float2) * (W + W + OSW * NFAST) +
        sizeof(float2) * (NFAST * OSW) + sizeof(float) * (NFAST * NFAST) + sizeof(double) * (NT / 32) * 8 +
        sizeof(int) * (3 * (NT / 32) + 8) + 64;
};

// |c| of the 2W x 2W surface at unshifted index (cy, cx).  The four parity
// planes live at float offsets poff(q) from the start of shared memory:
// planes 0, 1 in M, plane 2 over B, plane 3 over A.
template <int W>
__device__ __forceinline__ int poff(int q)
{
    constexpr int IMGF = 2 * W * (W + 1);  // one image region, in floats
    return q == 3 ? 0 : (q == 2 ? IMGF : 2 * IMGF + (q & 1) * W * W);
}
template <int W>
__device__ __forceinline__ float cmap(const float* sm, int cy, int cx)
{
    return sm[poff<W>(((cy & 1) << 1) | (cx & 1)) + (cy >> 1) * W + (cx >> 1)];
}
// fftshifted surface corrF[y][x] (findCPeak's layout)
template <int W>
__device__ __forceinline__ float fmap(const float* sm, int y, int x)
{
    const int cy = y + W < 2 * W ? y + W : y - W;
    const int cx = x + W < 2 * W ? x + W : x - W;
    return cmap<W>(sm, cy, cx);
}

template <int W, int NT>
__global__ void __launch_bounds__(NT, (W >= 48 ? 2 : 3)) strack_cmplx_kernel(CmplxArgs a)
{
    using S = CmplxSmem<W, NT>;
    constexpr int RS = S::RS, IMG = S::IMG;
    constexpr int W2 = 2 * W;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* A = reinterpret_cast<float2*>(smem_raw);
    float2* B = A + IMG;
    float* M = reinterpret_cast<float*>(B + IMG);
    float2* twW = reinterpret_cast<float2*>(M + 2 * W * W);
    float2* tau = twW + W;
    float2* osA = tau + W;
    float2* T = osA + OSW * NFAST;
    float* blk = reinterpret_cast<float*>(T + NFAST * OSW);
    double* red = reinterpret_cast<double*>(blk + NFAST * NFAST);
    int* isc = reinterpret_cast<int*>(red + (NT / 32) * 8);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    for (int e = tid; e < W; e += NT) {
        twW[e] = a.twW[e];
        tau[e] = a.tau[e];
    }
    for (int e = tid; e < OSW * NFAST; e += NT) osA[e] = a.osA[e];
    __syncthreads();

    float* smf = reinterpret_cast<float*>(smem_raw);
    const bool isFloat = a.sampleType == SB_CFLOAT32;
    const float thr = isFloat ? 1e-15f : 1e-9f;
    const float thrAll = thr * W * W;

    for (int it = blockIdx.x; it < a.nList; it += gridDim.x) {
        const int p = a.list[it];
        const PointPlan pl = a.plan[p];
        // ---------------------------------------------------- getPatches
        double s[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int e = tid; e < W * W; e += NT) {
            const int i = e / W, j = e % W;
            float2 z1 = load_sample(a.img1, a.nr1, pl.a1 + i, pl.r1 + j, a.sampleType, a.byteOrder);
            float2 z2 = load_sample(a.img2, a.nr2, pl.a2 + i, pl.r2 + j, a.sampleType, a.byteOrder);
            if (isFloat) {
                z1.x *= 1000.f; z1.y *= 1000.f;
                z2.x *= 1000.f; z2.y *= 1000.f;
            }
            if (a.hanning) {
                const float h = a.hanning[e];
                z2.x *= h;
                z2.y *= h;
            }
            const float pw1 = __fadd_rn(__fmul_rn(z1.x, z1.x), __fmul_rn(z1.y, z1.y));
            const float pw2 = __fadd_rn(__fmul_rn(z2.x, z2.x), __fmul_rn(z2.y, z2.y));
            if (pw1 < thr || pw2 < thr) s[6] += 1.0;
            s[0] += pw1;
            s[1] += pw2;
            s[2] += z1.x;
            s[3] += z1.y;
            s[4] += z2.x;
            s[5] += z2.y;
            A[i * RS + j] = z1;
            B[i * RS + j] = z2;
        }
        block_allsum<7, NT>(s, red);
        const bool haveData = !(s[6] > 20.0) && !(s[0] < thrAll || s[1] < thrAll);
        if (!haveData) {
            if (tid == 0) {
                a.rec[p].flags |= RF_DONE_C;
                a.rec[p].azset = -1;
                a.fit[it].point = p;
                a.fit[it].gate = 0;
            }
            continue;  // uniform across the block
        }
        // ---------------------------------------------------- Doppler (lag-1 sums)
        const double n = (double)(W * W);
        const double m1r = s[2] / n, m1i = s[3] / n, m2r = s[4] / n, m2i = s[5] / n;
        double d[4] = {0, 0, 0, 0};
        for (int e = tid; e < (W - 1) * W; e += NT) {
            const int i = e / W, j = e % W;
            const float2 p0 = A[i * RS + j], p1 = A[(i + 1) * RS + j];
            double ar = (double)p1.x - m1r, ai = (double)p1.y - m1i, br = (double)p0.x - m1r, bi = (double)p0.y - m1i;
            d[0] += ar * br + ai * bi;
            d[1] += ai * br - ar * bi;
            const float2 q0 = B[i * RS + j], q1 = B[(i + 1) * RS + j];
            ar = (double)q1.x - m2r; ai = (double)q1.y - m2i; br = (double)q0.x - m2r; bi = (double)q0.y - m2i;
            d[2] += ar * br + ai * bi;
            d[3] += ai * br - ar * bi;
        }
        block_allsum<4, NT>(d, red);
        const int azShift = dop_shift(d[0], d[1], d[2], d[3], W, W);
        const double p1 = s[0] / n, p2 = s[1] / n;
        // ---------------------------------------------------- baseline flattening
        if (a.baseOn) {
            const double xa0 = (pl.a1 - W / 2 - (a.na1 / 2)) / (double)a.na1;
            const double dX = 1. / (double)a.na1;
            const double ptod = -(4.0 * 3.14159265358979323846) / a.lambda;
            const int jb = (pl.r1 - W / 2 > 0 ? pl.r1 - W / 2 : 0);
            for (int e = tid; e < W * W; e += NT) {
                const int i = e / W, j = e % W;
                const double x = xa0 + i * dX;
                const double bn = a.Bn + xa0 * a.dBn + xa0 * xa0 * a.dBnQ;  // evaluated once, before the row loop
                const double bp = a.Bp + x * a.dBp + x * x * a.dBpQ;
                const double bsq = bn * bn + bp * bp;
                const int j1 = jb + j;
                double ph = -bn * a.sinThetaD[j1] - bp * a.cosThetaD[j1] + (0.5 * bsq * a.overRange[j1]);
                ph *= ptod;
                double sn, cs;
                sincos(ph, &sn, &cs);
                const float2 z = A[i * RS + j];
                A[i * RS + j] = make_float2((float)(z.x * cs - z.y * sn), (float)(z.x * sn + z.y * cs));
            }
            __syncthreads();
        }
        // ---------------------------------------------------- spectra, cross spectrum
        sbfft::fft2d_smem<W, -1, 2, NT>(A, RS, IMG, twW);
        for (int e = tid; e < W * W; e += NT) {
            const int i = e / W, j = e % W;
            A[i * RS + j] = sbfft::cconjmul(A[i * RS + j], B[i * RS + j]);
        }
        __syncthreads();
        // ---------------------------------------------------- padded inverse, four parities
        constexpr int EPT = (W * W + NT - 1) / NT;
#pragma unroll 1
        for (int par = 0; par < 4; ++par) {
            const int e1 = par >> 1, e2 = par & 1;
            float2* dst = par < 3 ? B : A;
            if (par < 3) {
                for (int e = tid; e < W * W; e += NT) {
                    const int k1 = e / W, k2 = e % W;
                    float2 v = A[((k1 + azShift) % W) * RS + k2];
                    if (e1) v = sbfft::cmul(v, tau[k1]);
                    if (e2) v = sbfft::cmul(v, tau[k2]);
                    dst[k1 * RS + k2] = v;
                }
            } else {
                float2 hold[EPT];
#pragma unroll
                for (int r = 0; r < EPT; ++r) {
                    const int e = tid + r * NT;
                    if (e < W * W) {
                        const int k1 = e / W, k2 = e % W;
                        float2 v = A[((k1 + azShift) % W) * RS + k2];
                        v = sbfft::cmul(v, tau[k1]);
                        v = sbfft::cmul(v, tau[k2]);
                        hold[r] = v;
                    }
                }
                __syncthreads();
#pragma unroll
                for (int r = 0; r < EPT; ++r) {
                    const int e = tid + r * NT;
                    if (e < W * W) dst[(e / W) * RS + (e % W)] = hold[r];
                }
            }
            __syncthreads();
            sbfft::fft2d_smem<W, 1, 1, NT>(dst, RS, 0, twW);
            float* plane = smf + poff<W>(par);
            if (par < 2) {
                for (int e = tid; e < W * W; e += NT) {
                    const float2 z = dst[(e / W) * RS + (e % W)];
                    plane[e] = sqrtf(z.x * z.x + z.y * z.y);
                }
            } else {
                float hv[EPT];
#pragma unroll
                for (int r = 0; r < EPT; ++r) {
                    const int e = tid + r * NT;
                    if (e < W * W) {
                        const float2 z = dst[(e / W) * RS + (e % W)];
                        hv[r] = sqrtf(z.x * z.x + z.y * z.y);
                    }
                }
                __syncthreads();
#pragma unroll
                for (int r = 0; r < EPT; ++r) {
                    const int e = tid + r * NT;
                    if (e < W * W) plane[e] = hv[r];
                }
            }
            __syncthreads();
        }
        // ---------------------------------------------------- findCPeak
        ArgMax best;
        best.v = 0.f;
        best.rank = 0x7fffffff;
        best.pos = 0;
        for (int e = tid; e < W2 * W2; e += NT) {
            const int y = e / W2, x = e % W2;
            const float v = fmap<W>(smf, y, x);
            const int rk = cpeak_rank(y, x, W);
            if (v > 0.f && am_better(v, rk, best.v, best.rank)) {
                best.v = v;
                best.rank = rk;
                best.pos = e;
            }
        }
        best = block_argmax<NT>(best, isc);
        int iMax = 0, jMax = 0;
        if (best.rank != 0x7fffffff) {
            iMax = best.pos / W2;
            jMax = best.pos % W2;
        }
        double cMax;
        const bool rejected = (iMax < (NFAST / 2) || iMax > (W2 - NFAST / 2) || jMax < (NFAST / 2) ||
                               jMax > (W2 - NFAST / 2));
        int gate = 0;
        if (rejected) {
            cMax = -1.0;
            iMax = -1000;
            jMax = -1000;
        } else {
            // ------------------------------------------------ overSampleC on the 8x8 block
            if (tid < NFAST * NFAST) {
                const int t1 = tid / NFAST, t2 = tid % NFAST;
                blk[tid] = fmap<W>(smf, iMax - NFAST / 2 + t1, jMax - NFAST / 2 + t2);
            }
            __syncthreads();
            const ArgMax ob = oversample_peak<NT>(blk, osA, T, isc);
            const int iMax1 = ob.pos / OSW + (NFAST * NOVER) / 2 - 2 * NOVER;
            const int jMax1 = ob.pos % OSW + (NFAST * NOVER) / 2 - 2 * NOVER;
            cMax = (double)ob.v / (NFAST * NFAST);
            cMax = a.hanCorr * cMax / (sqrt(p1 * p2) * pow((double)(W * W), 2));
            iMax = (iMax * NOVER) + iMax1 - (NOVER * NFAST) / 2;
            jMax = (jMax * NOVER) + jMax1 - (NOVER * NFAST) / 2;
            // ------------------------------------------------ samples for gaussPeak1D x 2
            const int iM = iMax / NOVER, jM = jMax / NOVER;
            gate = (iM - NGAUSS / 2) >= 0 && (iM + NGAUSS / 2) < W2 && (jM - NGAUSS / 2) >= 0 &&
                   (jM + NGAUSS / 2) < W2;
            if (gate && tid < 2 * NGAUSS) {
                const int f = tid / NGAUSS, k = tid % NGAUSS;
                FitJob* fj = &a.fit[it];
                if (f == 0) {
                    fj->samp[0][k] = fmap<W>(smf, iM, jM - NGAUSS / 2 + k);
                } else {
                    fj->samp[1][k] = fmap<W>(smf, iM - NGAUSS / 2 + k, jM);
                }
                if (k == 0) fj->x0[f] = (f == 0 ? jM : iM) - NGAUSS / 2;
            }
        }
        if (tid == 0) {
            PointRec* r = &a.rec[p];
            r->cMax[0] = cMax;
            r->iMax[0] = iMax;
            r->jMax[0] = jMax;
            r->azd = -(float)SB_LARGEINT;  // complexMatch resets aZDefocus (:379)
            r->azset = azShift;
            r->flags |= RF_DONE_C | RF_HD_C | (gate ? RF_GATE_C : 0u);
            a.fit[it].point = p;
            a.fit[it].gate = gate;
        }
        __syncthreads();
    }
}

template <int W, int NT>
static cudaError_t launch_cmplx(const CmplxArgs& a, int nCta, cudaStream_t st)
{
    const size_t sm = CmplxSmem<W, NT>::bytes;
    cudaError_t e = cudaFuncSetAttribute(strack_cmplx_kernel<W, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sm);
    if (e != cudaSuccess) return e;
    strack_cmplx_kernel<W, NT><<<nCta, NT, sm, st>>>(a);
    return cudaGetLastError();
}

template <int W, int NT>
static int occupancy_cmplx()
{
    int nb = 0;
    const size_t sm = CmplxSmem<W, NT>::bytes;
    cudaFuncSetAttribute(strack_cmplx_kernel<W, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, strack_cmplx_kernel<W, NT>, NT, sm);
    return nb;
}

bool cmplx_supported(int W) { return W == 16 || W == 24 || W == 32 || W == 48 || W == 64; }

int cmplx_blocks_per_sm(int W)
{
    switch (W) {
    case 16: return occupancy_cmplx<16, 128>();
    case 24: return occupancy_cmplx<24, 192>();
    case 32: return occupancy_cmplx<32, 256>();
    case 48: return occupancy_cmplx<48, 384>();
    case 64: return occupancy_cmplx<64, 512>();
    default: return 0;
    }
}

cudaError_t launch_strack_cmplx(int W, const CmplxArgs& a, int nCta, cudaStream_t st)
{
    switch (W) {
    case 16: return launch_cmplx<16, 128>(a, nCta, st);
    case 24: return launch_cmplx<24, 192>(a, nCta, st);
    case 32: return launch_cmplx<32, 256>(a, nCta, st);
    case 48: return launch_cmplx<48, 384>(a, nCta, st);
    case 64: return launch_cmplx<64, 512>(a, nCta, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace sbk
