// strack_amp.cu -- amplitude tries of strack (small window s = 1, large
// window s = LA = 2), one CTA per grid point with a per-CTA workspace in
// global memory (L2-resident) staged through shared memory.
//
// Follows getAmpPatches (Strack/speckleTrack.c:1006-1189), ampMatch
// (:398-484) and ampTrackFast (:489-597).  With Ws = wa*s and N = 2*Ws:
//  1. raw Ws x Ws patches -> forward DFTs F1, F2 (estDopCarrier1 first when
//     -noComplex and s = 1);
//  2. detected images |IDFT_N(zeroPadFFT(F, azShift))|^2 * scale, computed as
//     four Ws x Ws parity transforms each (the same regrouping as the complex
//     stage) and packed as z = I1 + i I2;
//  3. zero-count / empty-patch tests, sqrt, mean removal, powers p1, p2;
//  4. one forward N x N DFT of z = a1 + i a2 gives both real spectra
//     (F1[k] = (Z[k] + conj Z[-k])/2, F2[k] = (Z[k] - conj Z[-k])/2i); the
//     cross spectrum S = F1 conj F2 is Hermitian, so S[-k] = conj S[k];
//  5. inverse N x N DFT, |c|, findCPeak, Gaussian widths, 8x8 -> 96x96
//     oversampling of the peak, normalisation by N^4 * 64 * sqrt(p1 p2).
#include <cuda_runtime.h>

#include "strack_device.cuh"
#include "strack_kernels.h"

namespace sbk {

template <int WS>
struct AmpCfg {
    static constexpr int N = 2 * WS;
    static constexpr int NT = WS == 64 ? 384 : 256;  // 12 warps x 80 registers win at 64 only (781 vs 868 ms)
    static constexpr int TILE = sbfft::StagedTile<N, true>::elems > sbfft::StagedTile<WS, true>::elems
                                    ? sbfft::StagedTile<N, true>::elems
                                    : sbfft::StagedTile<WS, true>::elems;  // tile and the out-of-place tileB
    static constexpr size_t smem = sizeof(float2) * (2 * TILE + WS + N + WS + OSW * NFAST + NFAST * OSW) +
                                   sizeof(float) * NFAST * NFAST + sizeof(double) * (NT / 32 + 1) * 8 +
                                   sizeof(int) * (3 * (NT / 32) + 8) + 64;
    // workspace: F1, F2, work (Ws^2 each), z (N^2), mag (N^2 floats)
    static constexpr size_t scratch = (size_t)3 * WS * WS + (size_t)N * N + (size_t)N * N / 2;
    // CTAs per SM: a third at Ws = 128 (large try of window 64: 77.1 against
    // 91.7 ms over 6,894 points of an uncorrelated 2048 x 4096 pair); at
    // Ws = 96 it lost (85.1 against 76.5 ms)
    static constexpr int CTAS = NT == 256 && WS == 128 && 3 * (smem + 1024) <= 228 * 1024 ? 3 : 2;
};

template <int WS, bool GAUSS>
__global__ void __launch_bounds__(AmpCfg<WS>::NT, AmpCfg<WS>::CTAS) strack_amp_kernel(AmpArgs a)
{
    using C = AmpCfg<WS>;
    constexpr int N = C::N, NT = C::NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* tile = reinterpret_cast<float2*>(smem_raw);
    float2* tileB = tile + C::TILE;
    float2* twWs = tileB + C::TILE;
    float2* twN = twWs + WS;
    float2* tau = twN + N;
    float2* osA = tau + WS;
    float2* T = osA + OSW * NFAST;
    float* blk = reinterpret_cast<float*>(T + NFAST * OSW);
    double* red = reinterpret_cast<double*>(blk + NFAST * NFAST);
    int* isc = reinterpret_cast<int*>(red + (NT / 32 + 1) * 8);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    for (int e = tid; e < WS; e += NT) {
        twWs[e] = a.twWs[e];
        tau[e] = a.tau[e];
    }
    for (int e = tid; e < N; e += NT) twN[e] = a.tw2Ws[e];
    for (int e = tid; e < OSW * NFAST; e += NT) osA[e] = a.osA[e];
    __syncthreads();

    float2* F1 = a.scratch + (size_t)blockIdx.x * a.scratchPerCta;
    float2* F2 = F1 + WS * WS;
    float2* work = F2 + WS * WS;
    float2* z = work + WS * WS;
    float* mag = reinterpret_cast<float*>(z + (size_t)N * N);

    const bool isFloat = a.sampleType == SB_CFLOAT32;
    const float thr = isFloat ? 1.0e-15f : 1.0e-6f;
    const float scale = (float)(1. / ((size_t)WS * WS * WS * WS * OS * OS * OS));
    const int st = a.stage;

    const int nList = a.nListDev ? min(a.nList, *a.nListDev) : a.nList;
    for (int it = blockIdx.x; it < nList; it += gridDim.x) {
        const int p = a.list[it];
        const PointPlan pl = a.plan[p];
        // window corners (computeAmpImageLocations, speckleTrack.c:147-156):
        // a1a = aStart + i deltaA - (wA/2) s = a1 + wA/2 - (wA/2) s, from the plan
        const int a1a = pl.a1 + a.wA / 2 - a.wA / 2 * a.s;
        const int r1a = pl.r1 + a.wR / 2 - a.wR / 2 * a.s;
        const int r2a = r1a + (pl.r2 - pl.r1);
        const int a2a = a1a + (pl.a2 - pl.a1);
        // ---------------------------------------------------- raw patches
        double m[4] = {0, 0, 0, 0};
        for (int e = tid; e < WS * WS; e += NT) {
            const int i = e / WS, j = e % WS;
            const float2 z1 = load_sample(a.img1, a.nr1, a1a + i, r1a + j, a.sampleType, a.byteOrder);
            const float2 z2 = load_sample(a.img2, a.nr2, a2a + i, r2a + j, a.sampleType, a.byteOrder);
            F1[e] = z1;
            F2[e] = z2;
            m[0] += z1.x; m[1] += z1.y; m[2] += z2.x; m[3] += z2.y;
        }
        int azShift;
        const bool ownDop = (a.noComplex != 0 && st == 1);
        if (ownDop) {
            // estDopCarrier1(im1in, im2in, wAa, wRa) (speckleTrack.c:1141-1144)
            block_allsum<4, NT>(m, red);
            const double n = (double)(WS * WS);
            const double m1r = m[0] / n, m1i = m[1] / n, m2r = m[2] / n, m2i = m[3] / n;
            double d[4] = {0, 0, 0, 0};
            for (int e = tid; e < (WS - 1) * WS; e += NT) {
                const float2 p0 = F1[e], p1 = F1[e + WS];
                double ar = (double)p1.x - m1r, ai = (double)p1.y - m1i, br = (double)p0.x - m1r,
                       bi = (double)p0.y - m1i;
                d[0] += ar * br + ai * bi;
                d[1] += ai * br - ar * bi;
                const float2 q0 = F2[e], q1 = F2[e + WS];
                ar = (double)q1.x - m2r; ai = (double)q1.y - m2i; br = (double)q0.x - m2r; bi = (double)q0.y - m2i;
                d[2] += ar * br + ai * bi;
                d[3] += ai * br - ar * bi;
            }
            block_allsum<4, NT>(d, red);
            azShift = dop_shift(d[0], d[1], d[2], d[3], a.wAa, a.wA);
        } else {
            azShift = a.azEff ? a.azEff[p] : a.rec[p].azset;
            if (azShift < 0) azShift = 0;
        }
        __syncthreads();
        sbfft::fft2d_staged<WS, -1, NT, true>(F1, tile, twWs, tileB);
        sbfft::fft2d_staged<WS, -1, NT, true>(F2, tile, twWs, tileB);
        const int az = (int)((float)azShift * (float)WS / (float)a.wA);
        // ---------------------------------------------------- detected images
        // Four parity transforms per image as two row passes (rows of F and of
        // F tau; the Doppler roll and tau_e1 commute with the row transform)
        // and four column passes that fold the roll and tau_e1 into their
        // gather and write |c|^2 * scale into component q of z.  The second
        // image's epilogue also counts the samples under the threshold in
        // either image, and each accumulates its own intensity sum.
        double r3[3] = {0, 0, 0};
        {
            float* zf = reinterpret_cast<float*>(z);
            float cnt = 0.f;
            double s1 = 0.0, s2 = 0.0;
#pragma unroll 1
            for (int q = 0; q < 2; ++q) {
                float2* F = q == 0 ? F1 : F2;
                sbfft::staged_rows<WS, 1, NT, true>(
                    work, [F](int r, int k) { return F[(size_t)r * WS + k]; }, tile, tileB, twWs);
                sbfft::staged_rows<WS, 1, NT, true>(
                    F, [F, tau](int r, int k) { return sbfft::cmul(F[(size_t)r * WS + k], tau[k]); }, tile, tileB,
                    twWs);
#pragma unroll 1
                for (int par = 0; par < 4; ++par) {
                    const int e1 = par >> 1, e2 = par & 1;
                    const float2* R = e2 ? F : work;
                    auto src = [R, tau, az, e1](int k, int c) {
                        int r = k + az;
                        r = r >= WS ? r - WS : r;
                        const float2 v = R[(size_t)r * WS + c];
                        return e1 ? sbfft::cmul(v, tau[k]) : v;
                    };
                    auto dst = [zf, scale, e1, e2, q, thr, &cnt, &s1, &s2](int k, int c, float2 v) {
                        const float I = (v.x * v.x + v.y * v.y) * scale;
                        const size_t o = 2 * ((size_t)(2 * k + e1) * N + 2 * c + e2);
                        if (q == 0) {
                            zf[o] = I;
                            s1 += I;
                        } else {
                            zf[o + 1] = I;
                            s2 += I;
                            cnt += (zf[o] < thr || I < thr) ? 1.f : 0.f;
                        }
                    };
                    sbfft::staged_cols<WS, 1, NT, true>(src, dst, tile, tileB, twWs);
                }
            }
            r3[0] = cnt;
            r3[1] = s1;
            r3[2] = s2;
        }
        block_allsum<3, NT>(r3, red);
        const bool hd = !(r3[0] > 20.0) && !(r3[1] < 1.0e-6 || r3[2] < 1.0e-6);
        if (!hd) {
            if (tid == 0) {
                a.rec[p].flags |= (st == 1 ? RF_DONE_S : RF_DONE_L);
                if (ownDop) a.rec[p].azset = azShift;
                a.fit[it].point = p;
                a.fit[it].gate = -1;  // no data: nothing for the fit kernel to decide
            }
            continue;
        }
        double av[2] = {0, 0};
        for (int e = tid; e < N * N; e += NT) {
            float2 v = z[e];
            v.x = sqrtf(v.x);
            v.y = sqrtf(v.y);
            z[e] = v;
            av[0] += v.x;
            av[1] += v.y;
        }
        block_allsum<2, NT>(av, red);
        const double nn = (double)N * N;
        const double avg1 = av[0] / nn, avg2 = av[1] / nn;
        double pw[2] = {0, 0};
        for (int e = tid; e < N * N; e += NT) {
            float2 v = z[e];
            if (v.x > 1.0e-20f) v.x = (float)((double)v.x - avg1);
            v.y = (float)((double)v.y - avg2);
            z[e] = v;
            pw[0] += (double)(v.x * v.x);
            pw[1] += (double)(v.y * v.y);
        }
        block_allsum<2, NT>(pw, red);
        const double p1 = pw[0] / nn, p2 = pw[1] / nn;
        // ---------------------------------------------------- correlation
        sbfft::fft2d_staged<N, -1, NT, true>(z, tile, twN, tileB);
        for (int e = tid; e < N * N; e += NT) {
            const int k1 = e / N, k2 = e % N;
            const int e2 = ((N - k1) % N) * N + ((N - k2) % N);
            if (e2 < e) continue;
            const float2 Zk = z[e], Zm = z[e2];
            // F1 = (Zk + conj Zm)/2, F2 = (Zk - conj Zm)/(2i)
            const float2 f1 = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
            const float2 f2 = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
            const float2 s = sbfft::cconjmul(f1, f2);
            z[e] = s;
            z[e2] = make_float2(s.x, -s.y);
        }
        __syncthreads();
        sbfft::fft2d_staged<N, 1, NT, true>(z, tile, twN, tileB);
        ArgMax best;
        best.v = 0.f;
        best.rank = 0x7fffffff;
        best.pos = 0;
        for (int e = tid; e < N * N; e += NT) {
            const int cy = e / N, cx = e % N;
            const float2 c = z[e];
            const float v = sqrtf(c.x * c.x + c.y * c.y);
            const int y = cy + WS < N ? cy + WS : cy - WS;  // fftshift
            const int x = cx + WS < N ? cx + WS : cx - WS;
            mag[y * N + x] = v;
            const int rk = cpeak_rank(y, x, WS);
            if (v > 0.f && am_better(v, rk, best.v, best.rank)) {
                best.v = v;
                best.rank = rk;
                best.pos = y * N + x;
            }
        }
        best = block_argmax<NT>(best, isc);
        int iMax = 0, jMax = 0;
        double cMax = (best.rank != 0x7fffffff) ? (double)best.v : 0.0;
        if (best.rank != 0x7fffffff) {
            iMax = best.pos / N;
            jMax = best.pos % N;
        }
        if (iMax < NFAST / 2 || iMax > N - NFAST / 2 || jMax < NFAST / 2 || jMax > N - NFAST / 2) {
            cMax = -1.0;
            iMax = -1000;
            jMax = -1000;
        }
        // samples for the Gaussian widths (gate: speckleTrack.c:538-539, strict)
        const int gate = iMax > NGAUSS / 2 && iMax < N - NGAUSS / 2 && jMax > NGAUSS / 2 && jMax < N - NGAUSS / 2;
        if (gate && tid < 2 * NGAUSS) {
            const int f = tid / NGAUSS, k = tid % NGAUSS;
            FitJob* fj = &a.fit[it];
            if (f == 0)
                fj->samp[0][k] = mag[iMax * N + (jMax - NGAUSS / 2 + k)];
            else
                fj->samp[1][k] = mag[(iMax - NGAUSS / 2 + k) * N + jMax];
            if (k == 0) fj->x0[f] = (f == 0 ? jMax : iMax) - NGAUSS / 2;
        }
        const double cRaw = cMax;
        const int iC = iMax, jC = jMax;
        if (GAUSS && iMax >= -999) {
            // -gauss: cmpTrackGauss on the amplitude plane (:553-557; pScale
            // 16, no hanning correction), unless the fit kernel takes the
            // early return of ampTrackFast
            const double hw = (double)(N / 2) * (double)(N / 2);
            const double scale = 1.0 / (sqrt((p1 * 16.0) * (p2 * 16.0)) * pow(hw, 2));
            gauss2d_peak<NT>([=](int i, int j) { return mag[i * N + j]; }, N, scale, reinterpret_cast<float*>(T), blk, iMax,
                             jMax, cMax);
        } else if (iMax >= -999) {
            // 8x8 -> 96x96 oversampling (used unless the fit kernel takes the
            // early return of ampTrackFast, :551-553)
            if (tid < NFAST * NFAST) {
                const int t1 = tid / NFAST, t2 = tid % NFAST;
                blk[tid] = mag[(iMax - NFAST / 2 + t1) * N + (jMax - NFAST / 2 + t2)];
            }
            __syncthreads();
            const ArgMax ob = oversample_peak<NT>(blk, osA, T, isc);
            const int iMax1 = ob.pos / OSW + (NFAST * NOVER) / 2 - 2 * NOVER;
            const int jMax1 = ob.pos % OSW + (NFAST * NOVER) / 2 - 2 * NOVER;
            cMax = (double)ob.v;
            cMax = cMax / (pow((double)N, 2) * pow((double)N, 2) * pow((double)NFAST, 2));
            cMax = cMax / sqrt(p1 * p2);
            iMax = (iMax * NOVER) + iMax1 - (NOVER * NFAST) / 2;
            jMax = (jMax * NOVER) + jMax1 - (NOVER * NFAST) / 2;
        }
        if (tid == 0) {
            PointRec* r = &a.rec[p];
            r->cMax[st] = cMax;
            r->iMax[st] = iMax;
            r->jMax[st] = jMax;
            r->cRaw = cRaw;
            r->iC = iC;
            r->jC = jC;
            if (ownDop) r->azset = azShift;
            r->azUsed = azShift;
            r->flags |= (st == 1 ? (RF_DONE_S | RF_HD_S) : (RF_DONE_L | RF_HD_L));
            a.fit[it].point = p;
            a.fit[it].gate = gate;
        }
        __syncthreads();
    }
}

template <int WS, bool GAUSS>
static cudaError_t launch_amp_t(const AmpArgs& a, int nCta, cudaStream_t st)
{
    using C = AmpCfg<WS>;
    cudaError_t e = cudaFuncSetAttribute(strack_amp_kernel<WS, GAUSS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)C::smem);
    if (e != cudaSuccess) return e;
    strack_amp_kernel<WS, GAUSS><<<nCta, C::NT, C::smem, st>>>(a);
    return cudaGetLastError();
}

template <int WS>
static cudaError_t launch_amp(const AmpArgs& a, int nCta, cudaStream_t st)
{
    return a.gauss ? launch_amp_t<WS, true>(a, nCta, st) : launch_amp_t<WS, false>(a, nCta, st);
}

bool amp_supported(int Ws)
{
    return Ws == 16 || Ws == 24 || Ws == 32 || Ws == 48 || Ws == 64 || Ws == 96 || Ws == 128;
}

size_t amp_scratch_elems(int Ws)
{
    switch (Ws) {
    case 16: return AmpCfg<16>::scratch;
    case 24: return AmpCfg<24>::scratch;
    case 32: return AmpCfg<32>::scratch;
    case 48: return AmpCfg<48>::scratch;
    case 64: return AmpCfg<64>::scratch;
    case 96: return AmpCfg<96>::scratch;
    case 128: return AmpCfg<128>::scratch;
    default: return 0;
    }
}

int amp_threads(int) { return 256; }

int amp_blocks_per_sm(int Ws)
{
    switch (Ws) {
    case 16: return AmpCfg<16>::CTAS;
    case 24: return AmpCfg<24>::CTAS;
    case 32: return AmpCfg<32>::CTAS;
    case 48: return AmpCfg<48>::CTAS;
    case 64: return AmpCfg<64>::CTAS;
    case 96: return AmpCfg<96>::CTAS;
    case 128: return AmpCfg<128>::CTAS;
    default: return 2;
    }
}

cudaError_t launch_strack_amp(int Ws, const AmpArgs& a, int nCta, cudaStream_t st)
{
    switch (Ws) {
    case 16: return launch_amp<16>(a, nCta, st);
    case 24: return launch_amp<24>(a, nCta, st);
    case 32: return launch_amp<32>(a, nCta, st);
    case 48: return launch_amp<48>(a, nCta, st);
    case 64: return launch_amp<64>(a, nCta, st);
    case 96: return launch_amp<96>(a, nCta, st);
    case 128: return launch_amp<128>(a, nCta, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace sbk
