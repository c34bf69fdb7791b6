// strackw.cu -- corrTrackFast (Strackw/corrTrackFast.c:89-231) on the GPU:
// one CTA per grid point, per-CTA workspace in global memory staged through
// shared-memory tiles.
//
// Per point (W = wRa = wAa, N = 2W, E = edgePad + NFAST/4):
//  1. W x W raw patches of both images; estDopCarrier1 on them (:340);
//  2. forward W x W DFTs, zeroPad with the azimuth roll (:718-761) and the
//     N x N inverse, done as four W x W parity transforms per image; the
//     intensity |z|^2 * scale is kept (float), as detectPatch takes it;
//  3. detectPatch (:765-839): optional (2 navg + 1)^2 box sums in float in the
//     reference's order and clamps (the small chip's azimuth clamp uses
//     edgePadR, as in the reference), sqrt; the chip of image 2 is embedded in
//     zeros, image 1 is the full search area;
//  4. computeMeanSigma (:407-477): chip mean/variance and the search window's
//     mean/variance at every one of the (4E+1)^2 placements, in double, from
//     row and column prefix sums;
//  5. ampMatchEdge (:903-947): one forward N x N DFT of (search + i chip), the
//     Hermitian cross spectrum, one inverse; with both images' means removed
//     first, the result is the covariance term of getPeakCorr directly
//     (an exact identity that avoids the float cancellation of
//     c*scaleW - meanR*meanS);
//  6. getPeakCorr (:862-899): normalised correlation on the (4E+1)^2 lags,
//     argmax inside the user radius (row-major first maximum);
//  7. overSampleC (:951-990): the 21 x 21 block's symmetric zero pad to
//     336 x 336 evaluated on the searched 64 x 64 window only, as B X B^T with
//     the real kernel B[n][t] = 1 + 2 sum_{f=1..10} cos(2 pi f (n - 16 t)/336),
//     in double; cMax = sqrt(max |.|^2)/441, shifts in 1/32 px.
// Windows whose far edge leaves the image (the reference checks only the
// near corner, :170-171, then reads stale buffer rows) read zeros here.
#include <cuda_runtime.h>

#include <vector>

#include "capi_internal.h"
#include "strack_device.cuh"

namespace sbk {

constexpr int W_NOVER = 16;  // corrTrackFast.c:11
constexpr int W_NFAST = 20;  // corrTrackFast.c:12
constexpr int W_N1 = W_NFAST + 1;
constexpr int W_OSW = 64;    // searched window [168-32, 168+32)

struct SwArgs {
    const void* img1;
    const void* img2;
    int nr1, na1, nr2, na2;
    int sampleType, byteOrder;
    const int4* plan;  // r1, a1, r2, a2 of the points to match
    const int* list;   // grid index of each entry
    int nList;
    int eR, eA;        // edge pads including the internal +5
    int navgR, navgA;
    float scale;
    float2* scratch;
    size_t perCta;     // float2 elements
    const double* B;   // 64 x 21 oversampling kernel
    float* offR;
    float* offA;
    float* corr;
    uint8_t* type;
    unsigned long long* stats;  // [0] matched, [1] failed
};

struct DArg {
    double v;
    int rank;
};
__device__ __forceinline__ bool darg_better(double v, int r, double bv, int br)
{
    return v > bv || (v == bv && r < br);
}
template <int NT>
__device__ __forceinline__ DArg block_argmax_d(DArg a, double* dsc, int* isc)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double v = __shfl_xor_sync(0xffffffffu, a.v, o);
        const int r = __shfl_xor_sync(0xffffffffu, a.rank, o);
        if (darg_better(v, r, a.v, a.rank)) {
            a.v = v;
            a.rank = r;
        }
    }
    if (lane == 0) {
        dsc[warp] = a.v;
        isc[warp] = a.rank;
    }
    __syncthreads();
    DArg b;
    b.v = dsc[0];
    b.rank = isc[0];
    for (int w = 1; w < NT / 32; ++w)
        if (darg_better(dsc[w], isc[w], b.v, b.rank)) {
            b.v = dsc[w];
            b.rank = isc[w];
        }
    __syncthreads();
    return b;
}

__device__ __forceinline__ float2 sw_sample(const void* img, int nr, int na, int row, int col, int st, int bo)
{
    if (row < 0 || row >= na || col < 0 || col >= nr) return make_float2(0.f, 0.f);
    return load_sample(img, nr, row, col, st, bo);
}

template <int W>
struct SwCfg {
    static constexpr int N = 2 * W;
    // 256 threads with three CTAs per SM from W = 96 to 192 (a third CTA
    // beat 384 threads at two: 32.1 against 40.0 ms at W = 128, 76.4 against
    // 79.2 at 192 on the 2000 x 4000 shear pair); 384 threads at two CTAs at
    // 224 and 256 (114.3 against 116.9 ms at 224)
    static constexpr int NT = W >= 224 ? 384 : 256;
    static constexpr int TILE = sbfft::StagedTile<N, true>::elems > sbfft::StagedTile<W, true>::elems
                                    ? sbfft::StagedTile<N, true>::elems
                                    : sbfft::StagedTile<W, true>::elems;
    static constexpr int TILEB = TILE;  // out-of-place tile of the three-step transforms
    // oversampling kernel B (64 x 21), block X (21 x 21) and T (21 x 64), doubles
    static constexpr int OSD = W_OSW * W_N1 + W_N1 * W_N1 + W_N1 * W_OSW;
    // from W = 96 up they live in the (then idle) tiles, so that three CTAs fit an SM
    static constexpr bool OS_IN_TILE = 2 * TILE >= OSD;
    static constexpr size_t smem = sizeof(float2) * (TILE + TILEB + W + N + W) +
                                   (OS_IN_TILE ? 0 : sizeof(double) * OSD) + sizeof(double) * (NT / 32 + 1) * 8 +
                                   sizeof(int) * (3 * (NT / 32) + 8) + 64;
    // CTAs per SM (228 KB of shared memory, 1 KB reserved per CTA)
    static constexpr int CTAS = W >= 96 && W <= 192 && OS_IN_TILE && 3 * (smem + 1024) <= 228 * 1024 ? 3 : 2;
    static_assert((NT / 32) * 2 * N <= W * W, "per-warp prefix slices must fit in `work`");
    // workspace (float2 units): F1, F2, work (W^2 each), I1, I2 (N^2 floats
    // each), z (N^2), row sums RS1, RS2 (N x L doubles each), meanS, sigmaS,
    // ncc (L^2 doubles each) with L = 4E + 1, then H1, H2 (N^2 floats each)
    static size_t perCta(int L)
    {
        return (size_t)3 * W * W + (size_t)N * N + (size_t)N * N + (size_t)2 * N * L + (size_t)3 * L * L +
               (size_t)N * N + 64;
    }
};

template <int W>
__global__ void __launch_bounds__(SwCfg<W>::NT, SwCfg<W>::CTAS) strackw_kernel(SwArgs a)
{
    using C = SwCfg<W>;
    constexpr int N = C::N, NT = C::NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* tile = reinterpret_cast<float2*>(smem_raw);
    float2* tileB = tile + C::TILE;
    float2* twW = tileB + C::TILEB;
    float2* twN = twW + W;
    float2* tau = twN + N;
    double* osBase = C::OS_IN_TILE ? reinterpret_cast<double*>(tile) : reinterpret_cast<double*>(tau + W);
    double* Bm = osBase;                                    // 64 x 21
    double* X = Bm + W_OSW * W_N1;                          // 21 x 21 block
    double* T = X + W_N1 * W_N1;                            // 21 x 64
    double* red = C::OS_IN_TILE ? reinterpret_cast<double*>(tau + W) : T + W_N1 * W_OSW;
    int* isc = reinterpret_cast<int*>(red + (NT / 32 + 1) * 8);
    const int tid = threadIdx.x;

    for (int e = tid; e < W; e += NT) {
        double s, c;
        sincospi(-2.0 * e / W, &s, &c);
        twW[e] = make_float2((float)c, (float)s);
        sincospi((double)e / W, &s, &c);
        const double sg = e < W / 2 ? 1.0 : -1.0;
        tau[e] = make_float2((float)(sg * c), (float)(sg * s));
    }
    for (int e = tid; e < N; e += NT) {
        double s, c;
        sincospi(-2.0 * e / N, &s, &c);
        twN[e] = make_float2((float)c, (float)s);
    }
    if constexpr (!C::OS_IN_TILE)
        for (int e = tid; e < W_OSW * W_N1; e += NT) Bm[e] = a.B[e];
    __syncthreads();

    const int eR = a.eR, eA = a.eA;
    const int L = 4 * eR + 1, LA = 4 * eA + 1;  // lags (range, azimuth)
    const int wR2 = (W - 2 * eR) * OS, wA2 = (W - 2 * eA) * OS;
    float2* F1 = a.scratch + (size_t)blockIdx.x * a.perCta;
    float2* F2 = F1 + W * W;
    float2* work = F2 + W * W;
    float* I1 = reinterpret_cast<float*>(work + W * W);
    float* I2 = I1 + (size_t)N * N;
    float2* z = reinterpret_cast<float2*>(I2 + (size_t)N * N);
    double* RS1 = reinterpret_cast<double*>(z + (size_t)N * N);
    double* RS2 = RS1 + (size_t)N * L;
    double* meanS = RS2 + (size_t)N * L;
    double* sigmaS = meanS + (size_t)LA * L;
    double* ncc = sigmaS + (size_t)LA * L;
    float* H1 = reinterpret_cast<float*>(ncc + (size_t)LA * L);
    float* H2 = H1 + (size_t)N * N;
    const bool smooth = a.navgA > 1 || a.navgR > 1;

    for (int it = blockIdx.x; it < a.nList; it += gridDim.x) {
        const int4 pl = a.plan[it];  // r1, a1, r2, a2
        // ------------------------------------------------ patches, Doppler
        double m[4] = {0, 0, 0, 0};
        for (int e = tid; e < W * W; e += NT) {
            const int i = e / W, j = e % W;
            const float2 z1 = sw_sample(a.img1, a.nr1, a.na1, pl.y + i, pl.x + j, a.sampleType, a.byteOrder);
            const float2 z2 = sw_sample(a.img2, a.nr2, a.na2, pl.w + i, pl.z + j, a.sampleType, a.byteOrder);
            F1[e] = z1;
            F2[e] = z2;
            m[0] += z1.x; m[1] += z1.y; m[2] += z2.x; m[3] += z2.y;
        }
        block_allsum<4, NT>(m, red);
        {
            const double n = (double)(W * W);
            const double m1r = m[0] / n, m1i = m[1] / n, m2r = m[2] / n, m2i = m[3] / n;
            double d[4] = {0, 0, 0, 0};
            for (int e = tid; e < (W - 1) * W; e += NT) {
                const float2 p0 = F1[e], p1 = F1[e + W];
                double ar = (double)p1.x - m1r, ai = (double)p1.y - m1i, br = (double)p0.x - m1r,
                       bi = (double)p0.y - m1i;
                d[0] += ar * br + ai * bi;
                d[1] += ai * br - ar * bi;
                const float2 q0 = F2[e], q1 = F2[e + W];
                ar = (double)q1.x - m2r; ai = (double)q1.y - m2i; br = (double)q0.x - m2r; bi = (double)q0.y - m2i;
                d[2] += ar * br + ai * bi;
                d[3] += ai * br - ar * bi;
            }
            block_allsum<4, NT>(d, red);
            m[0] = (double)dop_shift(d[0], d[1], d[2], d[3], W, W);
        }
        int da = (int)m[0];
        if (da < 0 || da >= W) da = 0;
        sbfft::fft2d_staged<W, -1, NT, true>(F1, tile, twW, tileB);
        sbfft::fft2d_staged<W, -1, NT, true>(F2, tile, twW, tileB);
        // ------------------------------------------------ upsampled intensities
        // The 2W x 2W padded inverse as four parity transforms
        // c_e[m1][m2] = IDFT_W(X' tau_e1[k1] tau_e2[k2]), X'[k1] = F[(k1 + da) mod W]:
        // the row factor tau_e1 and the row roll commute with the row
        // transform, so two unrolled row passes (R0 = rows of F, R1 = rows of
        // F tau) serve the four parities, and each column pass reads its R with
        // the roll and tau_e1 folded into the gather and writes |c|^2 * scale
        // straight into the intensity plane.
        // intensity columns of image 2 that detectPatch reads: the chip
        // [eR OS, eR OS + wR2) widened by the range box sum (navgR) and one
        // column of slack, as parity-plane columns
        constexpr int GW = sbfft::StagedTile<W, true>::G;
        const int cLo = max(0, eR * OS - a.navgR - 1) / 2;
        const int cHi = min(N - 1, eR * OS + wR2 + a.navgR) / 2;
#pragma unroll 1
        for (int q = 0; q < 2; ++q) {
            float2* F = q == 0 ? F1 : F2;
            float* I = q == 0 ? I1 : I2;
            const float sc = a.scale;
            sbfft::staged_rows<W, 1, NT, true>(
                work, [F](int r, int k) { return F[(size_t)r * W + k]; }, tile, tileB, twW);
            sbfft::staged_rows<W, 1, NT, true>(
                F, [F, tau](int r, int k) { return sbfft::cmul(F[(size_t)r * W + k], tau[k]); }, tile, tileB, twW);
#pragma unroll 1
            for (int par = 0; par < 4; ++par) {
                const int e1 = par >> 1, e2 = par & 1;
                const float2* R = e2 ? F : work;
                auto src = [R, tau, da, e1](int k, int c) {
                    int r = k + da;
                    r = r >= W ? r - W : r;
                    const float2 v = R[(size_t)r * W + c];
                    return e1 ? sbfft::cmul(v, tau[k]) : v;
                };
                auto dst = [I, sc, e1, e2](int k, int c, float2 v) {
                    I[(size_t)(2 * k + e1) * N + 2 * c + e2] = (v.x * v.x + v.y * v.y) * sc;
                };
                // the chip (image 2) reads only the intensity columns of the
                // chip and its box-sum margin: column c of a parity plane
                // lands in intensity columns 2c and 2c + 1, so tiles of c
                // outside [cLo, cHi] are skipped (image 1: every column)
                sbfft::staged_cols_if<W, 1, NT, true>(
                    src, dst, [q, cLo, cHi](int c0) { return q == 0 || (c0 + GW - 1 >= cLo && c0 <= cHi); }, tile,
                    tileB, twW);
            }
        }
        // ------------------------------------------------ detectPatch
        // The (2 navg + 1)^2 box sums are separable: range sums into H1/H2
        // first, then azimuth sums of those, with the reference's clamps
        // (image 1: the N x N area; the chip: kmax/lmax, the azimuth limit
        // built from edgePadR as at :795).
        const int kmax = eR * OS + wA2 + a.navgA - 1;
        const int lmax = eR * OS + wR2 + a.navgR - 1;
        if (smooth) {
            // the chip's azimuth sums read H2 only on rows clamp(i + m, 0,
            // kmax) of the chip rows i and on the chip columns: H2 is formed
            // there (one row and column of slack), H1 everywhere
            const int hr0 = max(0, min(kmax, eA * OS - a.navgA) - 1);
            const int hr1 = min(N - 1, min(kmax, eA * OS + wA2 - 1 + a.navgA) + 1);
            const int hc0 = max(0, eR * OS - 1), hc1 = min(N - 1, eR * OS + wR2);
            for (int e = tid; e < N * N; e += NT) {
                const int i = e / N, j = e % N;
                const bool need2 = i >= hr0 && i <= hr1 && j >= hc0 && j <= hc1;
                float h1 = 0.f, h2 = 0.f;
                for (int nn = -a.navgR; nn <= a.navgR; nn++) {
                    int l = j + nn;
                    l = l > 0 ? l : 0;
                    const int l1 = l < N - 1 ? l : N - 1;
                    const int l2 = l < lmax ? l : lmax;
                    h1 += I1[(size_t)i * N + l1];
                    if (need2) h2 += I2[(size_t)i * N + l2];
                }
                H1[e] = h1;
                if (need2) H2[e] = h2;
            }
            __syncthreads();
        }
        double cs[3] = {0, 0, 0};
        for (int e = tid; e < N * N; e += NT) {
            const int i = e / N, j = e % N;
            // large patch (image 1): edge pads 0, clamps to the N x N area
            float v1;
            if (smooth) {
                float acc = 0.f;
                for (int mm = -a.navgA; mm <= a.navgA; mm++) {
                    int k = i + mm;
                    k = k > 0 ? k : 0;
                    k = k < N - 1 ? k : N - 1;
                    acc += H1[(size_t)k * N + j];
                }
                v1 = acc;
            } else {
                v1 = I1[e];
            }
            // small chip (image 2) embedded in zeros
            float v2 = 0.f;
            const int ci = i - eA * OS, cj = j - eR * OS;
            if (ci >= 0 && ci < wA2 && cj >= 0 && cj < wR2) {
                if (smooth) {
                    float acc = 0.f;
                    for (int mm = -a.navgA; mm <= a.navgA; mm++) {
                        int k = i + mm;
                        k = k > 0 ? k : 0;
                        k = k < kmax ? k : kmax;
                        acc += H2[(size_t)k * N + j];
                    }
                    v2 = acc;
                } else {
                    v2 = I2[e];
                }
                v2 = sqrtf(v2);
                cs[0] += v2;
                cs[1] += (double)(v2 * v2);
            }
            v1 = sqrtf(v1);
            cs[2] += v1;
            z[e] = make_float2(v1, v2);
        }
        block_allsum<3, NT>(cs, red);
        const double nchip = (double)(wR2 * wA2);
        const double meanR = cs[0] / nchip;
        const double sigmaR = cs[1] / (double)(wR2 * wA2 - 1.) - meanR * meanR;
        // ------------------------------------------------ search-window statistics
        // RS[l][s1] = sum_{s = s1 .. s1 + wR2 - 1} A1[l][s] (and of A1^2), one warp per row
        {
            const int lane = tid & 31, warp = tid >> 5;
            double* Pw = reinterpret_cast<double*>(work) + (size_t)warp * 2 * N;  // 16 N bytes per warp
            for (int row = warp; row < N; row += NT / 32) {
                double c1 = 0, c2 = 0;  // running carry of the prefix scan
                // prefix sums computed in chunks of 32 columns
                for (int base = 0; base < N; base += 32) {
                    const int s = base + lane;
                    const float x = z[(size_t)row * N + s].x;
                    double p1 = x, p2 = (double)(x * x);
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const double t1 = __shfl_up_sync(0xffffffffu, p1, o);
                        const double t2 = __shfl_up_sync(0xffffffffu, p2, o);
                        if (lane >= o) {
                            p1 += t1;
                            p2 += t2;
                        }
                    }
                    p1 += c1;
                    p2 += c2;
                    Pw[2 * s] = p1;  // inclusive prefix, this warp's slice of `work`
                    Pw[2 * s + 1] = p2;
                    c1 = __shfl_sync(0xffffffffu, p1, 31);
                    c2 = __shfl_sync(0xffffffffu, p2, 31);
                }
                __syncwarp();
                for (int s1 = lane; s1 < L; s1 += 32) {
                    const double* P = Pw;
                    const int hi = s1 + wR2 - 1;
                    const double a1 = P[2 * hi] - (s1 > 0 ? P[2 * (s1 - 1)] : 0.0);
                    const double a2 = P[2 * hi + 1] - (s1 > 0 ? P[2 * (s1 - 1) + 1] : 0.0);
                    RS1[(size_t)row * L + s1] = a1;
                    RS2[(size_t)row * L + s1] = a2;
                }
                __syncwarp();
            }
            __syncthreads();
        }
        // column prefix sums of the row-window sums (one thread per lag column;
        // rows unrolled so the loads run ahead of the dependent adds), then the
        // wA2-row window of every placement as a difference of two prefixes
        for (int s1 = tid; s1 < L; s1 += NT) {
            double c1 = 0.0, c2 = 0.0;
            int l = 0;
            for (; l + 8 <= N; l += 8) {
                double v1[8], v2[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    v1[u] = RS1[(size_t)(l + u) * L + s1];
                    v2[u] = RS2[(size_t)(l + u) * L + s1];
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    c1 += v1[u];
                    c2 += v2[u];
                    RS1[(size_t)(l + u) * L + s1] = c1;
                    RS2[(size_t)(l + u) * L + s1] = c2;
                }
            }
            for (; l < N; ++l) {
                c1 += RS1[(size_t)l * L + s1];
                c2 += RS2[(size_t)l * L + s1];
                RS1[(size_t)l * L + s1] = c1;
                RS2[(size_t)l * L + s1] = c2;
            }
        }
        __syncthreads();
        for (int e = tid; e < LA * L; e += NT) {
            const int l1 = e / L, s1 = e % L;
            const size_t hi = (size_t)(l1 + wA2 - 1) * L + s1, lo = (size_t)(l1 - 1) * L + s1;
            const double a1 = RS1[hi] - (l1 > 0 ? RS1[lo] : 0.0);
            const double a2 = RS2[hi] - (l1 > 0 ? RS2[lo] : 0.0);
            const double ms = a1 / nchip;
            meanS[e] = ms;
            sigmaS[e] = a2 / (double)(wR2 * wA2 - 1) - ms * ms;
        }
        __syncthreads();
        // ------------------------------------------------ correlation
        // getPeakCorr forms c*scaleW - meanR*meanS with c the correlation of
        // the raw amplitudes; both terms are ~mean^2 and their difference is
        // the covariance.  Correlating the chip minus its mean (on its
        // support) with the search image minus its global mean gives that
        // difference directly, because sum(chip - meanR) = 0 over the support:
        //   sum_x (chip[x] - meanR)(A1[x+t] - mA1) = c[t] - meanR * n * meanS[t].
        // Same quantity, without the float cancellation.
        // The mean removal is folded into the forward row pass; the Hermitian
        // split of the packed pair and the cross spectrum into the inverse row
        // pass, which reads Z[k] and Z[-k] and writes out of place into the
        // free H1/H2 area (Zi); the last column pass keeps only the lag rows
        // and columns getPeakCorr reads.
        {
            const float mA1 = (float)(cs[2] / ((double)N * N));
            const float mR = (float)meanR;
            const int cA = eA * OS, cR = eR * OS;
            auto srcFwd = [z, mA1, mR, cA, cR, wA2, wR2](int r, int k) {
                float2 v = z[(size_t)r * N + k];
                const int ci = r - cA, cj = k - cR;
                const bool in = ci >= 0 && ci < wA2 && cj >= 0 && cj < wR2;
                v.x -= mA1;
                v.y = in ? v.y - mR : 0.f;
                return v;
            };
            sbfft::staged_rows<N, -1, NT, true>(z, srcFwd, tile, tileB, twN);
            sbfft::staged_cols<N, -1, NT, true>([z](int k, int c) { return z[(size_t)k * N + c]; },
                                                [z](int k, int c, float2 v) { z[(size_t)k * N + c] = v; }, tile,
                                                tileB, twN);
        }
        float2* Zi = reinterpret_cast<float2*>(H1);
        {
            auto srcInv = [z](int r, int k) {
                const float2 Zk = z[(size_t)r * N + k];
                const float2 Zm = z[(size_t)(r == 0 ? 0 : N - r) * N + (k == 0 ? 0 : N - k)];
                const float2 f1 = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
                const float2 f2 = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
                return sbfft::cconjmul(f1, f2);
            };
            sbfft::staged_rows<N, 1, NT, true>(Zi, srcInv, tile, tileB, twN);
            const int nLo = LA - OS * eA, nHi = N - OS * eA;  // lag rows/cols used: [0, nLo) and [nHi, N)
            auto need = [nLo, nHi](int x) { return x < nLo || x >= nHi; };
            // tiles of columns that hold no lag are not transformed
            constexpr int GN = sbfft::StagedTile<N, true>::G;
            sbfft::staged_cols_if<N, 1, NT, true>([Zi](int k, int c) { return Zi[(size_t)k * N + c]; },
                                                  [Zi, need](int k, int c, float2 v) {
                                                      if (need(k) && need(c)) Zi[(size_t)k * N + c] = v;
                                                  },
                                                  [nLo, nHi](int c0) { return c0 < nLo || c0 + GN - 1 >= nHi; },
                                                  tile, tileB, twN);
        }
        // ------------------------------------------------ getPeakCorr
        const double wR2p = W - 2 * eR, wA2p = W - 2 * eA;
        const double scaleW = 1.0 / ((OS * OS * OS * OS) * W * wA2p * W * wR2p);
        const int lim = OS * (eA - W_NFAST / 4), limR = OS * (eR - W_NFAST / 4);
        DArg best;
        best.v = -1e30;
        best.rank = 0x7fffffff;
        for (int e = tid; e < LA * L; e += NT) {
            const int i = e / L, j = e % L;
            const int l = i - OS * eA, s = j - OS * eR;
            const int cy = l < 0 ? l + N : l, cx = s < 0 ? s + N : s;
            const float2 c = Zi[(size_t)cy * N + cx];
            double v = (double)c.x * scaleW;  // = |c| * scaleW - meanR * meanS (the covariance)
            v = v / sqrt(sigmaR * sigmaS[e]);
            ncc[e] = v;
            if (l >= -lim && s >= -limR && l <= lim && s <= limR && darg_better(v, e, best.v, best.rank)) {
                best.v = v;
                best.rank = e;
            }
        }
        best = block_argmax_d<NT>(best, red, isc);
        const int gidx = a.list[it];
        if (!(best.v >= 0.0) || best.rank == 0x7fffffff) {  // maxCorr < 0: no match (:511-512)
            if (tid == 0) {
                a.offR[gidx] = -2.0e9f;
                a.offA[gidx] = -2.0e9f;
                a.corr[gidx] = 0.0f;
                a.type[gidx] = SB_AMPMATCH;
                atomicAdd(&a.stats[1], 1ull);
            }
            __syncthreads();
            continue;
        }
        const int iMax = best.rank / L, jMax = best.rank % L;
        if constexpr (C::OS_IN_TILE)  // the tiles are idle until the next point's transforms
            for (int e = tid; e < W_OSW * W_N1; e += NT) Bm[e] = __ldg(a.B + e);
        for (int e = tid; e < W_N1 * W_N1; e += NT) {
            const int bi = e / W_N1, bj = e % W_N1;
            X[e] = ncc[(size_t)(iMax - W_NFAST / 2 + bi) * L + (jMax - W_NFAST / 2 + bj)];
        }
        __syncthreads();
        // T[t1][n2] = sum_t2 X[t1][t2] B[n2][t2]
        for (int e = tid; e < W_N1 * W_OSW; e += NT) {
            const int t1 = e / W_OSW, n2 = e % W_OSW;
            double acc = 0.0;
            for (int t2 = 0; t2 < W_N1; ++t2) acc += X[t1 * W_N1 + t2] * Bm[n2 * W_N1 + t2];
            T[e] = acc;
        }
        __syncthreads();
        DArg ob;
        ob.v = -1.0e30;
        ob.rank = 0x7fffffff;
        for (int e = tid; e < W_OSW * W_OSW; e += NT) {
            const int n1 = e / W_OSW, n2 = e % W_OSW;
            double acc = 0.0;
            for (int t1 = 0; t1 < W_N1; ++t1) acc += Bm[n1 * W_N1 + t1] * T[t1 * W_OSW + n2];
            const double v = acc * acc;
            if (darg_better(v, e, ob.v, ob.rank)) {
                ob.v = v;
                ob.rank = e;
            }
        }
        ob = block_argmax_d<NT>(ob, red, isc);
        if (tid == 0) {
            const int c0 = (W_N1 * W_NOVER) / 2 - W_NOVER * 2;  // 136
            const int iMax1 = ob.rank / W_OSW + c0, jMax1 = ob.rank % W_OSW + c0;
            const float cMax = (float)(sqrt(ob.v) / (W_N1 * W_N1));
            const int iMo = iMax * W_NOVER + iMax1 - (W_NOVER * W_NFAST) / 2;
            const int jMo = jMax * W_NOVER + jMax1 - (W_NOVER * W_NFAST) / 2;
            const float rShift1 = ((float)jMo - eR * OS * W_NOVER) / (W_NOVER * OS);
            const float aShift1 = ((float)iMo - eA * OS * W_NOVER) / (W_NOVER * OS);
            const float rShift = (float)(pl.z - pl.x), aShift = (float)(pl.w - pl.y);
            if (cMax > 0.0f) {
                a.offR[gidx] = rShift - rShift1;
                a.offA[gidx] = aShift - aShift1;
                atomicAdd(&a.stats[0], 1ull);
            } else {
                a.offR[gidx] = -2.0e9f;
                a.offA[gidx] = -2.0e9f;
                atomicAdd(&a.stats[1], 1ull);
            }
            a.corr[gidx] = cMax;
            a.type[gidx] = SB_AMPMATCH;
        }
        __syncthreads();
    }
}

__global__ void strackw_init_kernel(float* offR, float* offA, float* corr, uint8_t* type, int n)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    offR[k] = -2.0e9f;
    offA[k] = -2.0e9f;
    corr[k] = 0.0f;
    type[k] = SB_BAD;
}

template <int W>
static cudaError_t launch_sw(const SwArgs& a, int nCta, cudaStream_t st)
{
    using C = SwCfg<W>;
    cudaError_t e = cudaFuncSetAttribute(strackw_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem);
    if (e != cudaSuccess) return e;
    strackw_kernel<W><<<nCta, C::NT, C::smem, st>>>(a);
    return cudaGetLastError();
}

static int sw_ctas(int W)
{
    switch (W) {
    case 32: return SwCfg<32>::CTAS;
    case 48: return SwCfg<48>::CTAS;
    case 64: return SwCfg<64>::CTAS;
    case 96: return SwCfg<96>::CTAS;
    case 128: return SwCfg<128>::CTAS;
    case 192: return SwCfg<192>::CTAS;
    case 224: return SwCfg<224>::CTAS;
    default: return SwCfg<256>::CTAS;
    }
}

static bool sw_supported(int W)
{
    return W == 32 || W == 48 || W == 64 || W == 96 || W == 128 || W == 192 || W == 224 || W == 256;
}
static size_t sw_per_cta(int W, int L)
{
    switch (W) {
    case 32: return SwCfg<32>::perCta(L);
    case 48: return SwCfg<48>::perCta(L);
    case 64: return SwCfg<64>::perCta(L);
    case 96: return SwCfg<96>::perCta(L);
    case 128: return SwCfg<128>::perCta(L);
    case 192: return SwCfg<192>::perCta(L);
    case 224: return SwCfg<224>::perCta(L);
    default: return SwCfg<256>::perCta(L);
    }
}
static cudaError_t launch_sw_any(int W, const SwArgs& a, int nCta, cudaStream_t st)
{
    switch (W) {
    case 32: return launch_sw<32>(a, nCta, st);
    case 48: return launch_sw<48>(a, nCta, st);
    case 64: return launch_sw<64>(a, nCta, st);
    case 96: return launch_sw<96>(a, nCta, st);
    case 128: return launch_sw<128>(a, nCta, st);
    case 192: return launch_sw<192>(a, nCta, st);
    case 224: return launch_sw<224>(a, nCta, st);
    default: return launch_sw<256>(a, nCta, st);
    }
}

}  // namespace sbk

using namespace sbk;

namespace {

// bilinear interpolation with sentinels, the stand-in for mosaicSource's
// bilinearInterp (absent from the reference tree) shared with the oracle.
float bilinearW(const float* img, double x, double y, int nx, int ny, float minvalue, float noData)
{
    if (x < 0 || y < 0 || x > (double)(nx - 1) || y > (double)(ny - 1)) return noData;
    if (nx < 2 || ny < 2) return noData;
    int j = (int)x, i = (int)y;
    if (j >= nx - 1) j = nx - 2;
    if (i >= ny - 1) i = ny - 2;
    const double t = x - j, u = y - i;
    const float p1 = img[(size_t)i * nx + j], p2 = img[(size_t)i * nx + j + 1];
    const float p3 = img[(size_t)(i + 1) * nx + j + 1], p4 = img[(size_t)(i + 1) * nx + j];
    if (p1 <= minvalue || p2 <= minvalue || p3 <= minvalue || p4 <= minvalue) return noData;
    return (float)((1.0 - t) * (1.0 - u) * p1 + t * (1.0 - u) * p2 + t * u * p3 + (1.0 - t) * u * p4);
}

// findImage2Pos (corrTrackFast.c:257-292)
void findImage2PosW(const sb_track_params* p, int r1, int a1, int* r2, int* a2)
{
    double aShift, rShift;
    const double sc = (double)p->scaleFactor;
    if (p->polyShift) {
        rShift = p->rShiftPoly[0] + (double)(r1 * sc) * p->rShiftPoly[1] + (double)(a1 * sc) * p->rShiftPoly[2];
        aShift = p->aShiftPoly[0] + (double)(r1 * sc) * p->aShiftPoly[1] + (double)(a1 * sc) * p->aShiftPoly[2];
    } else {
        const sb_offset_grid* o = p->initOffsets;
        const float minvalue = (float)((float)-SB_LARGEINT * 0.9);
        const double range = (r1 - o->r0) / o->deltaR, azimuth = (a1 - o->a0) / o->deltaA;
        rShift = bilinearW(o->dr, range, azimuth, o->nr, o->na, minvalue, (float)-SB_LARGEINT);
        aShift = bilinearW(o->da, range, azimuth, o->nr, o->na, minvalue, (float)-SB_LARGEINT);
        if (rShift <= minvalue || aShift <= minvalue) {
            rShift = minvalue;
            aShift = minvalue;
        }
        if (rShift < (-SB_LARGEINT + 1)) {
            rShift = p->rShiftPoly[0] + (double)(r1 * sc) * p->rShiftPoly[1] + (double)(a1 * sc) * p->rShiftPoly[2];
            aShift = p->aShiftPoly[0] + (double)(r1 * sc) * p->aShiftPoly[1] + (double)(a1 * sc) * p->aShiftPoly[2];
        }
    }
    rShift /= sc;
    aShift /= sc;
    *r2 = (rShift >= 0) ? r1 + (int)(rShift + 0.5) : r1 + (int)(rShift - 0.5);
    *a2 = (aShift >= 0) ? a1 + (int)(aShift + 0.5) : a1 + (int)(aShift - 0.5);
}

// maskValue (corrTrackFast.c:1135-1154)
int maskValueW(const sb_track_params* p, int r1, int a1)
{
    const sb_mask* m = p->mask;
    if (!m) return 1;
    const int dr = (p->wRa / 2 - m->r0) * p->scaleFactor;
    const int da = (p->wAa / 2 - m->a0) * p->scaleFactor;
    const int ia1 = (a1 + da) / m->nal, ir1 = (r1 + dr) / m->nrl;
    if (ia1 < 0 || ia1 >= m->na || ir1 < 0 || ir1 >= m->nr) return 0;
    return (int)(signed char)m->mask[(size_t)ia1 * m->nr + ir1];
}

#define CKW(call, what)                                              \
    do {                                                             \
        cudaError_t _e = (call);                                     \
        if (_e != cudaSuccess) return sb_ctx_cuda(c, _e, what);      \
    } while (0)

}  // namespace

extern "C" int sb_strackw(sb_context* c, const sb_track_params* p, const sb_image* img1, const sb_image* img2,
                          sb_track_result* out)
{
    if (!c) return SB_ERR_ARG;
    c->err.clear();
    c->launches = 0;
    if (!p || !out || !img1 || !img2 || !img1->data || !img2->data)
        return sb_ctx_fail(c, SB_ERR_ARG, "null params, image or result");
    if (img1->sampleType != img2->sampleType || img1->byteOrder != img2->byteOrder)
        return sb_ctx_fail(c, SB_ERR_ARG, "images differ in sample type or byte order");
    if (p->nR <= 0 || p->nA <= 0) return sb_ctx_fail(c, SB_ERR_ARG, "empty grid");
    if (p->scaleFactor <= 0) return sb_ctx_fail(c, SB_ERR_ARG, "scaleFactor must be positive");
    if (p->polyShift == 0 && !p->initOffsets) return sb_ctx_fail(c, SB_ERR_ARG, "polyShift=0 needs initOffsets");
    if (!out->offR || !out->offA || !out->corr || !out->type) return sb_ctx_fail(c, SB_ERR_ARG, "null output grid");
    const int W = p->wRa;
    if (p->wRa != p->wAa) return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "search window must be square (wra == waa)");
    if (!sw_supported(W)) return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "search window %d not supported", W);
    const int eR = p->edgePadR + W_NFAST / 4, eA = p->edgePadA + W_NFAST / 4;
    if (eR != eA) return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "edgeR != edgeA not supported");
    if ((W - 2 * eR) <= 0 || p->edgePadR < W_NFAST / 4)
        return sb_ctx_fail(c, SB_ERR_ARG, "edge pad leaves no chip (wra=%d, edgepad=%d)", W, p->edgePadR);
    CKW(cudaSetDevice(c->device), "cudaSetDevice");
    cudaEventRecord(c->ev[0], c->stream);
    // ---- plan (host, raster order; corrTrackFast.c:144-172)
    const int n = p->nR * p->nA;
    std::vector<int4> plan;
    std::vector<int> list;
    std::vector<int> masked0;  // maskVal != 1: outputs stay -2e9 / 0 / type 0
    for (int i = 0; i < p->nA; i++) {
        const int a1 = p->aStart + i * p->deltaA - p->wAa / 2;
        for (int j = 0; j < p->nR; j++) {
            const int r1 = p->rStart + j * p->deltaR - p->wRa / 2;
            int r2, a2;
            findImage2PosW(p, r1, a1, &r2, &a2);
            const int mv = maskValueW(p, r1 * p->scaleFactor, a1 * p->scaleFactor);
            if (mv == 1 && r1 > 0 && r1 < img1->nr && a1 > 0 && a1 < img1->na && r2 > 0 && r2 < img2->nr && a2 > 0 &&
                a2 < img2->na) {
                plan.push_back(make_int4(r1, a1, r2, a2));
                list.push_back(i * p->nR + j);
            }
        }
    }
    const void *d1, *d2;
    int rc;
    if ((rc = sb_image_to_device(c, img1, "img1", &d1)) != SB_OK) return rc;
    if ((rc = sb_image_to_device(c, img2, "img2", &d2)) != SB_OK) return rc;
    cudaError_t e;
    const int nl = (int)list.size();
    int4* dplan = (int4*)sb_ctx_buf(c, "w_plan", sizeof(int4) * (nl + 1), &e);
    int* dlist = (int*)sb_ctx_buf(c, "w_list", sizeof(int) * (nl + 1), &e);
    float* dR = (float*)sb_ctx_buf(c, "offR", sizeof(float) * n, &e);
    float* dA = (float*)sb_ctx_buf(c, "offA", sizeof(float) * n, &e);
    float* dC = (float*)sb_ctx_buf(c, "corr", sizeof(float) * n, &e);
    uint8_t* dT = (uint8_t*)sb_ctx_buf(c, "type", n, &e);
    unsigned long long* dst = (unsigned long long*)sb_ctx_buf(c, "w_stats", 4 * sizeof(unsigned long long), &e);
    double* dB = (double*)sb_ctx_buf(c, "w_B", sizeof(double) * W_OSW * W_N1, &e);
    if (!dplan || !dlist || !dR || !dA || !dC || !dT || !dst || !dB)
        return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
    if (nl) {
        CKW(cudaMemcpyAsync(dplan, plan.data(), sizeof(int4) * nl, cudaMemcpyHostToDevice, c->stream), "plan");
        CKW(cudaMemcpyAsync(dlist, list.data(), sizeof(int) * nl, cudaMemcpyHostToDevice, c->stream), "list");
    }
    // the real oversampling kernel of the 21 -> 336 symmetric zero pad
    std::vector<double> B(W_OSW * W_N1);
    for (int nn = 0; nn < W_OSW; ++nn)
        for (int t = 0; t < W_N1; ++t) {
            const int d = (nn + (W_N1 * W_NOVER) / 2 - W_NOVER * 2) - W_NOVER * t;
            double v = 1.0;
            for (int f = 1; f <= W_NFAST / 2; ++f) v += 2.0 * cos(2.0 * 3.14159265358979323846 * f * d / (W_N1 * W_NOVER));
            B[nn * W_N1 + t] = v;
        }
    CKW(cudaMemcpyAsync(dB, B.data(), sizeof(double) * B.size(), cudaMemcpyHostToDevice, c->stream), "B");
    CKW(cudaMemsetAsync(dst, 0, 4 * sizeof(unsigned long long), c->stream), "memset");
    cudaEventRecord(c->ev[1], c->stream);
    strackw_init_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(dR, dA, dC, dT, n);
    CKW(cudaGetLastError(), "strackw_init");
    c->launches++;
    if (nl) {
        SwArgs a;
        a.img1 = d1;
        a.img2 = d2;
        a.nr1 = img1->nr; a.na1 = img1->na; a.nr2 = img2->nr; a.na2 = img2->na;
        a.sampleType = img1->sampleType;
        a.byteOrder = img1->byteOrder;
        a.plan = dplan;
        a.list = dlist;
        a.nList = nl;
        a.eR = eR;
        a.eA = eA;
        a.navgR = p->navgR;
        a.navgA = p->navgA;
        a.scale = 1.f / ((float)W * (float)W * (float)W * (float)W * (float)(OS * OS * OS * OS) *
                         (float)(OS * OS * (p->navgA + 1) * (p->navgR + 1)));
        a.B = dB;
        a.offR = dR; a.offA = dA; a.corr = dC; a.type = dT;
        a.stats = dst;
        const int L = 4 * eR + 1;
        a.perCta = sw_per_cta(W, L);
        int nCta = c->numSM * sw_ctas(W);
        if (nCta > nl) nCta = nl;
        a.scratch = (float2*)sb_ctx_buf(c, "w_scratch", sizeof(float2) * a.perCta * nCta, &e);
        if (!a.scratch) return sb_ctx_fail(c, SB_ERR_NOMEM, "strackw workspace allocation failed");
        cudaEventRecord(c->sev[0], c->stream);
        CKW(launch_sw_any(W, a, nCta, c->stream), "strackw");
        cudaEventRecord(c->sev[1], c->stream);
        c->launches++;
    }
    cudaEventRecord(c->ev[2], c->stream);
    const int od = out->onDevice;
    const cudaMemcpyKind k = od ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    CKW(cudaMemcpyAsync(out->offR, dR, sizeof(float) * n, k, c->stream), "out");
    CKW(cudaMemcpyAsync(out->offA, dA, sizeof(float) * n, k, c->stream), "out");
    CKW(cudaMemcpyAsync(out->corr, dC, sizeof(float) * n, k, c->stream), "out");
    CKW(cudaMemcpyAsync(out->type, dT, n, k, c->stream), "out");
    unsigned long long st[4];
    CKW(cudaMemcpyAsync(st, dst, sizeof(st), cudaMemcpyDeviceToHost, c->stream), "stats");
    cudaEventRecord(c->ev[3], c->stream);
    CKW(cudaStreamSynchronize(c->stream), "strackw");
    out->nComplex = 0;
    out->nAmp = (int64_t)st[0];
    out->nAmpL = 0;
    out->nFail = (int64_t)st[1];
    out->nAttempted = nl;
    cudaEventElapsedTime(&c->timing[0], c->ev[0], c->ev[3]);
    cudaEventElapsedTime(&c->timing[1], c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&c->timing[2], c->ev[1], c->ev[2]);
    cudaEventElapsedTime(&c->timing[3], c->ev[2], c->ev[3]);
    for (int q = 0; q < 8; ++q) c->stage[q] = 0.f;
    if (nl) cudaEventElapsedTime(&c->stage[0], c->sev[0], c->sev[1]);
    c->stage[5] = (float)nl;
    return SB_OK;
}
