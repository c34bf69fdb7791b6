// strack_device.cuh -- device helpers shared by the strack stage kernels:
// block reductions, the fftshift argmax of findCPeak, the 8x8 -> 96x96
// oversampling window, the Levenberg-Marquardt 1-D Gaussian peak fit and
// the 2-D Gaussian peak fit of the -gauss mode.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "fft_engine.cuh"
#include "strack_common.cuh"

namespace sbk {

constexpr int OSW = 48;  // oversampled search window: rows/cols [24, 72) of 96

__device__ __forceinline__ double warp_allsum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum K doubles over the block; every thread gets the totals.
// red: shared scratch of (NT/32 + 1)*K doubles.  Warp sums by shuffles, the
// cross-warp sum by warp 0 alone (the totals get their own slots, so the
// scratch may be reused by the next call without a third barrier).
template <int K, int NT>
__device__ __forceinline__ void block_allsum(double (&v)[K], double* red)
{
    constexpr int NW = NT / 32;
    static_assert(NW >= 1 && NW <= 32, "one to 32 warps");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_allsum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) red[warp * K + k] = v[k];
    }
    __syncthreads();
    if (warp == 0) {
        double t[K];
#pragma unroll
        for (int k = 0; k < K; ++k) t[k] = lane < NW ? red[lane * K + k] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            if (o < NW) {
#pragma unroll
                for (int k = 0; k < K; ++k) t[k] += __shfl_xor_sync(0xffffffffu, t[k], o);
            }
        }
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < K; ++k) red[NW * K + k] = t[k];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = red[NW * K + k];
}

// (value, rank) maximum: larger value wins, equal values -> smaller rank.
struct ArgMax {
    float v;
    int rank;
    int pos;
};
__device__ __forceinline__ bool am_better(float v, int rank, float bv, int brank)
{
    return v > bv || (v == bv && rank < brank);
}
__device__ __forceinline__ ArgMax warp_argmax(ArgMax a)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        float v = __shfl_xor_sync(0xffffffffu, a.v, o);
        int r = __shfl_xor_sync(0xffffffffu, a.rank, o);
        int p = __shfl_xor_sync(0xffffffffu, a.pos, o);
        if (am_better(v, r, a.v, a.rank)) {
            a.v = v;
            a.rank = r;
            a.pos = p;
        }
    }
    return a;
}
// Block argmax; all threads receive the result.  scratch: 3*(NT/32) words.
template <int NT>
__device__ __forceinline__ ArgMax block_argmax(ArgMax a, int* scratch)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    a = warp_argmax(a);
    if (lane == 0) {
        scratch[warp] = __float_as_int(a.v);
        scratch[NT / 32 + warp] = a.rank;
        scratch[2 * (NT / 32) + warp] = a.pos;
    }
    __syncthreads();
    ArgMax b;
    b.v = __int_as_float(scratch[0]);
    b.rank = scratch[NT / 32];
    b.pos = scratch[2 * (NT / 32)];
#pragma unroll
    for (int w = 1; w < NT / 32; ++w) {
        float v = __int_as_float(scratch[w]);
        int r = scratch[NT / 32 + w];
        if (am_better(v, r, b.v, b.rank)) {
            b.v = v;
            b.rank = r;
            b.pos = scratch[2 * (NT / 32) + w];
        }
    }
    __syncthreads();
    return b;
}

// Scan rank of position (y, x) of the fftshifted surface in findCPeak's loop
// (speckleTrack.c:750-788): for each (i < h, j < h) the four quadrants are
// visited in the order (i,j), (i+h,j+h), (i+h,j), (i,j+h).
__device__ __forceinline__ int cpeak_rank(int y, int x, int h)
{
    const int yi = y >= h, xi = x >= h;
    const int i = y - yi * h, j = x - xi * h;
    const int q = (!yi && !xi) ? 0 : (yi && xi) ? 1 : (yi ? 2 : 3);
    return (i * h + j) * 4 + q;
}

// 96-point oversampling as a matrix: output n (in [24,72)) of the inverse
// 96-point DFT of the zero-padded 8-point spectrum of x[t] is
//   sum_t A[n][t] x[t],  A[n][t] = sum_{f=-4..3} exp(+2 pi i f (n - 12 t) / 96)
// (zeroPadFFT places bins 0..3 at 0..3 and bins 4..7, Nyquist included, at
// 92..95; speckleTrack.c:2014-2038).  osA holds A for n = 24..71, row-major
// [n-24][t], computed on the host in double precision.
//
// Evaluates the 48 x 48 window of the 2-D oversampled block
// O = A X A^T for the 8x8 real block X (row-major in blk) and returns the
// first maximum of |O| in row-major order (strict >, as cmpTrackFast
// :685-699).  T: shared scratch of 8*48 float2.
template <int NT>
__device__ __forceinline__ ArgMax oversample_peak(const float* blk, const float2* osA, float2* T, int* scratch)
{
    const int tid = threadIdx.x;
    // T[t1][n2] = sum_t2 X[t1][t2] * A[n2][t2]
    for (int e = tid; e < NFAST * OSW; e += NT) {
        const int t1 = e / OSW, n2 = e % OSW;
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int t2 = 0; t2 < NFAST; ++t2) {
            const float x = blk[t1 * NFAST + t2];
            const float2 a = osA[n2 * NFAST + t2];
            acc.x = fmaf(x, a.x, acc.x);
            acc.y = fmaf(x, a.y, acc.y);
        }
        T[t1 * OSW + n2] = acc;
    }
    __syncthreads();
    ArgMax best;
    best.v = 0.f;
    best.rank = 0x7fffffff;
    best.pos = 0;
    for (int e = tid; e < OSW * OSW; e += NT) {
        const int n1 = e / OSW, n2 = e % OSW;
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int t1 = 0; t1 < NFAST; ++t1) {
            const float2 a = osA[n1 * NFAST + t1];
            const float2 t = T[t1 * OSW + n2];
            acc.x = fmaf(a.x, t.x, fmaf(-a.y, t.y, acc.x));
            acc.y = fmaf(a.x, t.y, fmaf(a.y, t.x, acc.y));
        }
        const float v = sqrtf(acc.x * acc.x + acc.y * acc.y);
        if (am_better(v, e, best.v, best.rank) && v > 0.f) {
            best.v = v;
            best.rank = e;
            best.pos = e;
        }
    }
    ArgMax r = block_argmax<NT>(best, scratch);
    if (r.rank == 0x7fffffff) {  // nothing above 0: the reference keeps index 0,0
        r.v = 0.f;
        r.pos = 0;
    }
    return r;
}

// 64-bit (value, rank) maximum over the block: key = bits(v) << 32 | ~rank, so
// the larger value wins and equal values go to the smaller rank.  scratch:
// NT/32 words of 8 bytes.  All threads receive the result.
__device__ __forceinline__ unsigned long long block_max_u64(unsigned long long v, unsigned long long* scratch)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
        v = u > v ? u : v;
    }
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    v = scratch[0];
    for (int w = 1; w < nw; ++w) v = scratch[w] > v ? scratch[w] : v;
    __syncthreads();
    return v;
}
__device__ __forceinline__ unsigned long long am_key(float v, unsigned rank)
{
    const unsigned vb = v > 0.f ? __float_as_uint(v) : 0u;  // zero and NaN never win
    return ((unsigned long long)vb << 32) | (0xffffffffu - rank);
}

// The same 48 x 48 window through the real form of the matrix:
//   A[n][t] = p(n) exp(+i pi t / 8) D[n][t],  |p(n)| = 1,
//   D[n][t] = 2 sum_{g = 1/2, 3/2, 5/2, 7/2} cos(2 pi g (n + 24 - 12 t) / 96),
// so |O| = |D Y D^T| with Y[t1][t2] = exp(i pi (t1 + t2) / 8) X[t1][t2]; the
// products with D are real x complex (half the multiplies of A X A^T).
// osD: D row-major [n][t] (48 x 8 floats, 16-byte aligned) followed by the
// 16 phases exp(i pi s / 8).  Yb: 64 float2, T: 8 * 48 float2 of scratch.
// One entry of T = Y D^T: T[t1][n2] = sum_t2 Y[t1][t2] D[n2][t2].
__device__ __forceinline__ float2 osr_T_entry(const float2* Yb, const float* osD, int t1, int n2)
{
    const float4* dr = reinterpret_cast<const float4*>(osD + n2 * NFAST);
    const float4 d0 = dr[0], d1 = dr[1];
    const float d[NFAST] = {d0.x, d0.y, d0.z, d0.w, d1.x, d1.y, d1.z, d1.w};
    float2 acc = make_float2(0.f, 0.f);
#pragma unroll
    for (int t2 = 0; t2 < NFAST; ++t2) {
        const float2 y = Yb[t1 * NFAST + t2];
        acc.x = fmaf(d[t2], y.x, acc.x);
        acc.y = fmaf(d[t2], y.y, acc.y);
    }
    return acc;
}

// Rows n1 = g, g + 8, ..., g + 40 of column n2 of O = D T, folded into the
// lane's best (|O|, first index) key.  lo is the lane's bound: a value whose
// |O|^2 lies more than 2^-20 (relative) below the |O|^2 of the lane's best
// can neither beat nor tie it after the correctly rounded sqrtf, so the sqrt
// and the key are evaluated only at or above lo (NaN never is, as NaN never
// won before).  Start with best = 0, lo = 0.
__device__ __forceinline__ void osr_O_rows(const float2* T, const float* osD, int g, int n2, unsigned long long& best,
                                           float& lo)
{
    constexpr int RPG = OSW / NFAST;
    float2 tv[NFAST];
#pragma unroll
    for (int t1 = 0; t1 < NFAST; ++t1) tv[t1] = T[t1 * OSW + n2];
#pragma unroll
    for (int u = 0; u < RPG; ++u) {
        const int n1 = g + NFAST * u;
        const float4* dr = reinterpret_cast<const float4*>(osD + n1 * NFAST);
        const float4 d0 = dr[0], d1 = dr[1];
        const float d[NFAST] = {d0.x, d0.y, d0.z, d0.w, d1.x, d1.y, d1.z, d1.w};
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int t1 = 0; t1 < NFAST; ++t1) {
            acc.x = fmaf(d[t1], tv[t1].x, acc.x);
            acc.y = fmaf(d[t1], tv[t1].y, acc.y);
        }
        const float m2 = fmaf(acc.x, acc.x, __fmul_rn(acc.y, acc.y));
        if (m2 >= lo) {
            const unsigned long long k = am_key(sqrtf(m2), (unsigned)(n1 * OSW + n2));
            if (k > best) {
                best = k;
                lo = m2 * (1.0f - 1.0f / 1048576.0f);
            }
        }
    }
}

__device__ __forceinline__ ArgMax osr_result(unsigned long long best)
{
    ArgMax r;
    if ((best >> 32) == 0ull) {  // nothing above 0: the reference keeps index 0,0
        r.v = 0.f;
        r.pos = 0;
    } else {
        r.v = __uint_as_float((unsigned)(best >> 32));
        r.pos = (int)(0xffffffffu - (unsigned)(best & 0xffffffffull));
    }
    r.rank = r.pos;
    return r;
}

// The same 48 x 48 window through the real form of the matrix:
//   A[n][t] = p(n) exp(+i pi t / 8) D[n][t],  |p(n)| = 1,
//   D[n][t] = 2 sum_{g = 1/2, 3/2, 5/2, 7/2} cos(2 pi g (n + 24 - 12 t) / 96),
// so |O| = |D Y D^T| with Y[t1][t2] = exp(i pi (t1 + t2) / 8) X[t1][t2]; the
// products with D are real x complex (half the multiplies of A X A^T).
// osD: D row-major [n][t] (48 x 8 floats, 16-byte aligned) followed by the
// 16 phases exp(i pi s / 8).  Yb: 64 float2, T: 8 * 48 float2 of scratch.
// Block version: all NT threads, block barriers.
template <int NT>
__device__ __forceinline__ ArgMax oversample_peak_real(const float* blk, const float* osD, float2* Yb, float2* T,
                                                       unsigned long long* scratch)
{
    const int tid = threadIdx.x;
    const float2* ph = reinterpret_cast<const float2*>(osD + OSW * NFAST);
    if (tid < NFAST * NFAST) {
        const float x = blk[tid];
        const float2 e = ph[tid / NFAST + tid % NFAST];
        Yb[tid] = make_float2(x * e.x, x * e.y);
    }
    __syncthreads();
    for (int e = tid; e < NFAST * OSW; e += NT) T[e] = osr_T_entry(Yb, osD, e / OSW, e % OSW);
    __syncthreads();
    // a thread keeps column n2 of T in registers and produces rows g, g + 8, ...
    unsigned long long best = 0ull;
    float lo = 0.f;
    for (int e = tid; e < NFAST * OSW; e += NT) osr_O_rows(T, osD, e / OSW, e % OSW, best, lo);
    return osr_result(block_max_u64(best, scratch));
}

// Warp version (one warp per patch, warp barriers only).  blk: the 8 x 8
// |c| block (any lane may read it); Yb, T: this warp's scratch.
__device__ __forceinline__ ArgMax oversample_peak_warp(const float* blk, const float* osD, float2* Yb, float2* T)
{
    const int lane = threadIdx.x & 31;
    const float2* ph = reinterpret_cast<const float2*>(osD + OSW * NFAST);
    for (int t = lane; t < NFAST * NFAST; t += 32) {
        const float x = blk[t];
        const float2 e = ph[t / NFAST + t % NFAST];
        Yb[t] = make_float2(x * e.x, x * e.y);
    }
    __syncwarp();
    for (int e = lane; e < NFAST * OSW; e += 32) T[e] = osr_T_entry(Yb, osD, e / OSW, e % OSW);
    __syncwarp();
    unsigned long long best = 0ull;
    float lo = 0.f;
    for (int e = lane; e < NFAST * OSW; e += 32) osr_O_rows(T, osD, e / OSW, e % OSW, best, lo);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long u = __shfl_xor_sync(0xffffffffu, best, o);
        best = u > best ? u : best;
    }
    __syncwarp();  // Yb and T are free for the next patch
    return osr_result(best);
}

// ---------------------------------------------------------------- LM fit
// gaussPeak1D (speckleTrack.c:2137-2202) with mrqminMod/mrqcofMod
// (:2309-2416) and a full-pivot Gauss-Jordan solve, in double precision.
// One warp per fit; lanes 0..17 hold the samples (x, y).  Every lane runs the
// 3x3 algebra redundantly on warp-reduced sums.

struct LMSums {
    double al[6];  // alpha 11, 21, 22, 31, 32, 33
    double be[3];
    double chisq;
};

__device__ __forceinline__ LMSums lm_cof(double x, double y, bool active, const double a[4])
{
    LMSums s;
    double dyda[4] = {0, 0, 0, 0};
    double ymod = 0.0;
    if (active) {
        const double sig = a[3];
        const double t = x - a[2];
        const double argx = 0.5 * t * t / (sig * sig);
        const double ex = exp(-argx);
        ymod = a[1] * ex;
        dyda[1] = ex;
        dyda[2] = ymod * t / (sig * sig);
        dyda[3] = ymod * t * t / (sig * sig * sig);
    }
    const double sig2i = active ? 1.0 / (0.1 * 0.1) : 0.0;
    const double dy = active ? y - ymod : 0.0;
    const double w1 = dyda[1] * sig2i, w2 = dyda[2] * sig2i, w3 = dyda[3] * sig2i;
    s.al[0] = w1 * dyda[1];
    s.al[1] = w2 * dyda[1];
    s.al[2] = w2 * dyda[2];
    s.al[3] = w3 * dyda[1];
    s.al[4] = w3 * dyda[2];
    s.al[5] = w3 * dyda[3];
    s.be[0] = dy * w1;
    s.be[1] = dy * w2;
    s.be[2] = dy * w3;
    s.chisq = dy * dy * sig2i;
#pragma unroll
    for (int k = 0; k < 6; ++k) s.al[k] = warp_allsum(s.al[k]);
#pragma unroll
    for (int k = 0; k < 3; ++k) s.be[k] = warp_allsum(s.be[k]);
    s.chisq = warp_allsum(s.chisq);
    return s;
}

__device__ __forceinline__ void lm_unpack(const LMSums& s, double al[4][4], double be[4])
{
    al[1][1] = s.al[0];
    al[2][1] = al[1][2] = s.al[1];
    al[2][2] = s.al[2];
    al[3][1] = al[1][3] = s.al[3];
    al[3][2] = al[2][3] = s.al[4];
    al[3][3] = s.al[5];
    be[1] = s.be[0];
    be[2] = s.be[1];
    be[3] = s.be[2];
}

// Gauss-Jordan with full pivoting (3x3, one right-hand side); false if singular.
__device__ __forceinline__ bool gaussj3(double a[4][4], double b[4])
{
    int indxc[4], indxr[4], ipiv[4] = {0, 0, 0, 0};
    int irow = 1, icol = 1;
    for (int i = 1; i <= 3; i++) {
        double big = 0.0;
        for (int j = 1; j <= 3; j++)
            if (ipiv[j] != 1)
                for (int k = 1; k <= 3; k++) {
                    if (ipiv[k] == 0) {
                        if (fabs(a[j][k]) >= big) {
                            big = fabs(a[j][k]);
                            irow = j;
                            icol = k;
                        }
                    } else if (ipiv[k] > 1)
                        return false;
                }
        ++(ipiv[icol]);
        if (irow != icol) {
            for (int l = 1; l <= 3; l++) {
                double t = a[irow][l];
                a[irow][l] = a[icol][l];
                a[icol][l] = t;
            }
            double t = b[irow];
            b[irow] = b[icol];
            b[icol] = t;
        }
        indxr[i] = irow;
        indxc[i] = icol;
        if (a[icol][icol] == 0.0) return false;
        const double pivinv = 1.0 / a[icol][icol];
        a[icol][icol] = 1.0;
        for (int l = 1; l <= 3; l++) a[icol][l] *= pivinv;
        b[icol] *= pivinv;
        for (int ll = 1; ll <= 3; ll++)
            if (ll != icol) {
                const double dum = a[ll][icol];
                a[ll][icol] = 0.0;
                for (int l = 1; l <= 3; l++) a[ll][l] -= a[icol][l] * dum;
                b[ll] -= b[icol] * dum;
            }
    }
    (void)indxr;
    (void)indxc;
    return true;
}

// Returns sigma = a[3]/2 of the fit (all lanes).
__device__ __forceinline__ double gauss_peak_1d(float sample, int xpos, int lane)
{
    const bool active = lane < NGAUSS;
    float mx = active ? sample : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const double maxC = (double)fmaxf(mx, 0.f);
    const double x = (double)xpos;
    const double y = active ? (double)sample / maxC : 0.0;
    const double xc = (double)__shfl_sync(0xffffffffu, xpos, NGAUSS / 2);
    double a[4] = {0.0, 1.0, xc, 2.0};
    double alamda = 0.001;
    LMSums s0 = lm_cof(x, y, active, a);
    double alpha[4][4], beta[4];
    lm_unpack(s0, alpha, beta);
    double ochisq = s0.chisq;
    double lasti = 2e9;
    for (int it = 0; it < 5; ++it) {
        double covar[4][4], da[4];
        for (int j = 1; j <= 3; j++) {
            for (int k = 1; k <= 3; k++) covar[j][k] = alpha[j][k];
            covar[j][j] = alpha[j][j] * (1.0 + alamda);
            da[j] = beta[j];
        }
        if (!gaussj3(covar, da)) break;
        double atry[4] = {0.0, a[1] + da[1], a[2] + da[2], a[3] + da[3]};
        LMSums s1 = lm_cof(x, y, active, atry);
        if (s1.chisq < ochisq) {
            alamda *= 0.1;
            ochisq = s1.chisq;
            lm_unpack(s1, alpha, beta);
            a[1] = atry[1];
            a[2] = atry[2];
            a[3] = atry[3];
        } else {
            alamda *= 10.0;
        }
        if (fabs(a[2] - lasti) < 0.001) break;
        lasti = a[2];
    }
    return a[3] * .5;
}

// Doppler roll from the lag-1 sums (estDopCarrier1, dopplerEstimation.c:25-40),
// rescaled to wA.  A NaN angle (all-zero sums) gives roll 0.
__device__ __forceinline__ int dop_shift(double sr1, double si1, double sr2, double si2, int nAz, int wA)
{
    const double PI_ = 3.14159265358979323846;
    const double an1 = (sr1 == 0.0 && si1 == 0.0) ? nan("") : atan2(si1, sr1);
    const double an2 = (sr2 == 0.0 && si2 == 0.0) ? nan("") : atan2(si2, sr2);
    const double v = (double)(nAz / 2) * (an1 + an2) * .5 / PI_;
    int shift = (v != v) ? 0 : ((v >= 0.0) ? (int)(v + 0.5) : (int)(v - 0.5));
    if (shift < 0) shift += nAz;
    return (int)((float)shift * (float)wA / (float)nAz);
}

// cmpTrackGauss (Strack/speckleTrack.c:2205-2303, the -gauss mode): a 2-D
// Gaussian (amplitude, centre and width per axis; myGauss :2421-2443) fitted
// to the 18 x 18 samples S of |c| * scale around the coarse peak by the
// Levenberg-Marquardt steps of mrqminMod (:2353-2416) in float, <= 8 steps,
// stopping when both centres move < 0.001.  Run by one warp: per-sample terms
// on the lanes, the 5 x 5 Gauss-Jordan solve (full pivoting) on every lane.
static __device__ __forceinline__ void lm2d_cof(const float* S, float i0, float j0, const float (&a)[6], float (&al)[6][6],
                                         float (&be)[6], float& chisq)
{
    const int lane = threadIdx.x & 31;
    float A[15], B[5], c2 = 0.f;
#pragma unroll
    for (int k = 0; k < 15; ++k) A[k] = 0.f;
#pragma unroll
    for (int k = 0; k < 5; ++k) B[k] = 0.f;
    for (int k = lane; k < NGAUSS * NGAUSS; k += 32) {
        const float px = i0 + (float)(k / NGAUSS), py = j0 + (float)(k % NGAUSS);
        const float dx = px - a[2], dyv = py - a[4];
        const float argx = 0.5f * (dx * dx) / (a[3] * a[3]);
        const float argy = 0.5f * (dyv * dyv) / (a[5] * a[5]);
        const float ex = expf(-argx - argy);
        const float y = a[1] * ex;
        const float d[5] = {ex, y * (px - a[2]) / (a[3] * a[3]), y * (px - a[2]) * (px - a[2]) / (a[3] * a[3] * a[3]),
                            y * (py - a[4]) / (a[5] * a[5]), y * (py - a[4]) * (py - a[4]) / (a[5] * a[5] * a[5])};
        const float dy = S[k] - y;
        int t = 0;
#pragma unroll
        for (int l = 0; l < 5; ++l) {
#pragma unroll
            for (int m = 0; m <= l; ++m) A[t++] += d[l] * d[m];
            B[l] += dy * d[l];
        }
        c2 += dy * dy;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 15; ++k) A[k] += __shfl_xor_sync(0xffffffffu, A[k], o);
#pragma unroll
        for (int k = 0; k < 5; ++k) B[k] += __shfl_xor_sync(0xffffffffu, B[k], o);
        c2 += __shfl_xor_sync(0xffffffffu, c2, o);
    }
    int t = 0;
#pragma unroll
    for (int l = 1; l <= 5; ++l) {
#pragma unroll
        for (int m = 1; m <= l; ++m) {
            al[l][m] = A[t];
            al[m][l] = A[t];
            ++t;
        }
        be[l] = B[l - 1];
    }
    chisq = c2;
}

// Gauss-Jordan with full pivoting (Numerical Recipes gaussj) on the 5 x 5
// system with one right-hand side; false when singular (the reference would
// exit; the fit ends instead).
static __device__ __noinline__ bool gaussj5(float (&m)[6][6], float (&b)[6])
{
    int ipiv[6] = {0, 0, 0, 0, 0, 0};
    int irow = 0, icol = 0;
    for (int i = 1; i <= 5; i++) {
        float big = 0.f;
        for (int j = 1; j <= 5; j++)
            if (ipiv[j] != 1)
                for (int k = 1; k <= 5; k++) {
                    if (ipiv[k] == 0) {
                        if (fabsf(m[j][k]) >= big) {
                            big = fabsf(m[j][k]);
                            irow = j;
                            icol = k;
                        }
                    } else if (ipiv[k] > 1)
                        return false;
                }
        ++ipiv[icol];
        if (irow != icol) {
            for (int l = 1; l <= 5; l++) {
                const float t = m[irow][l];
                m[irow][l] = m[icol][l];
                m[icol][l] = t;
            }
            const float t = b[irow];
            b[irow] = b[icol];
            b[icol] = t;
        }
        if (m[icol][icol] == 0.f) return false;
        const float pivinv = 1.0f / m[icol][icol];
        m[icol][icol] = 1.f;
        for (int l = 1; l <= 5; l++) m[icol][l] *= pivinv;
        b[icol] *= pivinv;
        for (int ll = 1; ll <= 5; ll++)
            if (ll != icol) {
                const float dum = m[ll][icol];
                m[ll][icol] = 0.f;
                for (int l = 1; l <= 5; l++) m[ll][l] -= m[icol][l] * dum;
                b[ll] -= b[icol] * dum;
            }
    }
    return true;
}

// The fit itself (warp 0); a[1..5] in and out.
static __device__ __noinline__ void cmp_track_gauss_warp(const float* S, float i0, float j0, float (&a)[6])
{
    float alpha[6][6], beta[6], chisq = 0.f, ochisq = 0.f, alamda = -1.f;
    float lasti = 2e9f, lastj = 2e9f;
    for (int it = 0; it < 8; ++it) {
        float covar[6][6], da[6], atry[6];
        if (alamda < 0.f) {
            alamda = 0.001f;
            lm2d_cof(S, i0, j0, a, alpha, beta, chisq);
            ochisq = chisq;
        }
        for (int j = 1; j <= 5; j++) {
            for (int k = 1; k <= 5; k++) covar[j][k] = alpha[j][k];
            covar[j][j] = alpha[j][j] * (1.0f + alamda);
            da[j] = beta[j];
        }
        if (!gaussj5(covar, da)) break;
        atry[0] = a[0];
        for (int l = 1; l <= 5; l++) atry[l] = a[l] + da[l];
        lm2d_cof(S, i0, j0, atry, covar, da, chisq);
        if (chisq < ochisq) {
            alamda *= 0.1f;
            ochisq = chisq;
            for (int j = 1; j <= 5; j++) {
                for (int k = 1; k <= 5; k++) alpha[j][k] = covar[j][k];
                beta[j] = da[j];
            }
            for (int l = 1; l <= 5; l++) a[l] = atry[l];
        } else {
            alamda *= 10.0f;
            chisq = ochisq;
        }
        if (fabsf(a[2] - lasti) < 0.001f && fabsf(a[4] - lastj) < 0.001f) break;
        lasti = a[2];
        lastj = a[4];
    }
}

// The whole of cmpTrackGauss for one CTA (all threads call it): the edge
// test on the N x N plane (peaks within 9 of the border, or rejected ones,
// fail), the 18 x 18 samples mag(i, j) * scale into S, the fit by warp 0
// (initial amplitude cMax * scale, widths 3), and the result in NOVER units:
// iMax = round(mux * NOVER), cMax = min(amp, 1); a width above 2000 fails.
// Failures return iMax = jMax = -LARGEINT and cMax = 0.  g6: 6 floats of
// shared scratch.
template <int NT, class Mag>
__device__ __forceinline__ void gauss2d_peak(Mag mag, int N, double scale, float* S, float* g6, int& iMax, int& jMax,
                                             double& cMax)
{
    if ((iMax - NGAUSS / 2) < 0 || (iMax + NGAUSS / 2) >= (N - 1) || (jMax - NGAUSS / 2) < 0 ||
        (jMax + NGAUSS / 2) >= (N - 1)) {
        iMax = -(int)SB_LARGEINT;
        jMax = -(int)SB_LARGEINT;
        cMax = 0.0;
        return;
    }
    const int tid = threadIdx.x;
    for (int e = tid; e < NGAUSS * NGAUSS; e += NT)
        S[e] = (float)((double)mag(iMax - NGAUSS / 2 + e / NGAUSS, jMax - NGAUSS / 2 + e % NGAUSS) * scale);
    __syncthreads();
    if (tid < 32) {
        float g[6] = {0.f, (float)(cMax * scale), (float)iMax, 3.f, (float)jMax, 3.f};
        cmp_track_gauss_warp(S, (float)(iMax - NGAUSS / 2), (float)(jMax - NGAUSS / 2), g);
        if (tid < 6) g6[tid] = g[tid];
    }
    __syncthreads();
    const float g1 = g6[1], g2 = g6[2], g3 = g6[3], g4 = g6[4], g5 = g6[5];
    __syncthreads();
    iMax = (int)round((double)(g2 * NOVER));
    jMax = (int)round((double)(g4 * NOVER));
    cMax = g1 < 1.0f ? (double)g1 : 1.0;
    if ((0.5 * g3) > 1000.0 || (0.5 * g5) > 1000.0) {
        iMax = -(int)SB_LARGEINT;
        jMax = -(int)SB_LARGEINT;
        cMax = 0.0;
    }
}

}  // namespace sbk
