// strack_cmplx.cu -- complex (speckle) matching stage of strack, one CTA per
// grid point, everything resident in shared memory.
//
// Follows getPatches (Strack/speckleTrack.c:1194-1330), estDopCarrier1
// (Strack/dopplerEstimation.c:25-88), phaseCorrectBaseline (:868-907),
// cmpPSWithPad (:604-643), cmpTrackFast (:648-709), findCPeak (:744-805),
// cmpTrackGauss (:2205-2303), gaussPeak1D's samples (:2137-2202),
// complexMatch (:349-394) and finalizeCmpxMatch (:714-739).
//
// The 2W x 2W inverse transform of the zero-padded cross spectrum is computed
// as four W x W inverse transforms, one per output parity (e1, e2): with the
// non-zero quadrants folded to X'[k1'][k2'] = S[(k1'+azShift) % W][k2'],
//   c[2 m1 + e1][2 m2 + e2] = IDFT_W(X' tau_e1[k1'] tau_e2[k2'])[m1][m2],
//   tau_0 = 1, tau_1[k'] = +-exp(+2 pi i k' / 2W) (minus for k' >= W/2),
// which is the same sum regrouped.  Only |c| is kept (four W x W float planes).
//
// After findCPeak the kernel hands the coarse peak and the |c|^2 samples
// around it to strack_peak.cu (overSampleC and the gaussPeak1D samples, a warp
// per patch); with -gauss (GAUSS) the 2-D fit runs here instead.  Thread
// counts per window are set where the kernel is launched (4W threads, 8W at
// W = 32), measured per window.
#include <cuda_runtime.h>

#include <type_traits>

#include "strack_device.cuh"
#include "strack_kernels.h"

namespace sbk {

template <int W, int NT>
struct CmplxSmem {
    static constexpr int RS = W + 1;    // odd row stride: row passes are bank-conflict free
    static constexpr int IMG = W * RS;  // float2 per buffer; three buffers X, Y, Z
    static constexpr int OSD = OSW * NFAST / 2 + 16;  // float2 of the real oversampling table
    static constexpr size_t bytes = sizeof(float2) * (3 * IMG + 2 * W + OSD + NFAST * NFAST + NFAST * OSW) +
                                    sizeof(float) * (NFAST * NFAST) + sizeof(double) * (NT / 32 + 1) * 8 + 64 + 16;
};

// |c|^2 of the 2W x 2W surface at unshifted index (cy, cx).  The parity plane
// (e1, e2) = (cy & 1, cx & 1) is a W x W float array at float offset poff(q),
// q = 2 e1 + e2, from the start of shared memory (buffers X | Y | Z of 2W(W+1)
// floats each): (0,0) X[0, W^2), (0,1) X[W^2, 2W^2), (1,0) the last W^2 floats
// of Y, (1,1) Z[0, W^2).
template <int W>
__device__ __forceinline__ int poff(int q)
{
    constexpr int IMGF = 2 * W * (W + 1);
    return q == 0 ? 0 : (q == 1 ? W * W : (q == 2 ? 2 * IMGF - W * W : 2 * IMGF));
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

// Rows per batch of window loads: the largest divisor of a thread's run of
// rows that is at most 8.
__host__ __device__ constexpr int load_batch(int rpt)
{
    return rpt % 8 == 0 ? 8 : rpt % 7 == 0 ? 7 : rpt % 6 == 0 ? 6 : rpt % 5 == 0 ? 5 : rpt % 4 == 0 ? 4
           : rpt % 3 == 0 ? 3 : rpt % 2 == 0 ? 2 : 1;
}

// A raw sample (8 bytes of complex float32 or 4 of complex int16, loaded as
// one word) to complex float: byte swap for big-endian files, complex float32
// scaled by 1000 (getPatches), int16 as is.
template <bool F32>
__device__ __forceinline__ float2 decode_sample(typename std::conditional<F32, uint2, uint32_t>::type w, bool msb)
{
    if constexpr (F32) {
        if (msb) {
            w.x = bswap32(w.x);
            w.y = bswap32(w.y);
        }
        return make_float2(__uint_as_float(w.x) * 1000.f, __uint_as_float(w.y) * 1000.f);
    } else {
        if (msb) w = bswap16x2(w);
        return make_float2((float)(int16_t)(w & 0xffffu), (float)(int16_t)(w >> 16));
    }
}

// Final store of a pair of column passes of the padded inverse, parities
// (0, E2) and (1, E2) (line l < W: e1 = 0, else e1 = 1, column l mod W):
// |c|^2 goes to the parity plane and the thread's running maximum of it is
// kept.  (|c| = sqrtf(|c|^2) is taken where a value is used; the argmax over
// |c| with findCPeak's tie order is recovered exactly afterwards, see
// cpeak_from_planes.)  fmaxf ignores NaN, so NaN never wins.
template <int W, int N1, int N2, int E2>
struct MagMax {
    float* plane0;  // parity (0, E2)
    float* plane1;  // parity (1, E2)
    float& pmax;
    __device__ __forceinline__ void operator()(int l, int k1, int k2, float2 z) const
    {
        const int e1 = l >= W;
        const int col = l - (e1 ? W : 0);
        const float p = z.x * z.x + z.y * z.y;
        (e1 ? plane1 : plane0)[(k1 + N1 * k2) * W + col] = p;
        pmax = fmaxf(pmax, p);
    }
};

// findCPeak (speckleTrack.c:744-805) over the four |c|^2 planes, given the
// block maximum pmax of |c|^2: the peak is the largest |c| = sqrtf(|c|^2)
// (> 0), ties to the first position in findCPeak's scan order (cpeak_rank).
// sqrtf is correctly rounded and monotone, so every position whose sqrtf
// equals sqrtf(pmax) has |c|^2 within a relative 2^-20 of pmax: only those
// are ranked.  Returns the fftshifted (iMax, jMax), or (0, 0) when nothing is
// above 0.  iscr: 2 NT/32 words, one set per reduction; the caller puts a
// block barrier between this and the next write to them.
template <int W, int NT>
__device__ __forceinline__ void cpeak_from_planes(const float* smf, float pmax, unsigned* iscr, int& iMax, int& jMax)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned u = __reduce_max_sync(0xffffffffu, __float_as_uint(pmax));  // |c|^2 >= 0: bits order as values
    if (lane == 0) iscr[warp] = u;
    __syncthreads();
    u = iscr[0];
#pragma unroll
    for (int w = 1; w < NT / 32; ++w) u = max(u, iscr[w]);
    const float pm = __uint_as_float(u);
    iMax = 0;
    jMax = 0;
    if (!(pm > 0.f)) return;  // uniform
    const float sm = sqrtf(pm);
    const float lo = pm * (1.0f - 1.0f / 1048576.0f);
    unsigned best = 0xffffffffu;
    constexpr int Q4 = W * W / 4;  // float4 per plane
    constexpr int U = 4;           // float4 loads in flight per thread
    for (int e0 = tid; e0 < 4 * Q4; e0 += U * NT) {
        float4 v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + u * NT;
            const int q = e / Q4, i4 = e - q * Q4;
            v[u] = e < 4 * Q4 ? reinterpret_cast<const float4*>(smf + poff<W>(q))[i4]
                              : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            // candidates are rare: one test per float4 keeps the sqrtf and
            // the rank work off the common path (the compiler predicates a
            // plain per-value test, sqrtf included)
            if (fmaxf(fmaxf(v[u].x, v[u].y), fmaxf(v[u].z, v[u].w)) < lo) continue;
            const int e = e0 + u * NT;
            const int q = e / Q4, i4 = e - q * Q4;
            const float vv[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                if (vv[c] >= lo && sqrtf(vv[c]) == sm) {
                    const int idx = 4 * i4 + c;
                    const int cy = 2 * (idx / W) + (q >> 1), cx = 2 * (idx % W) + (q & 1);
                    const int y = cy < W ? cy + W : cy - W, x = cx < W ? cx + W : cx - W;
                    best = min(best, (unsigned)cpeak_rank(y, x, W));
                }
            }
        }
    }
    best = __reduce_min_sync(0xffffffffu, best);
    if (lane == 0) iscr[NT / 32 + warp] = best;
    __syncthreads();
    best = iscr[NT / 32];
#pragma unroll
    for (int w = 1; w < NT / 32; ++w) best = min(best, iscr[NT / 32 + w]);
    const int q = best & 3, ij = best >> 2;
    iMax = ij / W + ((q == 1 || q == 2) ? W : 0);
    jMax = ij % W + ((q == 1 || q == 3) ? W : 0);
}

// phaseCorrectInt (Strack/speckleTrack.c:909-1000) on patch 1 (X, row
// stride RS): the ps x ps interferogram patch centred on the window is
// transformed, every bin below 0.99 of the peak power loses its real part and
// every bin its imaginary part (the reference's loop has no braces), the
// remaining bins are placed as zeroPadFFT places them in a (ps nal) x (ps nrl)
// array (for odd ps the last row and column are not copied) and the inverse
// transform is evaluated directly at the window's pixels; patch 1 is
// multiplied by conj(P) / |P| (or left alone where |P| < 1e-6).  The small
// forward DFT and the peak list use `work` (2 ps^2 float2, the free Y buffer).
template <int W, int RS, int NT>
__device__ __forceinline__ void phase_correct_int(const CmplxArgs& a, const PointPlan& pl, float2* X, float2* work,
                                                  double* red)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ps = a.intPs;
    const int ia1 = (pl.a1 + W / 2) / a.intNal - ps / 2;
    const int ir1 = (pl.r1 + W / 2) / a.intNrl - ps / 2;
    if (!(ir1 > 0 && ir1 + ps < a.intNr && ia1 > 0 && ia1 + ps < a.intNa)) return;  // inBounds, uniform
    const int n2 = ps * ps;
    float2* G = work;       // interferogram patch, then its spectrum
    float2* H = work + n2;  // row transform; then the peak list
    for (int e = tid; e < n2; e += NT) {
        uint32_t w = __ldg(a.intf + (size_t)(ia1 + e / ps) * a.intNr + ir1 + e % ps);
        if (a.intMSB) w = bswap16x2(w);
        G[e] = make_float2((float)(int16_t)(w & 0xffffu), (float)(int16_t)(w >> 16));
    }
    __syncthreads();
    for (int e = tid; e < n2; e += NT) {  // rows: H[i][k] = sum_j G[i][j] W^{jk}
        const int i = e / ps, k = e % ps;
        float2 acc = make_float2(0.f, 0.f);
        int t = 0;
        for (int j = 0; j < ps; ++j) {
            const float2 g = G[i * ps + j], w = a.twP[t];
            acc.x = fmaf(g.x, w.x, fmaf(-g.y, w.y, acc.x));
            acc.y = fmaf(g.x, w.y, fmaf(g.y, w.x, acc.y));
            t += k;
            t = t >= ps ? t - ps : t;
        }
        H[e] = acc;
    }
    __syncthreads();
    double pmax = 0.0;
    for (int e = tid; e < n2; e += NT) {  // columns: F[k1][k2] = sum_i H[i][k2] W^{i k1}
        const int k1 = e / ps, k2 = e % ps;
        float2 acc = make_float2(0.f, 0.f);
        int t = 0;
        for (int i = 0; i < ps; ++i) {
            const float2 h = H[i * ps + k2], w = a.twP[t];
            acc.x = fmaf(h.x, w.x, fmaf(-h.y, w.y, acc.x));
            acc.y = fmaf(h.x, w.y, fmaf(h.y, w.x, acc.y));
            t += k1;
            t = t >= ps ? t - ps : t;
        }
        G[e] = acc;
        pmax = fmax(pmax, (double)acc.x * acc.x + (double)acc.y * acc.y);
    }
    // block maximum of the bin power (double, non-negative: bits order as values)
    {
        unsigned long long u = (unsigned long long)__double_as_longlong(pmax);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long v = __shfl_xor_sync(0xffffffffu, u, o);
            u = v > u ? v : u;
        }
        unsigned long long* sc = reinterpret_cast<unsigned long long*>(red);
        if (lane == 0) sc[warp] = u;
        __syncthreads();
        u = sc[0];
#pragma unroll
        for (int w = 1; w < NT / 32; ++w) u = sc[w] > u ? sc[w] : u;
        __syncthreads();
        pmax = __longlong_as_double((long long)u);
    }
    // the surviving bins (real parts), in bin order, as (value, padded K1, K2)
    float* lv = reinterpret_cast<float*>(H);
    int* lk = reinterpret_cast<int*>(H) + n2;
    int* cntp = reinterpret_cast<int*>(red);
    const int h = ps / 2;
    if (warp == 0) {
        int cnt = 0;
        for (int e0 = 0; e0 < n2; e0 += 32) {
            const int e = e0 + lane;
            bool keep = false;
            float v = 0.f;
            int K = 0;
            if (e < n2) {
                const float2 f = G[e];
                const double p = (double)f.x * f.x + (double)f.y * f.y;
                const int k1 = e / ps, k2 = e % ps;
                v = p < 0.99 * pmax ? 0.f : f.x;
                const bool in1 = k1 < 2 * h, in2 = k2 < 2 * h;  // zeroPadFFT copies 2 (ps/2) rows and columns
                const int K1 = k1 < h ? k1 : a.intPSA - 2 * h + k1;
                const int K2 = k2 < h ? k2 : a.intPSR - 2 * h + k2;
                keep = v != 0.f && in1 && in2;
                K = (K1 << 16) | K2;
            }
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const int pos = cnt + __popc(m & ((1u << lane) - 1u));
                lv[pos] = v;
                lk[pos] = K;
            }
            cnt += __popc(m);
        }
        if (lane == 0) *cntp = cnt;
    }
    __syncthreads();
    const int nPeak = *cntp;
    const int i1 = a.intPSA / 2 - W / 2, j1 = a.intPSR / 2 - W / 2;
    for (int e = tid; e < W * W; e += NT) {
        const int i = e / W, j = e % W;
        float pr = 0.f, pim = 0.f;
        for (int q = 0; q < nPeak; ++q) {
            const int K1 = lk[q] >> 16, K2 = lk[q] & 0xffff;
            const int m1 = (int)(((long long)K1 * (i1 + i)) % a.intPSA);
            const int m2 = (int)(((long long)K2 * (j1 + j)) % a.intPSR);
            const float frac = (float)m1 / (float)a.intPSA + (float)m2 / (float)a.intPSR;
            float sn, cs;
            sincospif(2.0f * frac, &sn, &cs);
            pr = fmaf(lv[q], cs, pr);
            pim = fmaf(lv[q], sn, pim);
        }
        float cr = pr, ci = -pim, sc;
        if (fabsf(cr) < 1.0e-6f && fabsf(ci) < 1.0e-6f) {
            cr = 1.f;
            ci = 0.f;
            sc = 1.f;
        } else {
            sc = 1.0f / sqrtf(cr * cr + ci * ci);
        }
        const float2 z = X[i * RS + j];
        X[i * RS + j] = make_float2((z.x * cr - z.y * ci) * sc, (z.x * ci + z.y * cr) * sc);
    }
    __syncthreads();
}

template <int W, int NT, bool F32, bool GAUSS>
__global__ void __launch_bounds__(NT, (W >= 64 ? 2 : 3)) strack_cmplx_kernel(CmplxArgs a)
{
    using S = CmplxSmem<W, NT>;
    constexpr int RS = S::RS, IMG = S::IMG;
    constexpr int W2 = 2 * W;
    constexpr int N1 = sbfft::Split<W>::N1, N2 = sbfft::Split<W>::N2;
    static_assert((W * W) % NT == 0 && NT % W == 0, "whole rows per thread");
    constexpr int RPT = W * W / NT;  // consecutive rows per thread in the load phase
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* X = reinterpret_cast<float2*>(smem_raw);
    float2* Y = X + IMG;
    float2* Z = Y + IMG;
    float2* twW = Z + IMG;
    float2* tau = twW + W;
    float2* osD2 = tau + W;  // 16-byte aligned: every region before it is a multiple of 16 bytes
    float2* Yb = osD2 + S::OSD;
    float2* T = Yb + NFAST * NFAST;
    float* blk = reinterpret_cast<float*>(T + NFAST * OSW);
    double* red = reinterpret_cast<double*>(blk + NFAST * NFAST);
    int* azs = reinterpret_cast<int*>(red + (NT / 32 + 1) * 8);  // the patch's roll, set by thread 0
    const int tid = threadIdx.x;

    for (int e = tid; e < W; e += NT) {
        twW[e] = a.twW[e];
        tau[e] = a.tau[e];
    }
    __syncthreads();

    float* smf = reinterpret_cast<float*>(smem_raw);
    const float thr = F32 ? 1e-15f : 1e-9f;
    const float thrAll = thr * W * W;
    const int jc = tid % W, i0 = (tid / W) * RPT;  // load phase: column jc, rows i0 .. i0+RPT-1

    // list entries are loaded two patches ahead and plans one patch ahead,
    // so a patch's window loads never wait on the dependent list -> plan loads
    const int G = gridDim.x;
    int pNext = a.list[blockIdx.x];
    int pAfter = (int)blockIdx.x + G < a.nList ? a.list[blockIdx.x + G] : 0;
    PointPlan plNext = a.plan[pNext];
    for (int it = blockIdx.x; it < a.nList; it += G) {
        const int p = pNext;
        const PointPlan pl = plNext;
        if (it + G < a.nList) {
            pNext = pAfter;
            plNext = a.plan[pAfter];
            if (it + 2 * G < a.nList) pAfter = a.list[it + 2 * G];
        }
        // ---------------------------------------------------- getPatches
        // per-thread partial sums over the RPT rows in float, block totals in double
        float f[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        int nLow = 0;
        // batches of LB rows: every load of a batch is issued before any is
        // used (the Hanning taper and the byte order are predicates, not
        // branches, so nothing stops the compiler from hoisting them)
        constexpr int LB = load_batch(RPT);
        static_assert(RPT % LB == 0, "whole batches of rows");
        const bool msb = a.byteOrder == SB_MSB;
        const bool han = a.hanning != nullptr;
#pragma unroll
        for (int r0 = 0; r0 < RPT; r0 += LB) {
            using Raw = typename std::conditional<F32, uint2, uint32_t>::type;
            Raw w1[LB], w2[LB];
            float hv[LB];
#pragma unroll
            for (int u = 0; u < LB; ++u) {
                const int i = i0 + r0 + u;
                w1[u] = __ldg(reinterpret_cast<const Raw*>(a.img1) + ((size_t)(pl.a1 + i) * a.nr1 + pl.r1 + jc));
                w2[u] = __ldg(reinterpret_cast<const Raw*>(a.img2) + ((size_t)(pl.a2 + i) * a.nr2 + pl.r2 + jc));
                hv[u] = han ? __ldg(a.hanning + i * W + jc) : 1.f;
            }
#pragma unroll
            for (int u = 0; u < LB; ++u) {
            const int i = i0 + r0 + u;
            float2 z1 = decode_sample<F32>(w1[u], msb);
            float2 z2 = decode_sample<F32>(w2[u], msb);
            if (han) {
                z2.x *= hv[u];
                z2.y *= hv[u];
            }
            const float pw1 = __fadd_rn(__fmul_rn(z1.x, z1.x), __fmul_rn(z1.y, z1.y));
            const float pw2 = __fadd_rn(__fmul_rn(z2.x, z2.x), __fmul_rn(z2.y, z2.y));
            nLow += (pw1 < thr || pw2 < thr);
            f[0] += pw1;
            f[1] += pw2;
            f[2] += z1.x;
            f[3] += z1.y;
            f[4] += z2.x;
            f[5] += z2.y;
            X[i * RS + jc] = z1;
            Z[i * RS + jc] = z2;
            }
        }
        double s[7] = {f[0], f[1], f[2], f[3], f[4], f[5], (double)nLow};
        block_allsum<7, NT>(s, red);
        const bool haveData = !(s[6] > 20.0) && !(s[0] < thrAll || s[1] < thrAll);
        if (!haveData) {
            if (tid == 0) {
                a.rec[p].flags |= RF_DONE_C;
                a.rec[p].azset = -1;
                a.fit[it].point = p;
                a.fit[it].gate = 0;
                if constexpr (!GAUSS) {
                    a.peak[it].point = p;
                    a.peak[it].iC = PJ_NODATA;
                }
            }
            continue;  // uniform across the block
        }
        // ---------------------------------------------------- Doppler (lag-1 sums)
        // Each thread walks its own column run, the row below the run included.
        const double n = (double)(W * W);
        const double m1r = s[2] / n, m1i = s[3] / n, m2r = s[4] / n, m2i = s[5] / n;
        double d[4] = {0, 0, 0, 0};
        {
            float2 q1 = X[i0 * RS + jc], q2 = Z[i0 * RS + jc];
            double br1 = (double)q1.x - m1r, bi1 = (double)q1.y - m1i;
            double br2 = (double)q2.x - m2r, bi2 = (double)q2.y - m2i;
            const int rEnd = i0 + RPT < W ? RPT : RPT - 1;
#pragma unroll
            for (int r = 1; r <= RPT; ++r) {
                if (r <= rEnd) {
                    q1 = X[(i0 + r) * RS + jc];
                    q2 = Z[(i0 + r) * RS + jc];
                    const double ar1 = (double)q1.x - m1r, ai1 = (double)q1.y - m1i;
                    const double ar2 = (double)q2.x - m2r, ai2 = (double)q2.y - m2i;
                    d[0] += ar1 * br1 + ai1 * bi1;
                    d[1] += ai1 * br1 - ar1 * bi1;
                    d[2] += ar2 * br2 + ai2 * bi2;
                    d[3] += ai2 * br2 - ar2 * bi2;
                    br1 = ar1; bi1 = ai1;
                    br2 = ar2; bi2 = ai2;
                }
            }
        }
        block_allsum<4, NT>(d, red);
        // one thread evaluates the roll (two double atan2); the barriers of the
        // forward transforms publish it before the row pass reads it
        if (tid == 0) *azs = dop_shift(d[0], d[1], d[2], d[3], W, W);
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
                const float2 z = X[i * RS + j];
                X[i * RS + j] = make_float2((float)(z.x * cs - z.y * sn), (float)(z.x * sn + z.y * cs));
            }
            __syncthreads();
        }
        if (a.intf) phase_correct_int<W, RS, NT>(a, pl, X, Y, red);
        // ---------------------------------------------------- spectra of both patches (X and Z)
        sbfft::fft2d_smem<W, -1, 2, NT, RS, 2 * IMG>(X, twW);
        const int azShift = *azs;
        // ---------------------------------------------------- padded inverse
        // One dual row pass (over k2) makes R0 (e2 = 0, into Y) and R1 (e2 = 1,
        // times tau[k2], into Z) from the cross spectrum X conj(Z) with the
        // Doppler row shift folded in.  The per-row factor tau_e1[k1] commutes
        // with the row transform and is applied in the column passes, so two
        // row transforms serve the four parities.
        {
            const int sh = azShift;
            auto srcS = [X, Z, sh](int l, int k) {
                const int r = l + sh;
                const int o = (r >= W ? r - W : r) * RS + k;
                return sbfft::cconjmul(X[o], Z[o]);
            };
            auto mulTau = [tau](int, int k) { return tau[k]; };
            auto rowStore = [Y](int l, int k1, int k2, float2 z) {
                Y[(l % W) * RS + (l / W) * IMG + k1 + N1 * k2] = z;
            };
            sbfft::fft_lines_dual<N1, N2, 1, W, NT, RS, 1, IMG, true>(Y, srcS, mulTau, rowStore, twW);
        }
        // Dual column passes (over k1): R0 (Y) -> parities (0,0) into X and
        // (1,0) in place; R1 (Z) -> (0,1) into D and (1,1) in place.  Each ends
        // in |c| and the running argmax; the buffers are placed so that no pass
        // overwrites an input still needed or a finished plane.
        float pmax = 0.f;
        {
            auto mulTau = [tau](int, int k) { return tau[k]; };
            auto colY = [Y](int l, int k) { return Y[k * RS + l]; };
            sbfft::fft_lines_dual<N1, N2, 1, W, NT, 1, RS, IMG, false>(
                X, colY, mulTau, MagMax<W, N1, N2, 0>{smf + poff<W>(0), smf + poff<W>(2), pmax}, twW);
            float2* D = X + (W * W) / 2;  // spans the end of X and the start of Y
            auto colZ = [Z](int l, int k) { return Z[k * RS + l]; };
            sbfft::fft_lines_dual<N1, N2, 1, W, NT, 1, RS, 2 * IMG - (W * W) / 2, false>(
                D, colZ, mulTau, MagMax<W, N1, N2, 1>{smf + poff<W>(1), smf + poff<W>(3), pmax}, twW);
        }
        // ---------------------------------------------------- findCPeak
        int iMax, jMax;
        cpeak_from_planes<W, NT>(smf, pmax, reinterpret_cast<unsigned*>(red), iMax, jMax);
        double cMax;
        const bool rejected = (iMax < (NFAST / 2) || iMax > (W2 - NFAST / 2) || jMax < (NFAST / 2) ||
                               jMax > (W2 - NFAST / 2));
        if (rejected) {
            cMax = -1.0;
            iMax = -1000;
            jMax = -1000;
        }
        if constexpr (!GAUSS) {
            // ------------------------------------------------ hand the peak to the peak kernel
            // (overSampleC and the Gaussian-width samples run there, a warp per patch)
            PeakJob* pj = a.peak + it;
            constexpr int NB = NFAST * NFAST, NH = 4 * (NGAUSS + 3), NV = (NGAUSS + 3) * 4;
            if (!rejected) {
                for (int e = tid; e < NB + NH + NV; e += NT) {
                    int y, x;
                    if (e < NB) {
                        y = iMax - NFAST / 2 + e / NFAST;
                        x = jMax - NFAST / 2 + e % NFAST;
                    } else if (e < NB + NH) {
                        const int q = e - NB;
                        y = iMax - 2 + q / (NGAUSS + 3);
                        x = jMax - (NGAUSS / 2 + 2) + q % (NGAUSS + 3);
                    } else {
                        const int q = e - NB - NH;
                        y = iMax - (NGAUSS / 2 + 2) + q / 4;
                        x = jMax - 2 + q % 4;
                    }
                    // blk, hs, vs are consecutive: value e goes to float e of blk
                    if (y >= 0 && y < W2 && x >= 0 && x < W2) (&pj->blk[0][0])[e] = fmap<W>(smf, y, x);
                }
            }
            if (tid == 0) {
                pj->point = p;
                pj->iC = iMax;
                pj->jC = jMax;
                pj->p1 = p1;
                pj->p2 = p2;
                PointRec* r = &a.rec[p];
                r->azd = -(float)SB_LARGEINT;  // complexMatch resets aZDefocus (:379)
                r->azset = azShift;
                r->flags |= RF_DONE_C | RF_HD_C;
            }
            __syncthreads();
            continue;
        }
        // samples for gaussPeak1D x 2 through the peak (NOVER units in)
        auto fit_samples = [&](int iMx, int jMx) -> int {
            const int iM = iMx / NOVER, jM = jMx / NOVER;
            const int g =
                (iM - NGAUSS / 2) >= 0 && (iM + NGAUSS / 2) < W2 && (jM - NGAUSS / 2) >= 0 && (jM + NGAUSS / 2) < W2;
            if (g && tid < 2 * NGAUSS) {
                const int f = tid / NGAUSS, k = tid % NGAUSS;
                FitJob* fj = &a.fit[it];
                if (f == 0) {
                    fj->samp[0][k] = sqrtf(fmap<W>(smf, iM, jM - NGAUSS / 2 + k));
                } else {
                    fj->samp[1][k] = sqrtf(fmap<W>(smf, iM - NGAUSS / 2 + k, jM));
                }
                if (k == 0) fj->x0[f] = (f == 0 ? jM : iM) - NGAUSS / 2;
            }
            return g;
        };
        // cmpTrackGauss on the 2x grid (hanning correction as the oversampling's)
        const double scale = a.hanCorr / (sqrt(p1 * p2) * pow((double)(W * W), 2));
        if (!rejected) cMax = (double)sqrtf(fmap<W>(smf, iMax, jMax));
        gauss2d_peak<NT>([smf](int i, int j) { return sqrtf(fmap<W>(smf, i, j)); }, W2, scale,
                         reinterpret_cast<float*>(T), blk, iMax, jMax, cMax);
        const int gate = fit_samples(iMax, jMax);
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

template <int W, int NT, bool F32, bool GAUSS>
static cudaError_t launch_cmplx_t(const CmplxArgs& a, int nCta, cudaStream_t st)
{
    const size_t sm = CmplxSmem<W, NT>::bytes;
    cudaError_t e = cudaFuncSetAttribute(strack_cmplx_kernel<W, NT, F32, GAUSS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    strack_cmplx_kernel<W, NT, F32, GAUSS><<<nCta, NT, sm, st>>>(a);
    return cudaGetLastError();
}

template <int W, int NT>
static cudaError_t launch_cmplx(const CmplxArgs& a, int nCta, cudaStream_t st)
{
    const bool f32 = a.sampleType == SB_CFLOAT32;
    if (a.gauss)
        return f32 ? launch_cmplx_t<W, NT, true, true>(a, nCta, st) : launch_cmplx_t<W, NT, false, true>(a, nCta, st);
    return f32 ? launch_cmplx_t<W, NT, true, false>(a, nCta, st) : launch_cmplx_t<W, NT, false, false>(a, nCta, st);
}

template <int W, int NT>
static int occupancy_cmplx()
{
    int nb = 0;
    const size_t sm = CmplxSmem<W, NT>::bytes;
    cudaFuncSetAttribute(strack_cmplx_kernel<W, NT, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, strack_cmplx_kernel<W, NT, true, false>, NT, sm);
    return nb;
}

// Second thread count per window, for the autotuner (the default form's -gauss
// instantiation keeps the default count).
template <int W, int NT>
static cudaError_t launch_cmplx_alt(const CmplxArgs& a, int nCta, cudaStream_t st)
{
    const bool f32 = a.sampleType == SB_CFLOAT32;
    return f32 ? launch_cmplx_t<W, NT, true, false>(a, nCta, st) : launch_cmplx_t<W, NT, false, false>(a, nCta, st);
}

bool cmplx_supported(int W) { return W == 16 || W == 24 || W == 32 || W == 48 || W == 64; }

int cmplx_default_threads(int W)
{
    switch (W) {
    case 16: return 64;
    case 24: return 96;
    case 32: return 256;
    case 48: return 192;
    case 64: return 256;
    default: return 0;
    }
}

int cmplx_alt_threads(int W)
{
    switch (W) {
    case 16: return 128;
    case 24: return 192;
    case 32: return 128;
    case 48: return 384;
    case 64: return 512;
    default: return 0;
    }
}

int cmplx_blocks_per_sm(int W, int threads)
{
    const bool alt = threads != 0 && threads == cmplx_alt_threads(W);
    switch (W) {
    case 16: return alt ? occupancy_cmplx<16, 128>() : occupancy_cmplx<16, 64>();
    case 24: return alt ? occupancy_cmplx<24, 192>() : occupancy_cmplx<24, 96>();
    case 32: return alt ? occupancy_cmplx<32, 128>() : occupancy_cmplx<32, 256>();
    case 48: return alt ? occupancy_cmplx<48, 384>() : occupancy_cmplx<48, 192>();
    case 64: return alt ? occupancy_cmplx<64, 512>() : occupancy_cmplx<64, 256>();
    default: return 0;
    }
}

cudaError_t launch_strack_cmplx(int W, const CmplxArgs& a, int nCta, cudaStream_t st, int threads)
{
    const bool alt = threads != 0 && threads == cmplx_alt_threads(W) && !a.gauss;
    switch (W) {
    case 16: return alt ? launch_cmplx_alt<16, 128>(a, nCta, st) : launch_cmplx<16, 64>(a, nCta, st);
    case 24: return alt ? launch_cmplx_alt<24, 192>(a, nCta, st) : launch_cmplx<24, 96>(a, nCta, st);
    case 32: return alt ? launch_cmplx_alt<32, 128>(a, nCta, st) : launch_cmplx<32, 256>(a, nCta, st);
    case 48: return alt ? launch_cmplx_alt<48, 384>(a, nCta, st) : launch_cmplx<48, 192>(a, nCta, st);
    case 64: return alt ? launch_cmplx_alt<64, 512>(a, nCta, st) : launch_cmplx<64, 256>(a, nCta, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace sbk
