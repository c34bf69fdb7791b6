// strack_amps.cu -- amplitude tries of strack for small windows (Ws <= 64),
// one CTA per grid point with every array resident in shared memory.
//
// Same computation as strack_amp.cu (ampMatch / ampTrackFast,
// Strack/speckleTrack.c:398-597, getAmpPatches :1006-1189): per image the
// W x W spectrum, the 2W x 2W zero-padded inverse as four parity transforms
// (one dual row pass and two dual column passes, the Doppler roll and the
// parity factors folded into the gathers), intensity |c|^2 * scale written
// straight into the 2W x 2W pair plane z = (I1, I2); the no-data test, sqrt,
// mean removal; one packed forward 2W x 2W DFT of (A1 + i A2), the Hermitian
// split and cross spectrum folded into the inverse row pass, and the inverse
// column pass storing |c|^2 at its fftshifted position with a running
// maximum.  findCPeak is exact (the same |c|^2 rescan as the complex stage);
// the 8x8 -> 96x96 oversampling uses the real kernel D.
//
// Shared memory (Ws = 32): three Ws x (Ws+1) complex buffers F | R0 | X and
// the 2Ws x (2Ws+1) pair plane, ~65 KB: three CTAs per SM.  At Ws = 48 the
// layout needs 139 KB, one CTA per SM: 192 threads with up to 255 registers
// each (no spills) do the try 2.3x faster than the staged kernel that larger
// windows use (strack_amp.cu); 384 threads spilled.  At Ws = 64 the buffers
// alone take 226.5 KB, so the lean layout keeps the twiddle, parity and
// oversampling tables in global memory (read through L1), puts the
// oversampling scratch in the spectrum buffer (idle by then) and sizes the
// block reductions for four values: 232,224 bytes, one CTA per SM.
#include <cuda_runtime.h>

#include "strack_device.cuh"
#include "strack_kernels.h"

namespace sbk {

template <int WS, int NT>
struct AmpsSmem {
    static constexpr int N = 2 * WS;
    static constexpr int RS = WS + 1;
    static constexpr int S = WS * RS;       // one Ws buffer, float2
    static constexpr int ZS = N * (N + 1);  // pair plane, float2
    static constexpr int OSD = OSW * NFAST / 2 + 16;
    static constexpr size_t full = sizeof(float2) * (3 * S + ZS + 2 * WS + N + OSD + NFAST * NFAST + NFAST * OSW) +
                                   sizeof(float) * NFAST * NFAST + sizeof(double) * (NT / 32 + 1) * 8 + 64;
    static constexpr bool LEAN = full > 227 * 1024;
    // lean: block_allsum of at most four values needs (warps + 1) x 4 doubles
    static constexpr size_t bytes = LEAN ? sizeof(float2) * (3 * S + ZS) + sizeof(double) * (NT / 32 + 1) * 4 : full;
    static_assert(bytes <= 227 * 1024, "one CTA's dynamic shared memory");
};

// Exact findCPeak over an N x N plane of |c|^2 stored at fftshifted positions
// (y, x), given each thread's running maximum of |c|^2: the largest
// sqrtf(|c|^2) > 0, ties to the smallest cpeak_rank(y, x, N/2).  sqrtf is
// correctly rounded and monotone, so every tie has |c|^2 within 2^-20 of the
// maximum and only those positions are ranked.  Returns y * N + x, or -1 when
// nothing is above 0.
template <int N, int NT>
__device__ __forceinline__ int cpeak_plane(const float* mag, float pmax, unsigned* iscr)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned u = __reduce_max_sync(0xffffffffu, __float_as_uint(pmax));  // |c|^2 >= 0: bits order as values
    if (lane == 0) iscr[warp] = u;
    __syncthreads();
    u = iscr[0];
#pragma unroll
    for (int w = 1; w < NT / 32; ++w) u = max(u, iscr[w]);
    __syncthreads();
    const float pm = __uint_as_float(u);
    if (!(pm > 0.f)) return -1;  // uniform
    const float sm = sqrtf(pm);
    const float lo = pm * (1.0f - 1.0f / 1048576.0f);
    unsigned best = 0xffffffffu;
    for (int e = tid; e < N * N / 4; e += NT) {
        const float4 v = reinterpret_cast<const float4*>(mag)[e];
        if (fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)) < lo) continue;  // candidates are rare
        const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            if (vv[c] >= lo && sqrtf(vv[c]) == sm) {
                const int idx = 4 * e + c;
                best = min(best, (unsigned)cpeak_rank(idx / N, idx % N, N / 2));
            }
        }
    }
    best = __reduce_min_sync(0xffffffffu, best);
    if (lane == 0) iscr[warp] = best;
    __syncthreads();
    best = iscr[0];
#pragma unroll
    for (int w = 1; w < NT / 32; ++w) best = min(best, iscr[w]);
    __syncthreads();
    const int h = N / 2, q = best & 3, ij = best >> 2;
    const int y = ij / h + ((q == 1 || q == 2) ? h : 0);
    const int x = ij % h + ((q == 1 || q == 3) ? h : 0);
    return y * N + x;
}

template <int WS, int NT, bool GAUSS>
__global__ void __launch_bounds__(NT, (WS == 32 ? 3 : (WS >= 48 ? 1 : 2))) strack_amps_kernel(AmpArgs a)
{
    using M = AmpsSmem<WS, NT>;
    constexpr int N = M::N, RS = M::RS, S = M::S, ZR = N + 1;
    constexpr int W1 = sbfft::Split<WS>::N1, W2 = sbfft::Split<WS>::N2;
    constexpr int Z1 = sbfft::Split<N>::N1, Z2 = sbfft::Split<N>::N2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* F = reinterpret_cast<float2*>(smem_raw);
    float2* R0 = F + S;
    float2* X = R0 + S;
    float2* z = X + S;
    float* zf = reinterpret_cast<float*>(z);
    const int tid = threadIdx.x;
    const float2* twWs;
    const float2* tau;
    const float2* twN;
    const float* osD;
    float2* Yb;
    float2* T;
    float* blk;
    double* red;
    if constexpr (M::LEAN) {
        twWs = a.twWs;
        tau = a.tau;
        twN = a.tw2Ws;
        osD = reinterpret_cast<const float*>(a.osD);
        Yb = F;  // the spectrum buffer is idle once the pair plane is formed
        T = Yb + NFAST * NFAST;
        blk = reinterpret_cast<float*>(T + NFAST * OSW);
        red = reinterpret_cast<double*>(z + M::ZS);
    } else {
        float2* sTwWs = z + M::ZS;
        float2* sTau = sTwWs + WS;
        float2* sTwN = sTau + WS;
        float2* osD2 = sTwN + N;  // 16-byte aligned: every region before it has an even float2 count
        Yb = osD2 + M::OSD;
        T = Yb + NFAST * NFAST;
        blk = reinterpret_cast<float*>(T + NFAST * OSW);
        red = reinterpret_cast<double*>(blk + NFAST * NFAST);
        for (int e = tid; e < WS; e += NT) {
            sTwWs[e] = a.twWs[e];
            sTau[e] = a.tau[e];
        }
        for (int e = tid; e < N; e += NT) sTwN[e] = a.tw2Ws[e];
        for (int e = tid; e < M::OSD; e += NT) osD2[e] = a.osD[e];
        __syncthreads();
        twWs = sTwWs;
        tau = sTau;
        twN = sTwN;
        osD = reinterpret_cast<const float*>(osD2);
    }

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
        auto load = [&](float2* dst, int q) {
            for (int e = tid; e < WS * WS; e += NT) {
                const int i = e / WS, j = e % WS;
                dst[i * RS + j] = q == 0 ? load_sample(a.img1, a.nr1, a1a + i, r1a + j, a.sampleType, a.byteOrder)
                                         : load_sample(a.img2, a.nr2, a2a + i, r2a + j, a.sampleType, a.byteOrder);
            }
        };
        // ---------------------------------------------------- Doppler
        int azShift;
        const bool ownDop = (a.noComplex != 0 && st == 1);
        if (ownDop) {
            // estDopCarrier1(im1in, im2in, wAa, wRa) (speckleTrack.c:1141-1144)
            load(F, 0);
            load(R0, 1);
            __syncthreads();
            double m[4] = {0, 0, 0, 0};
            for (int e = tid; e < WS * WS; e += NT) {
                const float2 z1 = F[(e / WS) * RS + e % WS], z2 = R0[(e / WS) * RS + e % WS];
                m[0] += z1.x; m[1] += z1.y; m[2] += z2.x; m[3] += z2.y;
            }
            block_allsum<4, NT>(m, red);
            const double n = (double)(WS * WS);
            const double m1r = m[0] / n, m1i = m[1] / n, m2r = m[2] / n, m2i = m[3] / n;
            double d[4] = {0, 0, 0, 0};
            for (int e = tid; e < (WS - 1) * WS; e += NT) {
                const int i = e / WS, j = e % WS;
                const float2 p0 = F[i * RS + j], p1 = F[(i + 1) * RS + j];
                double ar = (double)p1.x - m1r, ai = (double)p1.y - m1i, br = (double)p0.x - m1r,
                       bi = (double)p0.y - m1i;
                d[0] += ar * br + ai * bi;
                d[1] += ai * br - ar * bi;
                const float2 q0 = R0[i * RS + j], q1 = R0[(i + 1) * RS + j];
                ar = (double)q1.x - m2r; ai = (double)q1.y - m2i; br = (double)q0.x - m2r; bi = (double)q0.y - m2i;
                d[2] += ar * br + ai * bi;
                d[3] += ai * br - ar * bi;
            }
            block_allsum<4, NT>(d, red);
            azShift = dop_shift(d[0], d[1], d[2], d[3], a.wAa, a.wA);
        } else {
            azShift = a.azEff ? a.azEff[p] : a.rec[p].azset;
            if (azShift < 0) azShift = 0;
            load(F, 0);
            __syncthreads();
        }
        const int az = (int)((float)azShift * (float)WS / (float)a.wA);
        // ---------------------------------------------------- detected images
        float cnt = 0.f;
        double s1 = 0.0, s2 = 0.0;
#pragma unroll 1
        for (int q = 0; q < 2; ++q) {
            if (q == 1) {
                load(F, 1);
                __syncthreads();
            }
            sbfft::fft2d_smem<WS, -1, 1, NT, RS, 0>(F, twWs);
            // layout F | R0 | X.  Rows: R0 = row IDFT(F), F = row IDFT(F tau[k2])
            // (the second output of a dual pass based at R0 is F, offset -S).
            auto rowF = [F](int l, int k) { return F[l * RS + k]; };
            auto tauK = [tau](int, int k) { return tau[k]; };
            auto rowStore = [R0](int l, int k1, int k2, float2 v) {
                R0[(l % WS) * RS - (l / WS) * S + k1 + W1 * k2] = v;
            };
            sbfft::fft_lines_dual<W1, W2, 1, WS, NT, RS, 1, -S, true>(R0, rowF, tauK, rowStore, twWs);
            // Columns: parity (0, e2) through X, (1, e2) in place over R_e2; the
            // last step writes |c|^2 * scale into component q of the pair plane.
            // The second image also counts samples under the threshold in either
            // image; each image sums its own intensities.
            auto epi = [&](int e2) {
                return [&, e2](int l, int k1, int k2, float2 v) {
                    const int e1 = l >= WS, m2 = l - (e1 ? WS : 0), m1 = k1 + W1 * k2;
                    const float I = (v.x * v.x + v.y * v.y) * scale;
                    const int o = 2 * ((2 * m1 + e1) * ZR + 2 * m2 + e2);
                    if (q == 0) {
                        zf[o] = I;
                        s1 += I;
                    } else {
                        zf[o + 1] = I;
                        s2 += I;
                        cnt += (zf[o] < thr || I < thr) ? 1.f : 0.f;
                    }
                };
            };
            auto colR0 = [R0, az](int l, int k) {
                const int r = k + az >= WS ? k + az - WS : k + az;
                return R0[r * RS + l];
            };
            sbfft::fft_lines_dual<W1, W2, 1, WS, NT, 1, RS, -S, true>(X, colR0, tauK, epi(0), twWs);  // X, R0
            auto colR1 = [F, az](int l, int k) {
                const int r = k + az >= WS ? k + az - WS : k + az;
                return F[r * RS + l];
            };
            sbfft::fft_lines_dual<W1, W2, 1, WS, NT, 1, RS, -2 * S, true>(X, colR1, tauK, epi(1), twWs);  // X, F
        }
        // ---------------------------------------------------- tests, amplitude, mean removal
        double r3[3] = {cnt, s1, s2};
        block_allsum<3, NT>(r3, red);
        const bool hd = !(r3[0] > 20.0) && !(r3[1] < 1.0e-6 || r3[2] < 1.0e-6);
        if (!hd) {
            if (tid == 0) {
                a.rec[p].flags |= (st == 1 ? RF_DONE_S : RF_DONE_L);
                if (ownDop) a.rec[p].azset = azShift;
                a.fit[it].point = p;
                a.fit[it].gate = -1;  // no data: nothing for the fit kernel to decide
            }
            __syncthreads();
            continue;  // uniform across the block
        }
        double av[2] = {0, 0};
        for (int e = tid; e < N * N; e += NT) {
            const int o = (e / N) * ZR + e % N;
            float2 v = z[o];
            v.x = sqrtf(v.x);
            v.y = sqrtf(v.y);
            z[o] = v;
            av[0] += v.x;
            av[1] += v.y;
        }
        block_allsum<2, NT>(av, red);
        const double nn = (double)N * N;
        const double avg1 = av[0] / nn, avg2 = av[1] / nn;
        double pw[2] = {0, 0};
        for (int e = tid; e < N * N; e += NT) {
            const int o = (e / N) * ZR + e % N;
            float2 v = z[o];
            if (v.x > 1.0e-20f) v.x = (float)((double)v.x - avg1);
            v.y = (float)((double)v.y - avg2);
            z[o] = v;
            pw[0] += (double)(v.x * v.x);
            pw[1] += (double)(v.y * v.y);
        }
        block_allsum<2, NT>(pw, red);
        const double p1 = pw[0] / nn, p2 = pw[1] / nn;
        // ---------------------------------------------------- correlation
        sbfft::fft2d_smem<N, -1, 1, NT, ZR, 0>(z, twN);
        // inverse rows read the cross spectrum F1 conj(F2) of the packed pair:
        // F1 = (Z[k] + conj Z[-k]) / 2, F2 = (Z[k] - conj Z[-k]) / 2i
        auto cross = [z](int l, int k) {
            const float2 Zk = z[l * ZR + k];
            const float2 Zm = z[(l == 0 ? 0 : N - l) * ZR + (k == 0 ? 0 : N - k)];
            const float2 f1 = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
            const float2 f2 = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
            return sbfft::cconjmul(f1, f2);
        };
        auto zStore = [z](int l, int k1, int k2, float2 v) { z[l * ZR + k1 + Z1 * k2] = v; };
        sbfft::fft_lines_io<Z1, Z2, 1, N, N, NT, ZR, 1, 0, true>(z, cross, zStore, twN);
        // inverse columns: |c|^2 at the fftshifted position, running maximum
        float pmax = 0.f;
        {
            auto colz = [z](int l, int k) { return z[k * ZR + l]; };
            auto mag = [zf, &pmax](int l, int k1, int k2, float2 v) {
                const int cy = k1 + Z1 * k2, cx = l;
                const int y = cy + WS < N ? cy + WS : cy - WS;
                const int x = cx + WS < N ? cx + WS : cx - WS;
                const float pv = v.x * v.x + v.y * v.y;
                zf[y * N + x] = pv;
                pmax = fmaxf(pmax, pv);
            };
            sbfft::fft_lines_io<Z1, Z2, 1, N, N, NT, 1, ZR, 0, false>(z, colz, mag, twN);
        }
        // ---------------------------------------------------- findCPeak, fits, oversampling
        const int pos = cpeak_plane<N, NT>(zf, pmax, reinterpret_cast<unsigned*>(red));
        int iMax = 0, jMax = 0;
        double cMax = 0.0;
        if (pos >= 0) {
            iMax = pos / N;
            jMax = pos % N;
            cMax = (double)sqrtf(zf[pos]);
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
                fj->samp[0][k] = sqrtf(zf[iMax * N + (jMax - NGAUSS / 2 + k)]);
            else
                fj->samp[1][k] = sqrtf(zf[(iMax - NGAUSS / 2 + k) * N + jMax]);
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
            gauss2d_peak<NT>([=](int i, int j) { return sqrtf(zf[i * N + j]); }, N, scale, reinterpret_cast<float*>(T), blk, iMax,
                             jMax, cMax);
        } else if (iMax >= -999) {
            // 8x8 -> 96x96 oversampling (used unless the fit kernel takes the
            // early return of ampTrackFast, :551-553)
            if (tid < NFAST * NFAST) {
                const int t1 = tid / NFAST, t2 = tid % NFAST;
                blk[tid] = sqrtf(zf[(iMax - NFAST / 2 + t1) * N + (jMax - NFAST / 2 + t2)]);
            }
            __syncthreads();
            const ArgMax ob = oversample_peak_real<NT>(blk, osD, Yb, T, reinterpret_cast<unsigned long long*>(red));
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

template <int WS, int NT, bool GAUSS>
static cudaError_t launch_amps_t(const AmpArgs& a, int nCta, cudaStream_t st)
{
    const size_t sm = AmpsSmem<WS, NT>::bytes;
    cudaError_t e = cudaFuncSetAttribute(strack_amps_kernel<WS, NT, GAUSS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    strack_amps_kernel<WS, NT, GAUSS><<<nCta, NT, sm, st>>>(a);
    return cudaGetLastError();
}

template <int WS, int NT>
static cudaError_t launch_amps(const AmpArgs& a, int nCta, cudaStream_t st)
{
    return a.gauss ? launch_amps_t<WS, NT, true>(a, nCta, st) : launch_amps_t<WS, NT, false>(a, nCta, st);
}

template <int WS, int NT>
static int occupancy_amps()
{
    int nb = 0;
    const size_t sm = AmpsSmem<WS, NT>::bytes;
    cudaFuncSetAttribute(strack_amps_kernel<WS, NT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, strack_amps_kernel<WS, NT, false>, NT, sm);
    return nb;
}

bool amps_supported(int Ws) { return Ws == 16 || Ws == 24 || Ws == 32 || Ws == 48 || Ws == 64; }

int amps_blocks_per_sm(int Ws)
{
    switch (Ws) {
    case 16: return occupancy_amps<16, 64>();
    case 24: return occupancy_amps<24, 192>();
    case 32: return occupancy_amps<32, 256>();
    case 48: return occupancy_amps<48, 192>();
    case 64: return occupancy_amps<64, 256>();
    default: return 0;
    }
}

cudaError_t launch_strack_amps(int Ws, const AmpArgs& a, int nCta, cudaStream_t st)
{
    switch (Ws) {
    case 16: return launch_amps<16, 64>(a, nCta, st);
    case 24: return launch_amps<24, 192>(a, nCta, st);
    case 32: return launch_amps<32, 256>(a, nCta, st);
    case 48: return launch_amps<48, 192>(a, nCta, st);
    case 64: return launch_amps<64, 256>(a, nCta, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace sbk
