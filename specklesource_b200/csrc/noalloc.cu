// noalloc.cu -- sb_amp_match_noalloc: the amplitude try of strack on
// caller-supplied patch pairs, with a workspace that is a file-scope device
// array instead of a cudaMalloc'd buffer, for callers that cannot allocate
// device memory while they run (see include/speckle_b200.h).
//
// The kernel is a variant of strack_amp_kernel (strack_amp.cu): same stages,
// but patches come from a contiguous caller array, the results go to plain
// per-patch arrays, the constant tables are computed in shared memory by each
// CTA, and the per-CTA workspace is a slice of g_noalloc_scratch.
#include <cuda_runtime.h>

#include "capi_internal.h"
#include "strack_device.cuh"

namespace sbk {

constexpr size_t kNoallocScratchElems = SB_NOALLOC_SCRATCH_BYTES / sizeof(float2);

// The workspace: every GPU that loads the library holds it until exit.
static __device__ __align__(256) float2 g_noalloc_scratch[kNoallocScratchElems];

template <int WS>
struct NoallocCfg {
    static constexpr int N = 2 * WS;
    static constexpr int NT = 256;
    static constexpr int TILE = sbfft::StagedTile<N, false>::elems > sbfft::StagedTile<WS, false>::elems
                                    ? sbfft::StagedTile<N, false>::elems
                                    : sbfft::StagedTile<WS, false>::elems;
    static constexpr size_t smem = sizeof(float2) * (TILE + WS + N + WS + OSW * NFAST + NFAST * OSW) +
                                   sizeof(float) * NFAST * NFAST + sizeof(double) * (NT / 32 + 1) * 8 +
                                   sizeof(int) * (3 * (NT / 32) + 8) + 64;
    // F1, F2, work (WS^2 each), z (N^2), mag (N^2 floats)
    static constexpr size_t perCta = (size_t)3 * WS * WS + (size_t)N * N + (size_t)N * N / 2;
};

struct NoallocArgs {
    const float2* p1;
    const float2* p2;
    int nPatch;
    const int* azShift;
    double* cMax;
    int* iMax;
    int* jMax;
    int* haveData;
    float2* scratch;  // device address of g_noalloc_scratch
};

template <int WS>
__global__ void __launch_bounds__(NoallocCfg<WS>::NT) amp_noalloc_kernel(NoallocArgs a)
{
    using C = NoallocCfg<WS>;
    constexpr int N = C::N, NT = C::NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* tile = reinterpret_cast<float2*>(smem_raw);
    float2* twWs = tile + C::TILE;
    float2* twN = twWs + WS;
    float2* tau = twN + N;
    float2* osA = tau + WS;
    float2* T = osA + OSW * NFAST;
    float* blk = reinterpret_cast<float*>(T + NFAST * OSW);
    double* red = reinterpret_cast<double*>(blk + NFAST * NFAST);
    int* isc = reinterpret_cast<int*>(red + (NT / 32 + 1) * 8);
    const int tid = threadIdx.x;

    // constant tables (forward twiddles, parity twiddles, oversampling matrix)
    for (int e = tid; e < WS; e += NT) {
        double s, c;
        sincospi(-2.0 * e / WS, &s, &c);
        twWs[e] = make_float2((float)c, (float)s);
        sincospi((double)e / WS, &s, &c);
        const double sg = e < WS / 2 ? 1.0 : -1.0;
        tau[e] = make_float2((float)(sg * c), (float)(sg * s));
    }
    for (int e = tid; e < N; e += NT) {
        double s, c;
        sincospi(-2.0 * e / N, &s, &c);
        twN[e] = make_float2((float)c, (float)s);
    }
    for (int e = tid; e < OSW * NFAST; e += NT) {
        const int n = e / NFAST, t = e % NFAST;
        const int d = (n + 24) - NOVER * t;
        double re = 0, im = 0;
        for (int f = -NFAST / 2; f < NFAST / 2; ++f) {
            double s, c;
            sincospi(2.0 * f * d / (NFAST * NOVER), &s, &c);
            re += c;
            im += s;
        }
        osA[e] = make_float2((float)re, (float)im);
    }
    __syncthreads();

    float2* F1 = a.scratch + (size_t)blockIdx.x * C::perCta;
    float2* F2 = F1 + WS * WS;
    float2* work = F2 + WS * WS;
    float2* z = work + WS * WS;
    float* mag = reinterpret_cast<float*>(z + (size_t)N * N);
    const float thr = 1.0e-15f;
    const float scale = (float)(1. / ((size_t)WS * WS * WS * WS * OS * OS * OS));

    for (int k = blockIdx.x; k < a.nPatch; k += gridDim.x) {
        const float2* s1 = a.p1 + (size_t)k * WS * WS;
        const float2* s2 = a.p2 + (size_t)k * WS * WS;
        double m[4] = {0, 0, 0, 0};
        for (int e = tid; e < WS * WS; e += NT) {
            const float2 z1 = s1[e], z2 = s2[e];
            F1[e] = z1;
            F2[e] = z2;
            m[0] += z1.x; m[1] += z1.y; m[2] += z2.x; m[3] += z2.y;
        }
        int az;
        if (a.azShift == nullptr) {
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
            az = dop_shift(d[0], d[1], d[2], d[3], WS, WS);
        } else {
            az = a.azShift[k] % WS;  // a roll is periodic in wa
            if (az < 0) az += WS;
        }
        __syncthreads();
        sbfft::fft2d_staged<WS, -1, NT>(F1, tile, twWs, nullptr);
        sbfft::fft2d_staged<WS, -1, NT>(F2, tile, twWs, nullptr);
#pragma unroll 1
        for (int q = 0; q < 2; ++q) {
            const float2* F = q == 0 ? F1 : F2;
#pragma unroll 1
            for (int par = 0; par < 4; ++par) {
                const int e1 = par >> 1, e2 = par & 1;
                for (int e = tid; e < WS * WS; e += NT) {
                    const int k1 = e / WS, k2 = e % WS;
                    float2 v = F[((k1 + az) % WS) * WS + k2];
                    if (e1) v = sbfft::cmul(v, tau[k1]);
                    if (e2) v = sbfft::cmul(v, tau[k2]);
                    work[e] = v;
                }
                __syncthreads();
                sbfft::fft2d_staged<WS, 1, NT>(work, tile, twWs, nullptr);
                for (int e = tid; e < WS * WS; e += NT) {
                    const int m1 = e / WS, m2 = e % WS;
                    const float2 w = work[e];
                    float* zz = reinterpret_cast<float*>(&z[(size_t)(2 * m1 + e1) * N + 2 * m2 + e2]);
                    zz[q] = (w.x * w.x + w.y * w.y) * scale;
                }
                __syncthreads();
            }
        }
        double r3[3] = {0, 0, 0};
        for (int e = tid; e < N * N; e += NT) {
            const float2 v = z[e];
            if (v.x < thr || v.y < thr) r3[0] += 1.0;
            r3[1] += v.x;
            r3[2] += v.y;
        }
        block_allsum<3, NT>(r3, red);
        const bool hd = !(r3[0] > 20.0) && !(r3[1] < 1.0e-6 || r3[2] < 1.0e-6);
        if (!hd) {
            if (tid == 0) {
                a.haveData[k] = 0;
                a.cMax[k] = 0.0;
                a.iMax[k] = -1000;
                a.jMax[k] = -1000;
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
        sbfft::fft2d_staged<N, -1, NT>(z, tile, twN, nullptr);
        for (int e = tid; e < N * N; e += NT) {
            const int k1 = e / N, k2 = e % N;
            const int e2 = ((N - k1) % N) * N + ((N - k2) % N);
            if (e2 < e) continue;
            const float2 Zk = z[e], Zm = z[e2];
            const float2 f1 = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
            const float2 f2 = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
            const float2 s = sbfft::cconjmul(f1, f2);
            z[e] = s;
            z[e2] = make_float2(s.x, -s.y);
        }
        __syncthreads();
        sbfft::fft2d_staged<N, 1, NT>(z, tile, twN, nullptr);
        ArgMax best;
        best.v = 0.f;
        best.rank = 0x7fffffff;
        best.pos = 0;
        for (int e = tid; e < N * N; e += NT) {
            const int cy = e / N, cx = e % N;
            const float2 c = z[e];
            const float v = sqrtf(c.x * c.x + c.y * c.y);
            const int y = cy + WS < N ? cy + WS : cy - WS;
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
        } else {
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
            a.haveData[k] = 1;
            a.cMax[k] = cMax;
            a.iMax[k] = iMax;
            a.jMax[k] = jMax;
        }
        __syncthreads();
    }
}

template <int WS>
static cudaError_t launch_noalloc(const NoallocArgs& a, int numSM, cudaStream_t st)
{
    using C = NoallocCfg<WS>;
    cudaError_t e =
        cudaFuncSetAttribute(amp_noalloc_kernel<WS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem);
    if (e != cudaSuccess) return e;
    long long nCta = 2LL * numSM;
    const long long fit = (long long)(kNoallocScratchElems / C::perCta);
    if (nCta > fit) nCta = fit;
    if (nCta > a.nPatch) nCta = a.nPatch;
    amp_noalloc_kernel<WS><<<(unsigned)nCta, C::NT, C::smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace sbk

using namespace sbk;

// Loads this file's module (which allocates g_noalloc_scratch on the current
// device) and all five kernel instances, so that neither happens inside a
// later sb_amp_match_noalloc call.  Called by sb_context_create with the
// context's device current.
cudaError_t sb_noalloc_prepare()
{
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa;
    if ((e = cudaFuncGetAttributes(&fa, amp_noalloc_kernel<16>)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&fa, amp_noalloc_kernel<24>)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&fa, amp_noalloc_kernel<32>)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&fa, amp_noalloc_kernel<48>)) != cudaSuccess) return e;
    return cudaFuncGetAttributes(&fa, amp_noalloc_kernel<64>);
}

extern "C" int sb_amp_match_noalloc(sb_context* c, const float* patches1, const float* patches2, int32_t nPatch,
                                    int32_t wa, const int32_t* azShift, double* cMax, int32_t* iMax, int32_t* jMax,
                                    int32_t* haveData)
{
    if (!c) return SB_ERR_ARG;
    c->err.clear();
    c->launches = 0;
    if (!patches1 || !patches2 || !cMax || !iMax || !jMax || !haveData)
        return sb_ctx_fail(c, SB_ERR_ARG, "null pointer argument");
    if (nPatch <= 0) return sb_ctx_fail(c, SB_ERR_ARG, "nPatch must be positive");
    if (wa > SB_NOALLOC_MAX_WA)
        return sb_ctx_fail(c, SB_ERR_ARG, "wa=%d exceeds the allocation-free maximum %d", wa, SB_NOALLOC_MAX_WA);
    if (wa != 16 && wa != 24 && wa != 32 && wa != 48 && wa != 64)
        return sb_ctx_fail(c, SB_ERR_ARG, "wa=%d not supported (16, 24, 32, 48 or 64)", wa);
    int nDev = 0;
    cudaError_t e = cudaGetDeviceCount(&nDev);
    if (e != cudaSuccess) return sb_ctx_cuda(c, e, "cudaGetDeviceCount");
    if (c->device < 0 || c->device >= nDev) return sb_ctx_fail(c, SB_ERR_ARG, "device ordinal out of range");
    e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return sb_ctx_cuda(c, e, "cudaSetDevice");
    if (c->noallocPrep != cudaSuccess) return sb_ctx_cuda(c, c->noallocPrep, "loading the allocation-free kernels");
    // The array's device address, looked up in the current CUDA context on
    // every call (the module is loaded already, so this allocates nothing).
    void* scratch = nullptr;
    e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
    if (e != cudaSuccess) return sb_ctx_cuda(c, e, "cudaGetSymbolAddress(workspace)");
    NoallocArgs a;
    a.p1 = reinterpret_cast<const float2*>(patches1);
    a.p2 = reinterpret_cast<const float2*>(patches2);
    a.nPatch = nPatch;
    a.azShift = azShift;
    a.cMax = cMax;
    a.iMax = iMax;
    a.jMax = jMax;
    a.haveData = haveData;
    a.scratch = reinterpret_cast<float2*>(scratch);
    switch (wa) {
    case 16: e = launch_noalloc<16>(a, c->numSM, c->stream); break;
    case 24: e = launch_noalloc<24>(a, c->numSM, c->stream); break;
    case 32: e = launch_noalloc<32>(a, c->numSM, c->stream); break;
    case 48: e = launch_noalloc<48>(a, c->numSM, c->stream); break;
    default: e = launch_noalloc<64>(a, c->numSM, c->stream); break;
    }
    if (e != cudaSuccess) return sb_ctx_cuda(c, e, "amp_noalloc_kernel");
    c->launches = 1;
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return sb_ctx_cuda(c, e, "sb_amp_match_noalloc");
    return SB_OK;
}
