// strack_cmplx_tc.cu -- the complex (speckle) matching stage of strack with
// the patch transforms as split-BF16 DFT-GEMMs on the tcgen05 tensor cores
// (the "split-BF16" form; strack_cmplx.cu is the plain FP32 form).
//
// Same stage as strack_cmplx.cu -- getPatches (Strack/speckleTrack.c:
// 1194-1330), estDopCarrier1 (Strack/dopplerEstimation.c:25-88),
// cmpPSWithPad (:604-643), the IFFT of cmpTrackFast (:648-709) and findCPeak
// (:744-805) -- for W = 64, handing the coarse peak to strack_peak.cu like the
// FP32 form.  Only the transforms change:
//
//   * a 64-point DFT over 128 lines is one real GEMM D[128 x 128] =
//     A[128 x 128] . B[128 x 128] in block form: A = [Re | Im] of the lines,
//     B = [[Fr, Fi], [-Fi, Fr]] with F[t][n] = exp(-2 pi i t n / 64); issued
//     as four 128 x 64 x 64 products (the minus sign by the MMA's negate-A
//     bit), each K = 64 as four K = 16 steps;
//   * split BF16, three products: x = hi + lo with hi = bf16(x),
//     lo = bf16(x - hi), for both operands; D accumulates hi.hi + hi.lo +
//     lo.hi in FP32 in TMEM (the lo.lo term, ~2^-16 relative, is dropped);
//   * the DFT matrix (hi, lo of Fr, Fi) stays in shared memory for the
//     CTA's lifetime; the line data are rewritten into the A operand between
//     passes straight from TMEM, so no intermediate leaves the SM.
//
// Six GEMM passes per patch (M = 128 lines each):
//   F1  K-major A: line = (window w, range column k), K = azimuth row i:
//       D1[(w,k)][n1] = sum_i X_w[i][k] F[i][n1]
//   F2  MN-major A (thread row = K): D2[(w,n1)][n2] = sum_k D1[(w,k)][n1] F[k][n2]
//       = the 2-D spectra Z_w[n1][n2]
//   the cross spectrum S = Z_1 conj(Z_2), rolled by the Doppler shift
//       X'[k1][k2] = S[(k1 + azShift) mod 64][k2] (cmpPSWithPad's quadrant map)
//   I1_e1 (e1 = 0, 1)  MN-major: the padded 128-point inverse along k1 as the
//       parity pair of 64-point inverses (strack_cmplx.cu), lines (e2, k2):
//       D3_e1[(e2,k2)][m1] = sum_k1 X'[k1][k2] tau_e1[k1] tau_e2[k2] G[k1][m1]
//   I2_e1  MN-major: D4_e1[(e2,m1)][m2] = sum_k2 D3_e1[(e2,k2)][m1] G[k2][m2]
//       = c[2 m1 + e1][2 m2 + e2], the 128 x 128 correlation surface.
// Every pass is a forward DFT: the inverses use inverse(x) = conj(forward(
// conj(x))), with the conjugates folded into the cross spectrum (conj(S) =
// conj(Z_1) Z_2) and the surface used as |c|^2 only.
//
// One CTA of 256 threads (8 warps) per patch, persistent over the list, two
// CTAs per SM: 100 KB of shared memory (A operand 64 KB, DFT matrix 32 KB) and
// 256 TMEM columns each (two 128-column accumulators).  Two threads share each
// TMEM lane L = line L of every pass: warps w and w + 4 read lanes
// 32 (w mod 4) .. +31 and own the halves [0, 32) and [32, 64) of the line's
// 64 values.  Waits on the MMA completion barrier are bounded: on time-out the
// kernel records an error and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "strack_device.cuh"
#include "strack_kernels.h"

namespace sbk {
namespace tcf {

constexpr int W = 64;
constexpr int NT = 256;                         // two threads per TMEM lane
constexpr int A_SUB = 128 * 128;                // bytes of one A sub-operand: 128 lines x 64 bf16
constexpr int B_SUB = 64 * 128;                 // bytes of one B sub-operand: 64 rows x 64 bf16
constexpr int OFF_A = 0;                        // Re hi | Re lo | Im hi | Im lo
constexpr int OFF_B = 4 * A_SUB;                // Fr hi | Fr lo | Fi hi | Fi lo
constexpr int OFF_MISC = OFF_B + 4 * B_SUB;     // barrier, TMEM address, reductions, tables
constexpr int MISC_BYTES = 3072;
constexpr int SMEM_BYTES = OFF_MISC + MISC_BYTES + 1024;  // + alignment of the base to 1024
constexpr int TMEM_COLS = 256;
constexpr long long kWaitLimit = 1LL << 22;     // try_wait rounds per MMA completion
constexpr long long kWaitCycles = 4000000000LL; // and at most ~2 s of SM clock cycles

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(su32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// shared-memory matrix descriptor, 128-byte swizzle (tcgen05 format version 1)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// instruction descriptor: D f32, A and B bf16, B K-major, M = 128, N = 64
__host__ __device__ constexpr uint32_t idesc(bool aMN, bool negA)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((negA ? 1u : 0u) << 13) | ((aMN ? 1u : 0u) << 15) |
           ((64u >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t id, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
        "l"(ad), "l"(bd), "r"(id), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}

// Two 32-column loads (the real and imaginary halves of an accumulator row)
// and one wait, in one statement so nothing reads the registers before the wait.
__device__ __forceinline__ void tmem_ld32x2(uint32_t ta, uint32_t tb, float (&va)[32], float (&vb)[32])
{
    uint32_t a[32], b[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%64];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%65];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3]), "=r"(a[4]), "=r"(a[5]), "=r"(a[6]), "=r"(a[7]), "=r"(a[8]), "=r"(a[9]), "=r"(a[10]), "=r"(a[11]), "=r"(a[12]), "=r"(a[13]), "=r"(a[14]), "=r"(a[15]), "=r"(a[16]), "=r"(a[17]), "=r"(a[18]), "=r"(a[19]), "=r"(a[20]), "=r"(a[21]), "=r"(a[22]), "=r"(a[23]), "=r"(a[24]), "=r"(a[25]), "=r"(a[26]), "=r"(a[27]), "=r"(a[28]), "=r"(a[29]), "=r"(a[30]), "=r"(a[31]),
          "=r"(b[0]), "=r"(b[1]), "=r"(b[2]), "=r"(b[3]), "=r"(b[4]), "=r"(b[5]), "=r"(b[6]), "=r"(b[7]), "=r"(b[8]), "=r"(b[9]), "=r"(b[10]), "=r"(b[11]), "=r"(b[12]), "=r"(b[13]), "=r"(b[14]), "=r"(b[15]), "=r"(b[16]), "=r"(b[17]), "=r"(b[18]), "=r"(b[19]), "=r"(b[20]), "=r"(b[21]), "=r"(b[22]), "=r"(b[23]), "=r"(b[24]), "=r"(b[25]), "=r"(b[26]), "=r"(b[27]), "=r"(b[28]), "=r"(b[29]), "=r"(b[30]), "=r"(b[31])
        : "r"(ta), "r"(tb)
        : "memory");
#pragma unroll
    for (int k = 0; k < 32; ++k) {
        va[k] = __uint_as_float(a[k]);
        vb[k] = __uint_as_float(b[k]);
    }
}

// ---------------------------------------------------------------- operand layout
// Both A layouts and B use the 128-byte swizzle: a 1024-byte atom is 8 rows of
// 128 bytes (64 bf16), and 16-byte chunk c of row r sits at chunk c ^ (r & 7).
//   K-major A (F1) and B: row = line (or B column n), 64 K values per row;
//     row r at (r / 8) * 1024 + (r % 8) * 128.
//   MN-major A: row = K index t, 64 line values per row; the two 64-line
//     halves (M atoms) of K rows 8g..8g+7 at g * 2048 + half * 1024.
__device__ __forceinline__ uint32_t row_kmajor(int r) { return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128); }
__device__ __forceinline__ uint32_t row_mnmajor(int t, int half)
{
    return (uint32_t)((t >> 3) * 2048 + half * 1024 + (t & 7) * 128);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b)
{
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}

// hi/lo split of 8 values: hi = bf16(x), lo = bf16(x - hi)
__device__ __forceinline__ void split8(const float (&x)[8], uint4& hi, uint4& lo)
{
    uint32_t h[4], l[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        h[q] = pack_bf16x2(x[2 * q], x[2 * q + 1]);
        const float h0 = __uint_as_float(h[q] << 16), h1 = __uint_as_float(h[q] & 0xffff0000u);
        l[q] = pack_bf16x2(x[2 * q] - h0, x[2 * q + 1] - h1);
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// stores chunk c (values 8c .. 8c+7) of one row of all four A sub-operands
__device__ __forceinline__ void put_chunk(unsigned char* A, uint32_t rowOff, int swz, int c, const float (&re)[8],
                                          const float (&im)[8])
{
    uint4 rh, rl, ih, il;
    split8(re, rh, rl);
    split8(im, ih, il);
    const uint32_t o = rowOff + (uint32_t)(((c ^ swz) & 7) << 4);
    *reinterpret_cast<uint4*>(A + 0 * A_SUB + o) = rh;
    *reinterpret_cast<uint4*>(A + 1 * A_SUB + o) = rl;
    *reinterpret_cast<uint4*>(A + 2 * A_SUB + o) = ih;
    *reinterpret_cast<uint4*>(A + 3 * A_SUB + o) = il;
}

// Issues one forward 64-point DFT pass (48 MMAs) from the A operand into the
// 128 TMEM columns at dcol (Re at dcol, Im at dcol + 64), and commits it to bar.
__device__ __forceinline__ void issue_pass(uint32_t aBase, uint32_t bBase, bool aMN, uint32_t tmem, uint32_t dcol,
                                           uint64_t* bar)
{
    // A sub-operands: 0 Re hi, 1 Re lo, 2 Im hi, 3 Im lo; B: 0 Fr hi, 1 Fr lo, 2 Fi hi, 3 Fi lo
    const uint32_t lboA = aMN ? 1024u : 16u, sboA = aMN ? 2048u : 1024u;
    const uint32_t kstepA = aMN ? 4096u : 32u;
    // (A part, B part, column offset, negate A): Re += Ar Fr - Ai Fi ; Im += Ar Fi + Ai Fr
    const int termA[4] = {0, 2, 0, 2};
    const int termB[4] = {0, 2, 2, 0};
    const uint32_t termD[4] = {0u, 0u, 64u, 64u};
    const bool termNeg[4] = {false, true, false, false};
    bool first[2] = {true, true};
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
#pragma unroll
            for (int s = 0; s < 3; ++s) {  // hi.hi, hi.lo, lo.hi
                const int ap = termA[t] + (s == 2 ? 1 : 0), bp = termB[t] + (s == 1 ? 1 : 0);
                const uint64_t ad = sdesc(aBase + ap * A_SUB + kk * kstepA, lboA, sboA);
                const uint64_t bd = sdesc(bBase + bp * B_SUB + kk * 32u, 16u, 1024u);
                const int di = termD[t] ? 1 : 0;
                mma_bf16(tmem + dcol + termD[t], ad, bd, idesc(aMN, termNeg[t]), first[di] ? 0u : 1u);
                first[di] = false;
            }
        }
    }
    mma_commit(bar);
}

// |c|^2 planes in shared memory: plane q = 2 e1 + e2, 64 x 64 floats, the
// float4 chunk of row m1 swizzled by m1 & 15 (the rows are written by 32
// lanes at once).
__device__ __forceinline__ int pidx(int q, int m1, int m2)
{
    return q * 4096 + m1 * 64 + ((((m2 >> 2) ^ (m1 & 15)) & 15) << 2) + (m2 & 3);
}
// fftshifted surface corrF[y][x] (findCPeak's layout): c[cy][cx] with
// cy = (y + 64) mod 128, cx = (x + 64) mod 128; c[2 m1 + e1][2 m2 + e2]
__device__ __forceinline__ float fmap_tc(const float* P, int y, int x)
{
    const int cy = y < W ? y + W : y - W, cx = x < W ? x + W : x - W;
    return P[pidx(((cy & 1) << 1) | (cx & 1), cy >> 1, cx >> 1)];
}

}  // namespace tcf

using namespace tcf;

// A raw sample (8 bytes of complex float32 or 4 of complex int16, loaded as
// one word) to complex float: byte swap for big-endian files, complex float32
// scaled by 1000 (getPatches), int16 as is.
template <bool F32>
__device__ __forceinline__ float2 tc_decode(typename std::conditional<F32, uint2, uint32_t>::type w, bool msb)
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

template <bool F32>
__global__ void __launch_bounds__(tcf::NT, 2) strack_cmplx_tc_kernel(CmplxArgs a)
{
    extern __shared__ unsigned char smem_dyn[];
    // 1024-byte aligned base (the swizzle atoms must be)
    unsigned char* sm = smem_dyn + ((1024u - (su32(smem_dyn) & 1023u)) & 1023u);
    unsigned char* A = sm + OFF_A;
    unsigned char* Bm = sm + OFF_B;
    unsigned char* misc = sm + OFF_MISC;
    uint64_t* bar = reinterpret_cast<uint64_t*>(misc);                  // 8 B
    uint32_t* tslot = reinterpret_cast<uint32_t*>(misc + 8);            // 4 B
    int* azs = reinterpret_cast<int*>(misc + 12);                       // 4 B
    double* red = reinterpret_cast<double*>(misc + 16);                 // (8 + 1) x 19 doubles = 1368 B
    float2* tau = reinterpret_cast<float2*>(misc + 1408);               // 64 x 8 B
    unsigned* iscr = reinterpret_cast<unsigned*>(misc + 1920);          // 16 words
    uint32_t* lowm = reinterpret_cast<uint32_t*>(misc + 2048);          // 128 lines x 2 halves
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // two threads per TMEM lane: warps 0-3 and 4-7 cover lanes 0-127 twice;
    // thread (L, h) owns line L and the half h of its 64 values
    const int L = ((warp & 3) << 5) | lane, h = warp >> 2;
    const int w = L >> 6, k = L & 63;
    const uint32_t aBase = su32(A), bBase = su32(Bm);

    // ---- DFT matrix F[t][n] = exp(-2 pi i t n / 64) as hi/lo bf16, K-major rows n
    for (int e = tid; e < 64 * 8; e += NT) {
        const int n = e >> 3, c = e & 7;
        float re[8], im[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int t = 8 * c + q;
            double s, co;
            sincospi(-2.0 * (double)((t * n) & 63) / 64.0, &s, &co);
            re[q] = (float)co;
            im[q] = (float)s;
        }
        uint4 rh, rl, ih, il;
        split8(re, rh, rl);
        split8(im, ih, il);
        const uint32_t o = row_kmajor(n) + (uint32_t)(((c ^ n) & 7) << 4);
        *reinterpret_cast<uint4*>(Bm + 0 * B_SUB + o) = rh;
        *reinterpret_cast<uint4*>(Bm + 1 * B_SUB + o) = rl;
        *reinterpret_cast<uint4*>(Bm + 2 * B_SUB + o) = ih;
        *reinterpret_cast<uint4*>(Bm + 3 * B_SUB + o) = il;
    }
    for (int e = tid; e < W; e += NT) tau[e] = a.tau[e];
    if (tid == 0) {
        mbar_init(bar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_async_smem();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tslot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t tlane = tmem + ((uint32_t)((warp & 3) * 32) << 16);  // this warp's lane quarter
    uint32_t phase = 0;
    bool failed = false;

    // one completed MMA pass: every thread waits (bounded) for the barrier
    // phase; the outcome is made block-uniform
    auto wait_pass = [&]() -> bool {
        long long n = 0;
        bool ok = true;
        const long long t0 = clock64();
        while (!mbar_try(bar, phase & 1u)) {
            if (++n > kWaitLimit || clock64() - t0 > kWaitCycles) {
                ok = false;
                break;
            }
        }
        phase++;
        tc_fence_after();
        return !__syncthreads_or(!ok);
    };
    // all threads' A writes -> async proxy -> one thread issues the pass
    auto run_pass = [&](bool aMN, uint32_t dcol) {
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            issue_pass(aBase, bBase, aMN, tmem, dcol, bar);
        }
    };
    // the half h of a 128-column accumulator (Re at dcol, Im at dcol + 64) into
    // chunks 4h .. 4h+3 of an A row
    auto drain_half = [&](uint32_t dcol, uint32_t rowOff, int swz) {
        float vr[32], vi[32];
        tmem_ld32x2(tlane + dcol + 32 * h, tlane + dcol + 64 + 32 * h, vr, vi);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float re[8], im[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                re[q] = vr[8 * c + q];
                im[q] = vi[8 * c + q];
            }
            put_chunk(A, rowOff, swz, 4 * h + c, re, im);
        }
    };

    const float thr = F32 ? 1e-15f : 1e-9f;
    const float thrAll = thr * W * W;

    // list entries two patches ahead, plans one patch ahead (no dependent
    // list -> plan -> window load chain at the start of a patch)
    const int G = gridDim.x;
    int pNext = a.list[blockIdx.x];
    int pAfter = (int)blockIdx.x + G < a.nList ? a.list[blockIdx.x + G] : 0;
    PointPlan plNext = a.plan[pNext];
    for (int it = blockIdx.x; it < a.nList && !failed; it += G) {
        const int p = pNext;
        const PointPlan pl = plNext;
        if (it + G < a.nList) {
            pNext = pAfter;
            plNext = a.plan[pAfter];
            if (it + 2 * G < a.nList) pAfter = a.list[it + 2 * G];
        }
        // ------------------------------------------------ getPatches: column k of window w, rows [32 h, 32 h + 32)
        // power / mean sums in float per thread, totals in double; lag-1 sums
        // along azimuth in double (mean-corrected after the reduction)
        const void* img = w ? a.img2 : a.img1;
        const int nr = w ? a.nr2 : a.nr1;
        const int r0 = (w ? pl.a2 : pl.a1), c0 = (w ? pl.r2 : pl.r1) + k;
        // raw loads sixteen rows at a time (the taper and the byte order are
        // predicates), decoded where they are used
        using Raw = typename std::conditional<F32, uint2, uint32_t>::type;
        const Raw* base = reinterpret_cast<const Raw*>(img);
        const bool msb = a.byteOrder == SB_MSB;
        const bool han = w && a.hanning;
        auto raw_at = [&](int i) { return __ldg(base + ((size_t)(r0 + i) * nr + c0)); };
        auto han_at = [&](int i) { return han ? __ldg(a.hanning + i * W + k) : 1.f; };
        auto decode = [&](Raw wv, float hv) {
            float2 v = tc_decode<F32>(wv, msb);
            if (han) {
                v.x *= hv;
                v.y *= hv;
            }
            return v;
        };
        float fp = 0.f, fr = 0.f, fi = 0.f;
        uint32_t low = 0;  // rows of this half whose power is below the threshold
        double lr = 0, li = 0, nr_ = 0, ni_ = 0, pr_ = 0, pi_ = 0;  // sum z[i] conj z[i-1], sum z[1..], sum z[..62]
        float2 prev = make_float2(0.f, 0.f);
        if (h) prev = decode(raw_at(31), han_at(31));  // the pair (31, 32) belongs to half 1
        const uint32_t rowOff = row_kmajor(L);
#pragma unroll 1
        for (int g2 = 0; g2 < 4; g2 += 2) {
            Raw wr[16];
            float hvv[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                wr[q] = raw_at(32 * h + 8 * g2 + q);
                hvv[q] = han_at(32 * h + 8 * g2 + q);
            }
#pragma unroll
        for (int gg = 0; gg < 2; ++gg) {  // 8 rows per chunk of the K-major F1 operand
            const int g = g2 + gg;
            float re[8], im[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int i = 32 * h + 8 * g + q;
                const float2 v = decode(wr[8 * gg + q], hvv[8 * gg + q]);
                const float pw = __fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y));
                low |= (uint32_t)(pw < thr) << (8 * g + q);
                fp += pw;
                fr += v.x;
                fi += v.y;
                if (i > 0) {
                    lr += (double)v.x * prev.x + (double)v.y * prev.y;
                    li += (double)v.y * prev.x - (double)v.x * prev.y;
                    nr_ += v.x;
                    ni_ += v.y;
                }
                if (i < W - 1) {
                    pr_ += v.x;
                    pi_ += v.y;
                }
                prev = v;
                re[q] = v.x;
                im[q] = v.y;
            }
            put_chunk(A, rowOff, L & 7, 4 * h + g, re, im);
        }
        }
        // getPatches counts the positions where either window's power is low
        lowm[2 * L + h] = low;
        __syncthreads();
        const int nLow = w ? 0 : __popc(lowm[2 * L + h] | lowm[2 * (L + 64) + h]);
        // block totals: [0..1] power, [2..5] sums (re, im) of windows 1, 2,
        // [6] low positions, [7..18] lag, next, prev sums of windows 1, 2
        double s[19];
#pragma unroll
        for (int q = 0; q < 2; ++q) {  // compile-time indices: the array stays in registers
            const bool mine = (w == q);
            s[q] = mine ? (double)fp : 0.0;
            s[2 + 2 * q] = mine ? (double)fr : 0.0;
            s[3 + 2 * q] = mine ? (double)fi : 0.0;
            s[7 + 6 * q] = mine ? lr : 0.0;
            s[8 + 6 * q] = mine ? li : 0.0;
            s[9 + 6 * q] = mine ? nr_ : 0.0;
            s[10 + 6 * q] = mine ? ni_ : 0.0;
            s[11 + 6 * q] = mine ? pr_ : 0.0;
            s[12 + 6 * q] = mine ? pi_ : 0.0;
        }
        s[6] = (double)nLow;
        block_allsum<19, NT>(s, red);
        const bool haveData = !(s[6] > 20.0) && !(s[0] < thrAll || s[1] < thrAll);
        if (!haveData) {
            if (tid == 0) {
                a.rec[p].flags |= RF_DONE_C;
                a.rec[p].azset = -1;
                a.fit[it].point = p;
                a.fit[it].gate = 0;
                a.peak[it].point = p;
                a.peak[it].iC = PJ_NODATA;
            }
            __syncthreads();
            continue;  // uniform
        }
        const double nn = (double)(W * W), npair = (double)((W - 1) * W);
        const double p1 = s[0] / nn, p2 = s[1] / nn;
        if (tid == 0) {
            // sum (a[i+1] - m) conj(a[i] - m) = L - conj(m) N - m conj(P) + npair |m|^2
            double d[4];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const double mr = s[2 + 2 * q] / nn, mi = s[3 + 2 * q] / nn;
                const double Lr = s[7 + 6 * q], Li = s[8 + 6 * q], Nr = s[9 + 6 * q], Ni = s[10 + 6 * q];
                const double Pr = s[11 + 6 * q], Pi = s[12 + 6 * q];
                // conj(m) N = (mr Nr + mi Ni) + i (mr Ni - mi Nr); m conj(P) = (mr Pr + mi Pi) + i (mi Pr - mr Pi)
                d[2 * q] = Lr - (mr * Nr + mi * Ni) - (mr * Pr + mi * Pi) + npair * (mr * mr + mi * mi);
                d[2 * q + 1] = Li - (mr * Ni - mi * Nr) - (mi * Pr - mr * Pi);
            }
            *azs = dop_shift(d[0], d[1], d[2], d[3], W, W);
        }
        // ------------------------------------------------ F1: azimuth transforms of both windows
        run_pass(false, 0);
        if (!wait_pass()) { failed = true; break; }
        // ------------------------------------------------ F2: range transforms (D1 -> MN-major A, K row k of atom w)
        drain_half(0, row_mnmajor(k, w), k & 7);
        run_pass(true, 128);
        if (!wait_pass()) { failed = true; break; }
        // ------------------------------------------------ cross spectrum, conjugated: conj(Z1) Z2
        // thread (w, n1, h) holds Z_w[n1][32 h .. 32 h + 31]; it computes the
        // 16 columns 32 h + 16 w + j and takes the other window's 16 values
        // from its partner (line L ^ 64, same half) through shared memory
        float2 S[16];
        {
            float vr[32], vi[32];
            tmem_ld32x2(tlane + 128 + 32 * h, tlane + 192 + 32 * h, vr, vi);
            float2* xb = reinterpret_cast<float2*>(A);  // 16 x 256 float2: [j][thread]
            tc_fence_before();
            __syncthreads();  // F2's operand reads are complete (waited): the area is free
            // compile-time register indices, selected by the window (no local array)
#pragma unroll
            for (int j = 0; j < 16; ++j)  // the columns the partner computes
                xb[j * NT + tid] = w ? make_float2(vr[j], vi[j]) : make_float2(vr[16 + j], vi[16 + j]);
            __syncthreads();
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const float2 o = xb[j * NT + (tid ^ 64)];
                const float2 own = w ? make_float2(vr[16 + j], vi[16 + j]) : make_float2(vr[j], vi[j]);
                const float2 z1 = w ? o : own;
                const float2 z2 = w ? own : o;
                S[j] = make_float2(z1.x * z2.x + z1.y * z2.y, z1.x * z2.y - z1.y * z2.x);  // conj(z1) z2
            }
            tc_fence_before();
            __syncthreads();  // everyone has read xb before the area becomes the A operand
        }
        const int az = *azs;
        const int krow = (k - az) & 63;  // K row k1' = n1 - azShift (mod 64) holds S row n1 = k
        const int k2base = 32 * h + 16 * w;
        // ------------------------------------------------ I1_e1: inverse along k1 (two parities)
#pragma unroll 1
        for (int e1 = 0; e1 < 2; ++e1) {
            // conj(tau_e1[k1']) on the row; conj(tau_e2[k2]) on M atom e2
            const float2 tr = e1 ? make_float2(tau[krow].x, -tau[krow].y) : make_float2(1.f, 0.f);
#pragma unroll
            for (int e2 = 0; e2 < 2; ++e2) {
                const uint32_t ro = row_mnmajor(krow, e2);
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    float re[8], im[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const int j = 8 * c + q;
                        float2 v = S[j];
                        v = make_float2(v.x * tr.x - v.y * tr.y, v.x * tr.y + v.y * tr.x);
                        if (e2) {
                            const float2 t2 = make_float2(tau[k2base + j].x, -tau[k2base + j].y);
                            v = make_float2(v.x * t2.x - v.y * t2.y, v.x * t2.y + v.y * t2.x);
                        }
                        re[q] = v.x;
                        im[q] = v.y;
                    }
                    put_chunk(A, ro, krow & 7, (k2base >> 3) + c, re, im);
                }
            }
            run_pass(true, e1 ? 128 : 0);
            if (!wait_pass()) { failed = true; break; }
        }
        if (failed) break;
        // ------------------------------------------------ I2_e1: inverse along k2
        // thread (e2, k2, h) holds D3_e1[(e2,k2)][m1] for m1 in half h: K row k2 of M atom e2
#pragma unroll 1
        for (int e1 = 0; e1 < 2; ++e1) {
            const uint32_t dcol = e1 ? 128u : 0u;
            drain_half(dcol, row_mnmajor(k, w), k & 7);
            run_pass(true, dcol);
            if (!wait_pass()) { failed = true; break; }
        }
        if (failed) break;
        // ------------------------------------------------ |c|^2 planes (thread (e2, m1, h): row m1, half h of (e1, e2))
        float* P = reinterpret_cast<float*>(A);
        float pmax = 0.f;
        {
            const int e2 = w, m1 = k;
#pragma unroll 1
            for (int e1 = 0; e1 < 2; ++e1) {
                const int q = 2 * e1 + e2;
                float vr[32], vi[32];
                tmem_ld32x2(tlane + (e1 ? 128u : 0u) + 32 * h, tlane + (e1 ? 128u : 0u) + 64 + 32 * h, vr, vi);
#pragma unroll
                for (int c4 = 0; c4 < 8; ++c4) {
                    float4 o;
                    o.x = vr[4 * c4 + 0] * vr[4 * c4 + 0] + vi[4 * c4 + 0] * vi[4 * c4 + 0];
                    o.y = vr[4 * c4 + 1] * vr[4 * c4 + 1] + vi[4 * c4 + 1] * vi[4 * c4 + 1];
                    o.z = vr[4 * c4 + 2] * vr[4 * c4 + 2] + vi[4 * c4 + 2] * vi[4 * c4 + 2];
                    o.w = vr[4 * c4 + 3] * vr[4 * c4 + 3] + vi[4 * c4 + 3] * vi[4 * c4 + 3];
                    pmax = fmaxf(pmax, fmaxf(fmaxf(o.x, o.y), fmaxf(o.z, o.w)));
                    *reinterpret_cast<float4*>(P + pidx(q, m1, 32 * h + 4 * c4)) = o;
                }
            }
        }
        // ------------------------------------------------ findCPeak (exact tie order, as strack_cmplx.cu)
        // the block maximum of |c|^2, then every value whose sqrtf equals its
        // sqrtf is ranked in findCPeak's scan order; each thread rescans the
        // 64 values it wrote
        int iMax = 0, jMax = 0;
        {
            unsigned u = __reduce_max_sync(0xffffffffu, __float_as_uint(pmax));
            if (lane == 0) iscr[warp] = u;
            tc_fence_before();
            __syncthreads();
            u = iscr[0];
#pragma unroll
            for (int q = 1; q < NT / 32; ++q) u = max(u, iscr[q]);
            const float pm = __uint_as_float(u);
            if (pm > 0.f) {  // uniform
                const float smx = sqrtf(pm);
                const float lo = pm * (1.0f - 1.0f / 1048576.0f);
                unsigned best = 0xffffffffu;
                const int e2 = w, m1 = k;
                // only a thread whose own maximum reaches lo holds candidates
#pragma unroll 1
                for (int e1 = 0; e1 < (pmax >= lo ? 2 : 0); ++e1) {
                    const int q = 2 * e1 + e2;
#pragma unroll
                    for (int c4 = 0; c4 < 8; ++c4) {
                        const int m2b = 32 * h + 4 * c4;
                        const float4 v4 = *reinterpret_cast<const float4*>(P + pidx(q, m1, m2b));
                        const float vv[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
                        for (int t = 0; t < 4; ++t) {
                            if (vv[t] >= lo && sqrtf(vv[t]) == smx) {
                                const int cy = 2 * m1 + e1, cx = 2 * (m2b + t) + e2;
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
                for (int q = 1; q < NT / 32; ++q) best = min(best, iscr[NT / 32 + q]);
                const int qq = best & 3, ij = best >> 2;
                iMax = ij / W + ((qq == 1 || qq == 2) ? W : 0);
                jMax = ij % W + ((qq == 1 || qq == 3) ? W : 0);
            }
        }
        const bool rejected = (iMax < (NFAST / 2) || iMax > (2 * W - NFAST / 2) || jMax < (NFAST / 2) ||
                               jMax > (2 * W - NFAST / 2));
        if (rejected) {
            iMax = -1000;
            jMax = -1000;
        }
        // ------------------------------------------------ hand the peak to the peak kernel
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
                if (y >= 0 && y < 2 * W && x >= 0 && x < 2 * W) (&pj->blk[0][0])[e] = fmap_tc(P, y, x);
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
            r->azset = az;
            r->flags |= RF_DONE_C | RF_HD_C;
        }
        // debug dump of the first list entry's surface (tests of the transform passes)
        if (a.tcDebug && it == 0) {
            for (int e = tid; e < 4 * 4096; e += NT) {
                const int q = e >> 12, m1 = (e >> 6) & 63, m2 = e & 63;
                a.tcDebug[e] = P[pidx(q, m1, m2)];
            }
        }
        tc_fence_before();
        __syncthreads();  // the planes are read before the next patch's F1 operand overwrites them
    }
    if (failed && tid == 0 && a.tcErr) atomicExch(a.tcErr, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

template <bool F32>
static cudaError_t launch_tc_t(const CmplxArgs& a, int nCta, cudaStream_t st)
{
    cudaError_t e = cudaFuncSetAttribute(strack_cmplx_tc_kernel<F32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         SMEM_BYTES);
    if (e != cudaSuccess) return e;
    // the largest shared-memory carveout, so that two CTAs fit on an SM
    e = cudaFuncSetAttribute(strack_cmplx_tc_kernel<F32>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    strack_cmplx_tc_kernel<F32><<<nCta, NT, SMEM_BYTES, st>>>(a);
    return cudaGetLastError();
}

bool cmplx_tc_supported(int W_) { return W_ == tcf::W; }

int cmplx_tc_threads() { return NT; }

// Resident CTAs per SM from the SM's register file, shared memory and thread
// slots and the kernel's attributes.  (On the B200 the runtime's occupancy
// calculator reports one CTA for this kernel where the launch statistics show
// two resident; the resources are counted here instead.)
int cmplx_tc_blocks_per_sm()
{
    int dev = 0;
    cudaDeviceProp pr;
    cudaFuncAttributes fa;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&pr, dev) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, strack_cmplx_tc_kernel<true>) != cudaSuccess)
        return 0;
    const int regsPerWarp = ((fa.numRegs * 32 + 255) / 256) * 256;  // allocation unit of 256 registers per warp
    const int byRegs = pr.regsPerMultiprocessor / (regsPerWarp * (NT / 32));
    const size_t perCta = (size_t)SMEM_BYTES + fa.sharedSizeBytes + pr.reservedSharedMemPerBlock;
    const int bySmem = (int)(pr.sharedMemPerMultiprocessor / perCta);
    const int byThreads = pr.maxThreadsPerMultiProcessor / NT;
    int nb = byRegs < bySmem ? byRegs : bySmem;
    nb = nb < byThreads ? nb : byThreads;
    // two 256-column TMEM allocations fill an SM's 512 columns: never more
    return nb > 2 ? 2 : nb;
}

cudaError_t launch_strack_cmplx_tc(const CmplxArgs& a, int nCta, cudaStream_t st)
{
    return a.sampleType == SB_CFLOAT32 ? launch_tc_t<true>(a, nCta, st) : launch_tc_t<false>(a, nCta, st);
}

}  // namespace sbk
