// fft_engine.cuh -- batched complex DFTs in shared memory for sm_100a.
//
// Conventions match FFTW 2 as used by the reference (fftwnd_one,
// Strack/speckleTrack.c:1507-1550): unnormalised, forward = exp(-2 pi i jk/N)
// (DIR = -1), backward = exp(+2 pi i jk/N) (DIR = +1).
//
// A length-N line (N = N1 * N2) is transformed in place in two steps
// (the "four-step" factorisation, x index n = N2*n1 + n2, X index
// k = k1 + N1*k2):
//   step 1: for every (line, n2): radix-N1 DFT over n1 in registers, times the
//           twiddle W_N^{n2 k1}, stored back to the same slots;
//   step 2: for every (line, k1): radix-N2 DFT over the N2 contiguous slots,
//           held in registers until every thread has loaded, then stored to
//           natural order k1 + N1*k2.
// Threads are mapped line-fastest, so with an odd row stride (N+1 float2) or
// unit line stride (column passes) every access pattern is bank-conflict free.
//
// Register DFTs of composite size R are built at compile time by splitting off
// the smallest prime factor; prime factors use the direct sum.  Twiddles come
// from a table W_TN^e = exp(-2 pi i e/TN), e < TN, read with compile-time
// indices (uniform across the warp, so broadcast) for the inter-step twiddles,
// while the twiddles inside the register DFTs are compile-time constants;
// factors of +-1, +-i are applied without a multiply.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sbfft {

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cconjmul(float2 a, float2 b)  // a * conj(b)
{
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

constexpr int smallest_factor(int n)
{
    for (int p = 2; p * p <= n; ++p)
        if (n % p == 0) return p;
    return n;
}

// ---------------------------------------------------------------- compile-time twiddles
// cos and sin of 2 pi e / n for integers, evaluated by the compiler: octant
// reduction with exact integer arithmetic, then the Taylor series of sin and
// cos on [0, pi/4] in double (14 terms: truncation below 1e-20), rounded once
// to float where used.  Compile-time twiddles become immediate operands.
struct CxPair {
    double c, s;
};
constexpr double kQuarterPi = 0.78539816339744830961566084581987572;
__host__ __device__ constexpr double cx_sin(double x)
{
    double term = x, sum = x;
    for (int k = 1; k < 14; ++k) {
        term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double cx_cos(double x)
{
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 14; ++k) {
        term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr CxPair cx_cossin(int e, int n)  // (cos, sin)(2 pi e / n)
{
    const long long r = ((e % n) + n) % n;
    const long long m = 8 * r;                  // theta / (pi/4) = m / n
    const int oct = (int)(m / n);
    const long long fnum = m - (long long)oct * n;  // phi = (pi/4) fnum / n
    const double phi = kQuarterPi * (double)fnum / (double)n;
    const double psi = kQuarterPi * (double)(n - fnum) / (double)n;  // pi/4 - phi
    const double Sp = cx_sin(phi), Cp = cx_cos(phi), Sq = cx_sin(psi), Cq = cx_cos(psi);
    switch (oct) {
    case 0: return {Cp, Sp};
    case 1: return {Sq, Cq};
    case 2: return {-Sp, Cp};
    case 3: return {-Cq, Sq};
    case 4: return {-Cp, -Sp};
    case 5: return {-Sq, -Cq};
    case 6: return {Sp, -Cp};
    default: return {Cq, -Sq};
    }
}

// v * W_TN^{E} for the direction DIR (W = exp(DIR * 2 pi i / TN)); E reduced mod TN.
template <int E, int TN, int DIR>
__device__ __forceinline__ float2 twmul(float2 v, const float2* __restrict__ tw)
{
    constexpr int e = ((E % TN) + TN) % TN;
    if constexpr (e == 0) {
        return v;
    } else if constexpr (4 * e == 2 * TN) {
        return make_float2(-v.x, -v.y);
    } else if constexpr (4 * e == TN) {
        // exp(DIR * i pi/2) = DIR * i
        return DIR > 0 ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
    } else if constexpr (4 * e == 3 * TN) {
        return DIR > 0 ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
    } else {
        constexpr CxPair w = cx_cossin(e, TN);
        constexpr float wr = (float)w.c;
        constexpr float wi = (float)(DIR > 0 ? w.s : -w.s);
        return cmul(v, make_float2(wr, wi));
    }
}

// Runtime-index twiddle multiply (inter-step twiddles).
template <int DIR>
__device__ __forceinline__ float2 twmul_rt(float2 v, const float2* __restrict__ tw, int e)
{
    float2 w = tw[e];
    if (DIR > 0) w.y = -w.y;
    return cmul(v, w);
}

// ---------------------------------------------------------------- register DFT
template <int R, int DIR, int TN>
struct RegDFT {
    static_assert(TN % R == 0, "twiddle table size must be a multiple of R");
    static constexpr int P = (R % 4 == 0 && R > 4) ? 4 : smallest_factor(R);  // radix 4 first
    static constexpr int M = R / P;

    template <int Q, int K>
    __device__ __forceinline__ static float2 sub_tw(float2 v, const float2* tw)
    {
        return twmul<Q * K * (TN / R), TN, DIR>(v, tw);
    }

    // direct P-point DFT of t[] into out[r] (prime P)
    template <int Pp>
    __device__ __forceinline__ static void small_dft(float2 (&t)[Pp], float2 (&o)[Pp], const float2* tw)
    {
        if constexpr (Pp == 2) {
            o[0] = cadd(t[0], t[1]);
            o[1] = csub(t[0], t[1]);
        } else if constexpr (Pp == 4) {
            float2 a0 = cadd(t[0], t[2]), a1 = csub(t[0], t[2]);
            float2 b0 = cadd(t[1], t[3]), b1 = csub(t[1], t[3]);
            float2 jb1 = DIR > 0 ? make_float2(-b1.y, b1.x) : make_float2(b1.y, -b1.x);
            o[0] = cadd(a0, b0);
            o[2] = csub(a0, b0);
            o[1] = cadd(a1, jb1);
            o[3] = csub(a1, jb1);
        } else {
#pragma unroll
            for (int r = 0; r < Pp; ++r) o[r] = t[0];
            small_dft_acc<Pp, 1>(t, o, tw);
        }
    }
    template <int Pp, int Q>
    __device__ __forceinline__ static void small_dft_acc(float2 (&t)[Pp], float2 (&o)[Pp], const float2* tw)
    {
        if constexpr (Q < Pp) {
            small_dft_acc_r<Pp, Q, 0>(t, o, tw);
            small_dft_acc<Pp, Q + 1>(t, o, tw);
        }
    }
    template <int Pp, int Q, int Rr>
    __device__ __forceinline__ static void small_dft_acc_r(float2 (&t)[Pp], float2 (&o)[Pp], const float2* tw)
    {
        if constexpr (Rr < Pp) {
            o[Rr] = cadd(o[Rr], twmul<((Q * Rr) % Pp) * (TN / Pp), TN, DIR>(t[Q], tw));
            small_dft_acc_r<Pp, Q, Rr + 1>(t, o, tw);
        }
    }

    template <int K>
    __device__ __forceinline__ static void combine(float2 (&sub)[P][M], float2 (&v)[R], const float2* tw)
    {
        if constexpr (K < M) {
            float2 t[P], o[P];
            t[0] = sub[0][K];
            combine_tw<K, 1>(sub, t, tw);
            small_dft<P>(t, o, tw);
#pragma unroll
            for (int r = 0; r < P; ++r) v[K + M * r] = o[r];
            combine<K + 1>(sub, v, tw);
        }
    }
    template <int K, int Q>
    __device__ __forceinline__ static void combine_tw(float2 (&sub)[P][M], float2 (&t)[P], const float2* tw)
    {
        if constexpr (Q < P) {
            t[Q] = sub_tw<Q, K>(sub[Q][K], tw);
            combine_tw<K, Q + 1>(sub, t, tw);
        }
    }

    __device__ __forceinline__ static void run(float2 (&v)[R], const float2* __restrict__ tw)
    {
        if constexpr (R == 1) {
            return;
        } else if constexpr (R == 4) {
            float2 o[4];
            small_dft<4>(v, o, tw);
#pragma unroll
            for (int r = 0; r < 4; ++r) v[r] = o[r];
        } else if constexpr (P == R) {
            float2 o[R];
            small_dft<R>(v, o, tw);
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = o[r];
        } else {
            float2 sub[P][M];
#pragma unroll
            for (int q = 0; q < P; ++q)
#pragma unroll
                for (int t = 0; t < M; ++t) sub[q][t] = v[q + P * t];
#pragma unroll
            for (int q = 0; q < P; ++q) RegDFT<M, DIR, TN>::run(sub[q], tw);
            combine<0>(sub, v, tw);
        }
    }
};

// ---------------------------------------------------------------- line FFTs
// Step 2 of the line transforms (see fft_lines_io): radix-N2 DFTs over the N2
// contiguous slots of every (line, k1), all loaded before the first store;
// outputs go to dst(l, k1, k2, value).  Ends with a barrier.
template <int N1, int N2, int DIR, int NL, int NLI, int NT, int LS, int ES, int IS, typename Dst>
__device__ __forceinline__ void fft_step2(float2* base, Dst dst, const float2* __restrict__ tw)
{
    constexpr int N = N1 * N2;
    constexpr int T2 = NL * N1;
    constexpr int R2 = (T2 + NT - 1) / NT;
    const int tid = threadIdx.x;
    float2 v2[R2][N2];
#pragma unroll
    for (int r = 0; r < R2; ++r) {
        const int t = tid + r * NT;
        if (T2 % NT == 0 || t < T2) {
            const int l = t % NL, k1 = t / NL;
            const float2* p = base + (l % NLI) * LS + (l / NLI) * IS + (N2 * k1) * ES;
#pragma unroll
            for (int n2 = 0; n2 < N2; ++n2) v2[r][n2] = p[n2 * ES];
            RegDFT<N2, DIR, N>::run(v2[r], tw);
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R2; ++r) {
        const int t = tid + r * NT;
        if (T2 % NT == 0 || t < T2) {
            const int l = t % NL, k1 = t / NL;
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2) dst(l, k1, k2, v2[r][k2]);
        }
    }
    __syncthreads();
}

// Lines are addressed as base + (l % NLI) * LS + (l / NLI) * IS (NLI lines per
// image, several images side by side).  Element k of a line is at k * ES.
// All strides are compile-time constants, so addresses fold to immediates.
//
// Step 1 takes its inputs from `src(l, k)` and step 2 hands its outputs to
// `dst(l, k1, k2, value)` (output index k = k1 + N1 * k2, k2 a compile-time
// constant after unrolling); `base` holds the intermediate.  With the identity
// functors the transform is in place.  src may gather from another buffer or
// apply an element-wise map (in place is then still safe: step 1 of a thread
// writes exactly the slots it read).  When src reads slots of `base` that other
// threads write in step 1 (a permuting gather within the same buffer), set
// SYNC1: every input is loaded before the first store.  dst is called after a
// barrier that follows the last read of `base`, so it may overwrite `base`.
template <int N1, int N2, int DIR, int NL, int NLI, int NT, int LS, int ES, int IS, bool SYNC1, typename Src,
          typename Dst>
__device__ __forceinline__ void fft_lines_io(float2* base, Src src, Dst dst, const float2* __restrict__ tw)
{
    constexpr int N = N1 * N2;
    constexpr int T1 = NL * N2;
    constexpr int R1 = (T1 + NT - 1) / NT;
    const int tid = threadIdx.x;
    float2 v[R1][N1];
    auto step1 = [&](int r) {
        const int t = tid + r * NT;
        const int l = t % NL, n2 = t / NL;
        float2* p = base + (l % NLI) * LS + (l / NLI) * IS + n2 * ES;
        RegDFT<N1, DIR, N>::run(v[r], tw);
        // k1 * n2 < N1 * N2 = N: the twiddle index needs no reduction
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1) v[r][k1] = twmul_rt<DIR>(v[r][k1], tw, k1 * n2);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) p[(N2 * k1) * ES] = v[r][k1];
    };
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        const int t = tid + r * NT;
        if (T1 % NT == 0 || t < T1) {
            const int l = t % NL, n2 = t / NL;
#pragma unroll
            for (int n1 = 0; n1 < N1; ++n1) v[r][n1] = src(l, N2 * n1 + n2);
            if constexpr (!SYNC1) step1(r);
        }
    }
    if constexpr (SYNC1) {
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int t = tid + r * NT;
            if (T1 % NT == 0 || t < T1) step1(r);
        }
    }
    __syncthreads();
    fft_step2<N1, N2, DIR, NL, NLI, NT, LS, ES, IS>(base, dst, tw);
}

// In-place transform of the lines (identity src/dst).
template <int N1, int N2, int DIR, int NL, int NLI, int NT, int LS, int ES, int IS>
__device__ __forceinline__ void fft_lines(float2* base, const float2* __restrict__ tw)
{
    auto at = [base](int l, int k) -> float2* { return base + (l % NLI) * LS + (l / NLI) * IS + k * ES; };
    auto src = [at](int l, int k) { return *at(l, k); };
    auto dst = [at](int l, int k1, int k2, float2 z) { *at(l, k1 + N1 * k2) = z; };
    fft_lines_io<N1, N2, DIR, NL, NLI, NT, LS, ES, IS, false>(base, src, dst, tw);
}

// Two transforms of the same NL input lines in one pass: with u = src(l, k),
// the lines at base get DFT(u) and the lines at base + IS get
// DFT(u * mul(l, k)).  Each input is read once; step 2 then runs over all
// 2 NL lines (dst sees l in [0, 2 NL): l / NL selects the transform).
// SYNC1 as in fft_lines_io.
template <int N1, int N2, int DIR, int NL, int NT, int LS, int ES, int IS, bool SYNC1, typename Src, typename Mul,
          typename Dst>
__device__ __forceinline__ void fft_lines_dual(float2* base, Src src, Mul mul, Dst dst,
                                               const float2* __restrict__ tw)
{
    constexpr int N = N1 * N2;
    constexpr int T1 = NL * N2;
    constexpr int R1 = (T1 + NT - 1) / NT;
    const int tid = threadIdx.x;
    float2 va[R1][N1], vb[R1][N1];
    auto step1 = [&](int r) {
        const int t = tid + r * NT;
        const int l = t % NL, n2 = t / NL;
        RegDFT<N1, DIR, N>::run(va[r], tw);
        RegDFT<N1, DIR, N>::run(vb[r], tw);
        float2* pa = base + l * LS + n2 * ES;
        float2* pb = pa + IS;
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) {
            if (k1 > 0) {
                float2 w = tw[k1 * n2];
                if (DIR > 0) w.y = -w.y;
                va[r][k1] = cmul(va[r][k1], w);
                vb[r][k1] = cmul(vb[r][k1], w);
            }
            pa[(N2 * k1) * ES] = va[r][k1];
            pb[(N2 * k1) * ES] = vb[r][k1];
        }
    };
#pragma unroll
    for (int r = 0; r < R1; ++r) {
        const int t = tid + r * NT;
        if (T1 % NT == 0 || t < T1) {
            const int l = t % NL, n2 = t / NL;
#pragma unroll
            for (int n1 = 0; n1 < N1; ++n1) {
                const int k = N2 * n1 + n2;
                const float2 u = src(l, k);
                va[r][n1] = u;
                vb[r][n1] = cmul(u, mul(l, k));
            }
            if constexpr (!SYNC1) step1(r);
        }
    }
    if constexpr (SYNC1) {
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int t = tid + r * NT;
            if (T1 % NT == 0 || t < T1) step1(r);
        }
    }
    __syncthreads();
    fft_step2<N1, N2, DIR, 2 * NL, NL, NT, LS, ES, IS>(base, dst, tw);
}

// Factorisation used for each supported transform length.
template <int N>
struct Split;
template <> struct Split<8>   { static constexpr int N1 = 2,  N2 = 4;  };
template <> struct Split<16>  { static constexpr int N1 = 4,  N2 = 4;  };
template <> struct Split<24>  { static constexpr int N1 = 3,  N2 = 8;  };
template <> struct Split<32>  { static constexpr int N1 = 4,  N2 = 8;  };
template <> struct Split<48>  { static constexpr int N1 = 6,  N2 = 8;  };
template <> struct Split<64>  { static constexpr int N1 = 8,  N2 = 8;  };
template <> struct Split<96>  { static constexpr int N1 = 6,  N2 = 16; };
template <> struct Split<128> { static constexpr int N1 = 8,  N2 = 16; };
template <> struct Split<192> { static constexpr int N1 = 12, N2 = 16; };
template <> struct Split<224> { static constexpr int N1 = 14, N2 = 16; };
template <> struct Split<256> { static constexpr int N1 = 16, N2 = 16; };
template <> struct Split<384> { static constexpr int N1 = 24, N2 = 16; };
template <> struct Split<448> { static constexpr int N1 = 28, N2 = 16; };
template <> struct Split<512> { static constexpr int N1 = 32, N2 = 16; };

// 2-D transform of NIMG row-major N x N images in shared memory (row stride
// RS float2, image stride IS float2): rows (range) then columns (azimuth).
template <int N, int DIR, int NIMG, int NT, int RS, int IS>
__device__ __forceinline__ void fft2d_smem(float2* base, const float2* __restrict__ tw)
{
    constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
    fft_lines<N1, N2, DIR, N * NIMG, N, NT, RS, 1, IS>(base, tw);  // rows: line = row
    fft_lines<N1, N2, DIR, N * NIMG, N, NT, 1, RS, IS>(base, tw);  // columns: line = column
}

// ---------------------------------------------------------------- three-step lines
// Large lengths N = N1 N2 N3 (x index n = M n1 + N3 n2 + n3 with M = N2 N3,
// X index k = k1 + N1 k2 + N1 N2 k3): step A radix-N1 over n1 with twiddle
// W_N^{k1 m}; step B radix-N2 over n2 inside each block of M with twiddle
// W_N^{N1 k2 n3}; step C radix-N3 over the contiguous n3, handed to
// out(l, k, value).  A and B are in place in `base`; C reads `base` and must
// write elsewhere (out may not alias base), so nothing is held across a
// barrier and every step needs at most max(N1, N2, N3) complex registers.
template <int N> struct Split3;
template <> struct Split3<16>  { static constexpr int N1 = 2, N2 = 2, N3 = 4; };
template <> struct Split3<24>  { static constexpr int N1 = 2, N2 = 3, N3 = 4; };
template <> struct Split3<32>  { static constexpr int N1 = 2, N2 = 4, N3 = 4; };
template <> struct Split3<48>  { static constexpr int N1 = 3, N2 = 4, N3 = 4; };
template <> struct Split3<64>  { static constexpr int N1 = 4, N2 = 4, N3 = 4; };
template <> struct Split3<96>  { static constexpr int N1 = 6, N2 = 4, N3 = 4; };
template <> struct Split3<128> { static constexpr int N1 = 8, N2 = 4, N3 = 4; };
template <> struct Split3<192> { static constexpr int N1 = 3, N2 = 8, N3 = 8; };
template <> struct Split3<224> { static constexpr int N1 = 7, N2 = 4, N3 = 8; };
template <> struct Split3<256> { static constexpr int N1 = 4, N2 = 8, N3 = 8; };
template <> struct Split3<384> { static constexpr int N1 = 6, N2 = 8, N3 = 8; };
template <> struct Split3<448> { static constexpr int N1 = 7, N2 = 8, N3 = 8; };
template <> struct Split3<512> { static constexpr int N1 = 8, N2 = 8, N3 = 8; };

template <int N1, int N2, int N3, int DIR, int NL, int NT, int LS, int ES, typename Out>
__device__ __forceinline__ void fft_lines3(float2* base, Out out, const float2* __restrict__ tw)
{
    constexpr int N = N1 * N2 * N3, M = N2 * N3;
    const int tid = threadIdx.x;
    for (int t = tid; t < NL * M; t += NT) {
        const int l = t % NL, m = t / NL;
        float2* p = base + l * LS + m * ES;
        float2 v[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) v[n1] = p[(M * n1) * ES];
        RegDFT<N1, DIR, N>::run(v, tw);
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1) v[k1] = twmul_rt<DIR>(v[k1], tw, k1 * m);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) p[(M * k1) * ES] = v[k1];
    }
    __syncthreads();
    for (int t = tid; t < NL * N1 * N3; t += NT) {
        const int l = t % NL, r = t / NL;
        const int n3 = r % N3, k1 = r / N3;
        float2* p = base + l * LS + (M * k1 + n3) * ES;
        float2 v[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) v[n2] = p[(N3 * n2) * ES];
        RegDFT<N2, DIR, N>::run(v, tw);
#pragma unroll
        for (int k2 = 1; k2 < N2; ++k2) v[k2] = twmul_rt<DIR>(v[k2], tw, N1 * k2 * n3);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) p[(N3 * k2) * ES] = v[k2];
    }
    __syncthreads();
    for (int t = tid; t < NL * N1 * N2; t += NT) {
        const int l = t % NL, r = t / NL;
        const int k2 = r % N2, k1 = r / N2;
        const float2* p = base + l * LS + (M * k1 + N3 * k2) * ES;
        float2 v[N3];
#pragma unroll
        for (int n3 = 0; n3 < N3; ++n3) v[n3] = p[n3 * ES];
        RegDFT<N3, DIR, N>::run(v, tw);
#pragma unroll
        for (int k3 = 0; k3 < N3; ++k3) out(l, k1 + N1 * k2 + N1 * N2 * k3, v[k3]);
    }
    __syncthreads();
}

// 2-D transform of an N x N row-major array anywhere in memory (row stride N;
// normally a per-CTA global workspace) staged through shared-memory tiles of
// G lines: rows first, then columns.  THREE selects the three-step line form
// (Split3<N>; fewest registers, G = 8 lines per tile), which writes its last
// step out of place into `tileB`; the two-step form (Split<N>) works in place
// and takes tileB = nullptr.  Tile sizes: StagedTile<N, THREE>.
template <int N, bool THREE>
struct StagedTile {
    static constexpr int G = THREE ? 8 : ((N % 16 == 0) ? 16 : 8);
    static constexpr int elems = (G * (N + 1) > N * (G + 1)) ? G * (N + 1) : N * (G + 1);
    static constexpr int elemsB = THREE ? elems : 0;
};

// Line transforms of one staged tile (rows: G lines of N at stride N+1;
// columns: lines at stride 1, elements at stride G+1).  Returns the tile
// holding the result (tile, or tileB for the three-step form).
template <int N, int DIR, int NT, bool THREE, int LS, int ES>
__device__ __forceinline__ const float2* staged_tile_fft(float2* tile, float2* tileB, const float2* __restrict__ tw)
{
    constexpr int G = StagedTile<N, THREE>::G;
    if constexpr (THREE) {
        constexpr int N1 = Split3<N>::N1, N2 = Split3<N>::N2, N3 = Split3<N>::N3;
        auto out = [tileB](int l, int k, float2 v) { tileB[l * LS + k * ES] = v; };
        fft_lines3<N1, N2, N3, DIR, G, NT, LS, ES>(tile, out, tw);
        return tileB;
    } else {
        constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
        fft_lines<N1, N2, DIR, G, G, NT, LS, ES, 0>(tile, tw);
        return tile;
    }
}

// Row pass of a staged N x N transform: row r of gout becomes DFT_N(src(r, .)).
// src(r, k) may read row r of gout itself (in place): a tile of G rows is
// loaded completely before it is written back.
template <int N, int DIR, int NT, bool THREE, typename Src>
__device__ __forceinline__ void staged_rows(float2* gout, Src src, float2* tile, float2* tileB,
                                            const float2* __restrict__ tw)
{
    constexpr int G = StagedTile<N, THREE>::G;
    const int tid = threadIdx.x;
    for (int r0 = 0; r0 < N; r0 += G) {
#pragma unroll 4
        for (int e = tid; e < G * N; e += NT) {
            const int l = e / N, k = e % N;
            tile[l * (N + 1) + k] = src(r0 + l, k);
        }
        __syncthreads();
        const float2* res = staged_tile_fft<N, DIR, NT, THREE, N + 1, 1>(tile, tileB, tw);
#pragma unroll 4
        for (int e = tid; e < G * N; e += NT) {
            const int l = e / N, k = e % N;
            gout[(size_t)(r0 + l) * N + k] = res[l * (N + 1) + k];
        }
        __syncthreads();
    }
}

// Column pass of a staged N x N transform: column c becomes DFT_N(src(., c)),
// handed element by element to dst(k, c, value).  keep(c0) (uniform across
// the block) skips the tile of columns c0 .. c0+G-1 when false: a pass whose
// consumer reads only some columns transforms only the tiles holding them.
template <int N, int DIR, int NT, bool THREE, typename Src, typename Dst, typename Keep>
__device__ __forceinline__ void staged_cols_if(Src src, Dst dst, Keep keep, float2* tile, float2* tileB,
                                               const float2* __restrict__ tw)
{
    constexpr int G = StagedTile<N, THREE>::G;
    const int tid = threadIdx.x;
    for (int c0 = 0; c0 < N; c0 += G) {
        if (!keep(c0)) continue;
#pragma unroll 4
        for (int e = tid; e < N * G; e += NT) {
            const int k = e / G, l = e % G;
            tile[k * (G + 1) + l] = src(k, c0 + l);
        }
        __syncthreads();
        const float2* res = staged_tile_fft<N, DIR, NT, THREE, 1, G + 1>(tile, tileB, tw);
#pragma unroll 4
        for (int e = tid; e < N * G; e += NT) {
            const int k = e / G, l = e % G;
            dst(k, c0 + l, res[k * (G + 1) + l]);
        }
        __syncthreads();
    }
}

template <int N, int DIR, int NT, bool THREE, typename Src, typename Dst>
__device__ __forceinline__ void staged_cols(Src src, Dst dst, float2* tile, float2* tileB,
                                            const float2* __restrict__ tw)
{
    staged_cols_if<N, DIR, NT, THREE>(src, dst, [](int) { return true; }, tile, tileB, tw);
}

// 2-D transform of an N x N row-major array anywhere in memory (row stride N;
// normally a per-CTA global workspace) staged through the tiles: rows, then
// columns, in place.
template <int N, int DIR, int NT, bool THREE = false>
__device__ __forceinline__ void fft2d_staged(float2* g, float2* tile, const float2* __restrict__ tw,
                                             float2* tileB)
{
    staged_rows<N, DIR, NT, THREE>(g, [g](int r, int k) { return g[(size_t)r * N + k]; }, tile, tileB, tw);
    staged_cols<N, DIR, NT, THREE>([g](int k, int c) { return g[(size_t)k * N + c]; },
                                   [g](int k, int c, float2 v) { g[(size_t)k * N + c] = v; }, tile, tileB, tw);
}

}  // namespace sbfft
