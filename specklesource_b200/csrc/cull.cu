// cull.cu -- the cullst passes on the GPU (Cullst/cullst.c:71-101).
//
//  cullSTData (cullSTData.c:13-125): the median test runs in place in raster
//    order, so a cull changes the neighbourhoods of later points.  The GPU
//    first solves that recurrence as a parallel fixpoint (cull_fix_kernel on
//    revisit lists, exact when it converges); otherwise it keeps the order with a row
//    wavefront: one warp per grid row
//    (rows claimed in increasing order from a counter, so the row a warp waits
//    on is always held by a running warp), each warp walks its row left to
//    right and, before deciding column j, waits until the previous row has
//    finished column j + bR/2 (transitively every earlier row in the box is
//    done that far).  Both medians (the 1-based k = ngood/2 smallest of the
//    valid neighbours, what Numerical Recipes' select returns) come from a
//    warp-wide radix select over order-preserving float keys.  Waits are
//    bounded: on time-out the kernel records an error and releases its row.
//  cullStats (cullStats.c:19-144), cullSmooth (cullSmooth.c:29-103): one
//    thread per point.  The plane fit is least squares with singular values
//    below 1e-5 * max dropped (svdfit), via the 3x3 normal matrix's Jacobi
//    eigen-decomposition, in double precision.
//  cullls (Cullls/cullls.c:23-56) runs the same kernels: its median pass
//    (cullLSData.c:13-138) adds the slow-flow limits and the NODATA test to
//    the decision rule (StRule), its stats (cullLSStats.c) the quantisation
//    variance, its smoothing (cullLSSmooth.c) is the unweighted box mean of
//    cullls_smooth_kernel, and its islands pass is cullIslands'.
//  cullIslands (cullIslands.c:13-198): union-find labelling (links to the
//    smaller index, so each root is its component's first pixel in raster
//    order), labels numbered by first appearance, bounding boxes, and the cull
//    of components no wider or taller than islandThresh -- except the one
//    labelled last, which the reference's loops (i < maxLabel) skip.
#include <cuda/atomic>
#include <cuda_runtime.h>
#include <stdint.h>

#include "capi_internal.h"

namespace sbk {

constexpr float kCulled = -2.0e9f;  // (float)-LARGEINT
constexpr float kValidLim = -2.0e9f; // (float)(1 - LARGEINT): 1 - 2e9 rounds to -2e9 in float

__device__ __forceinline__ bool valid_pt(float r, float a) { return r > kValidLim && a > kValidLim; }

// ---------------------------------------------------------------- pre-pass

// The decision rule of one median pass.  cullst (cullSTData.c:80-123): cull
// unless more than nGood valid neighbours and both deviations from the box
// medians within maxA/maxR.  cullls (cullLSData.c:63-134) adds: the limits
// become slowMaxA/slowMaxR when every valid point of the box carries a
// slowMask bit in slowType, and the point's own offA must exceed selfLim.
struct StRule {
    int nGood;
    double maxR, maxA;
    double slowMaxR, slowMaxA;
    const uint8_t* slowType;  // null: no slow-flow test (cullst)
    unsigned slowMask;
    bool selfTest;            // cullls: the point's offA must exceed selfLim (false for NaN)
    double selfLim;
};

struct CullArgs {
    float* offR;
    float* offA;
    const float* corr;
    uint8_t* type;
    const uint8_t* mask;
    int nR, nA;
    int bR, bA;
    StRule rule;
    float corrThresh;
    int singleMT;
    int* rowCounter;
    int* progress;
    int* errFlag;
    unsigned long long* nCulled;
};

__global__ void cull_prepass_kernel(CullArgs a)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.nR * a.nA) return;
    if (a.corr[k] < a.corrThresh) {  // cullSTData.c:38-43
        a.offR[k] = kCulled;
        a.offA[k] = kCulled;
        a.type[k] = 0;
    }
    if (a.mask) {  // :44-61 (singleMT is only honoured with a mask)
        const unsigned char mv = a.mask[k] & 4;
        if (mv > 0 && (signed char)a.type[k] > 2) {
            a.offR[k] = kCulled;
            a.offA[k] = kCulled;
            a.type[k] = 0;
        }
        if (a.singleMT > 0 && (signed char)a.type[k] != a.singleMT) {
            a.offR[k] = kCulled;
            a.offA[k] = kCulled;
            a.type[k] = 0;
        }
    }
}

// ---------------------------------------------------------------- median pass

__device__ __forceinline__ uint32_t fkey(float f)
{
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fkey_inv(uint32_t k)
{
    const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

// k-th smallest key (1-based) among the lane's NV keys flagged by vmask.
template <int NV>
__device__ __forceinline__ uint32_t warp_kth(const uint32_t (&key)[NV], uint32_t vmask, int k)
{
    uint32_t prefix = 0;
    int below = 0;
#pragma unroll 1
    for (int bit = 31; bit >= 0; --bit) {
        const uint32_t hi = (bit == 31) ? 0u : (0xffffffffu << (bit + 1));
        int c = 0;
#pragma unroll
        for (int v = 0; v < NV; ++v)
            c += ((vmask >> v) & 1u) && ((key[v] & hi) == prefix) && !((key[v] >> bit) & 1u);
        c = __reduce_add_sync(0xffffffffu, c);
        if (below + c < k)
            below += c, prefix |= (1u << bit);
    }
    return prefix;
}

// One point's decision, by a whole warp (uniform result).  kr/ka: the lanes'
// keys of the valid box points (vm), notSlow: this lane saw a valid point
// without the slow bit; oR/oA: the point's own offsets.
template <int NV>
__device__ __forceinline__ bool st_decide(const StRule& r, const uint32_t (&kr)[NV], const uint32_t (&ka)[NV],
                                          uint32_t vm, int ngood, bool notSlow, float oR, float oA)
{
    const bool slow = r.slowType != nullptr && !__any_sync(0xffffffffu, notSlow);
    if ((unsigned)ngood > (unsigned)r.nGood && (!r.selfTest || (double)oA > r.selfLim)) {
        int mid = ngood / 2;
        if (mid < 1) mid = 1;
        const float medR = fkey_inv(warp_kth<NV>(kr, vm, mid));
        const float medA = fkey_inv(warp_kth<NV>(ka, vm, mid));
        const double dA = (double)(oA - medA), dR = (double)(oR - medR);
        return fabs(dA) > (slow ? r.slowMaxA : r.maxA) || fabs(dR) > (slow ? r.slowMaxR : r.maxR);
    }
    return true;
}

template <int NV>
__global__ void cull_median_kernel(CullArgs a, long long spinLimit)
{
    const int lane = threadIdx.x & 31;
    const int hA = a.bA / 2, hR = a.bR / 2;
    const int boxW = 2 * hR + 1;
    cuda::atomic_ref<int, cuda::thread_scope_device> ctr(*a.rowCounter);
    unsigned long long culledHere = 0;
    while (true) {
        int row = 0;
        if (lane == 0) row = ctr.fetch_add(1, cuda::memory_order_relaxed);
        row = __shfl_sync(0xffffffffu, row, 0);
        if (row >= a.nA) break;
        const int i1 = row - hA > 0 ? row - hA : 0;
        const int i2 = row + hA < a.nA - 1 ? row + hA : a.nA - 1;
        bool timedOut = false;
        for (int j = 0; j < a.nR; ++j) {
            // wait for the previous row to finish column j + hR
            if (row > 0) {
                const int need = (j + hR + 1 < a.nR) ? j + hR + 1 : a.nR;
                cuda::atomic_ref<int, cuda::thread_scope_device> prev(a.progress[row - 1]);
                int ok = 1;
                if (lane == 0) {
                    long long spins = 0;
                    while (prev.load(cuda::memory_order_acquire) < need) {
                        if (++spins > spinLimit) {
                            ok = 0;
                            break;
                        }
                        __nanosleep(64);
                    }
                }
                ok = __shfl_sync(0xffffffffu, ok, 0);
                if (!ok) {
                    timedOut = true;
                    break;
                }
                (void)prev.load(cuda::memory_order_acquire);  // every lane acquires what lane 0 saw
                __syncwarp();
            }
            const int j1 = j - hR > 0 ? j - hR : 0;
            const int j2 = j + hR < a.nR - 1 ? j + hR : a.nR - 1;
            const int rows = i2 - i1 + 1, cols = j2 - j1 + 1;
            const int cnt = rows * cols;
            uint32_t kr[NV], ka[NV];
            uint32_t vm = 0;
            bool notSlow = false;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const int e = lane + 32 * v;
                kr[v] = ka[v] = 0;
                if (e < cnt) {
                    const int ii = i1 + e / cols, jj = j1 + e % cols;
                    const size_t q = (size_t)ii * a.nR + jj;
                    const float r = __ldcg(&a.offR[q]), az = __ldcg(&a.offA[q]);
                    if (valid_pt(r, az)) {
                        vm |= 1u << v;
                        kr[v] = fkey(r);
                        ka[v] = fkey(az);
                        if (a.rule.slowType && !(a.rule.slowType[q] & a.rule.slowMask)) notSlow = true;
                    }
                }
            }
            int ngood = 0;
#pragma unroll
            for (int v = 0; v < NV; ++v) ngood += (vm >> v) & 1u;
            ngood = __reduce_add_sync(0xffffffffu, ngood);
            const size_t c = (size_t)row * a.nR + j;
            const bool cull =
                st_decide<NV>(a.rule, kr, ka, vm, ngood, notSlow, __ldcg(&a.offR[c]), __ldcg(&a.offA[c]));
            if (lane == 0) {
                if (cull) {
                    a.offR[c] = kCulled;
                    a.offA[c] = kCulled;
                    culledHere++;
                }
                cuda::atomic_ref<int, cuda::thread_scope_device> mine(a.progress[row]);
                mine.store(j + 1, cuda::memory_order_release);
            }
            __syncwarp();
            (void)boxW;
        }
        if (timedOut) {
            if (lane == 0) {
                atomicExch(a.errFlag, 1);
                cuda::atomic_ref<int, cuda::thread_scope_device> mine(a.progress[row]);
                mine.store(a.nR, cuda::memory_order_release);
            }
        }
    }
    if (lane == 0 && culledHere) atomicAdd(a.nCulled, culledHere);
}

// ---------------------------------------------------------------- median pass, parallel fixpoint
// The sequential pass decides point p from the values at the start of the pass
// and from the decisions of the points before p (raster order) in its box:
// C[p] = decide(p, {C[q] : q < p, q in box(p)}).  This recurrence over a DAG
// has exactly one solution, the sequential result.  Jacobi iteration
// C_{t+1} = decide(., C_t) from C_0 = 0 reaches it, and a step that changes
// nothing proves it was reached (a fixpoint of the recurrence is its solution).
// Step t decides only the points on its revisit list (every point at t = 0;
// after that the later box neighbours of the points that flipped in step
// t - 1): any other point has no predecessor that changed, so its decision
// is already C_t's.  The decisions of a step are read from C_t and the flips
// applied afterwards (cull_fix_apply_kernel), so every step is exactly a
// Jacobi step.  offR/offA are not modified until the fixpoint is applied;
// one warp per point, medians as in the wavefront kernel.
struct FixArgs {
    const float* offR;
    const float* offA;
    const uint8_t* c;        // C_t
    const int* list;         // revisit list; null: every point (step 0)
    const unsigned* count;   // its length (ignored when list is null)
    int* flipped;            // points whose decision flips in this step
    unsigned* nFlipped;
    int nR, nA, bR, bA;
    StRule rule;
};

template <int NV>
__global__ void cull_fix_kernel(FixArgs a)
{
    const int lane = threadIdx.x & 31;
    const int hA = a.bA / 2, hR = a.bR / 2;
    const long long n = a.list ? (long long)*a.count : (long long)a.nR * a.nA;
    const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long t = w0; t < n; t += nw) {
        const long long p = a.list ? (long long)a.list[t] : t;
        const int i = (int)(p / a.nR), j = (int)(p % a.nR);
        const int i1 = i - hA > 0 ? i - hA : 0, i2 = i + hA < a.nA - 1 ? i + hA : a.nA - 1;
        const int j1 = j - hR > 0 ? j - hR : 0, j2 = j + hR < a.nR - 1 ? j + hR : a.nR - 1;
        const int cols = j2 - j1 + 1, cnt = (i2 - i1 + 1) * cols;
        uint32_t kr[NV], ka[NV];
        uint32_t vm = 0;
        bool notSlow = false;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const int e = lane + 32 * v;
            kr[v] = ka[v] = 0;
            if (e < cnt) {
                const long long q = (long long)(i1 + e / cols) * a.nR + (j1 + e % cols);
                const float r = a.offR[q], az = a.offA[q];
                if (valid_pt(r, az) && !(q < p && a.c[q])) {
                    vm |= 1u << v;
                    kr[v] = fkey(r);
                    ka[v] = fkey(az);
                    if (a.rule.slowType && !(a.rule.slowType[q] & a.rule.slowMask)) notSlow = true;
                }
            }
        }
        int ngood = 0;
#pragma unroll
        for (int v = 0; v < NV; ++v) ngood += (vm >> v) & 1u;
        ngood = __reduce_add_sync(0xffffffffu, ngood);
        const bool cull = st_decide<NV>(a.rule, kr, ka, vm, ngood, notSlow, a.offR[p], a.offA[p]);
        if (lane == 0 && (cull ? 1 : 0) != a.c[p]) a.flipped[atomicAdd(a.nFlipped, 1u)] = (int)p;
    }
}

// Applies a step's flips to C and lists the points to decide next: the later
// points (raster order) whose box holds a flipped point, each once per step
// (mark[] holds the step that listed it).  One warp per flipped point: the
// lanes take its later box neighbours 32 at a time and reserve their list
// slots with one atomic per warp.
__global__ void cull_fix_apply_kernel(uint8_t* c, const int* flipped, const unsigned* nFlipped, int* next,
                                      unsigned* nNext, int* mark, int stamp, int nR, int nA, int bR, int bA)
{
    const int lane = threadIdx.x & 31;
    const unsigned nf = *nFlipped;
    const int hA = bA / 2, hR = bR / 2;
    const unsigned w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned nw = (gridDim.x * blockDim.x) >> 5;
    for (unsigned k = w0; k < nf; k += nw) {
        const int q = flipped[k];
        if (lane == 0) c[q] ^= 1;
        const int i = q / nR, j = q % nR;
        const int i2 = i + hA < nA - 1 ? i + hA : nA - 1;
        const int j1 = j - hR > 0 ? j - hR : 0, j2 = j + hR < nR - 1 ? j + hR : nR - 1;
        const int cols = j2 - j1 + 1;
        const int sameRow = j2 - j;                 // (i, j+1 .. j2)
        const int total = sameRow + (i2 - i) * cols;  // then rows i+1 .. i2, columns j1 .. j2
        for (int b = 0; b < total; b += 32) {
            const int e = b + lane;
            int pp = -1;
            if (e < total) {
                const int y = e < sameRow ? i : i + 1 + (e - sameRow) / cols;
                const int x = e < sameRow ? j + 1 + e : j1 + (e - sameRow) % cols;
                pp = y * nR + x;
                if (atomicExch(mark + pp, stamp) == stamp) pp = -1;  // listed already in this step
            }
            const unsigned fresh = __ballot_sync(0xffffffffu, pp >= 0);
            unsigned base = 0;
            if (lane == 0 && fresh) base = atomicAdd(nNext, (unsigned)__popc(fresh));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (pp >= 0) next[base + __popc(fresh & ((1u << lane) - 1u))] = pp;
        }
    }
}

// Writes the culls of the converged pass; counts them.
__global__ void cull_apply_kernel(float* offR, float* offA, const uint8_t* c, long long n,
                                  unsigned long long* nCulled)
{
    unsigned long long k = 0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        if (c[p]) {
            offR[p] = kCulled;
            offA[p] = kCulled;
            k++;
        }
    }
    k = __reduce_add_sync(0xffffffffu, (unsigned)k);
    if ((threadIdx.x & 31) == 0 && k) atomicAdd(nCulled, k);
}

// ---------------------------------------------------------------- stats

__device__ void jacobi3(double A[3][3], double e[3], double V[3][3])
{
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) V[i][j] = (i == j);
    for (int sweep = 0; sweep < 60; sweep++) {
        const double off = fabs(A[0][1]) + fabs(A[0][2]) + fabs(A[1][2]);
        if (off == 0.0) break;
        for (int pq = 0; pq < 3; pq++) {
            const int P = pq == 2 ? 1 : 0, Q = pq == 0 ? 1 : 2;
            if (A[P][Q] == 0.0) continue;
            const double theta = (A[Q][Q] - A[P][P]) / (2.0 * A[P][Q]);
            const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            const double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
            for (int k = 0; k < 3; k++) {
                const double akp = A[k][P], akq = A[k][Q];
                A[k][P] = cs * akp - sn * akq;
                A[k][Q] = sn * akp + cs * akq;
            }
            for (int k = 0; k < 3; k++) {
                const double apk = A[P][k], aqk = A[Q][k];
                A[P][k] = cs * apk - sn * aqk;
                A[Q][k] = sn * apk + cs * aqk;
            }
            for (int k = 0; k < 3; k++) {
                const double vkp = V[k][P], vkq = V[k][Q];
                V[k][P] = cs * vkp - sn * vkq;
                V[k][Q] = sn * vkp + cs * vkq;
            }
        }
    }
    for (int i = 0; i < 3; i++) e[i] = A[i][i];
}

// svdfit with basis (x0, ii, jj) over the valid points of a box
__device__ void plane_fit(double x0, const float* off, const float* other, int nR, int i1, int i2, int j1, int j2,
                          double coef[3])
{
    double AtA[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Atb[3] = {0, 0, 0};
    for (int ii = i1; ii <= i2; ii++)
        for (int jj = j1; jj <= j2; jj++) {
            const size_t q = (size_t)ii * nR + jj;
            const float r = off[q], o = other[q];
            if (!valid_pt(r, o)) continue;
            const double f[3] = {x0, (double)(float)ii, (double)(float)jj};
            for (int u = 0; u < 3; u++) {
                Atb[u] += f[u] * (double)r;
                for (int v = 0; v < 3; v++) AtA[u][v] += f[u] * f[v];
            }
        }
    double e[3], V[3][3];
    jacobi3(AtA, e, V);
    double s[3], smax = 0;
    for (int u = 0; u < 3; u++) {
        s[u] = e[u] > 0 ? sqrt(e[u]) : 0.0;
        smax = s[u] > smax ? s[u] : smax;
    }
    const double thresh = 1.0e-5 * smax;
    coef[0] = coef[1] = coef[2] = 0.0;
    for (int u = 0; u < 3; u++) {
        if (s[u] < thresh || s[u] == 0.0) continue;
        const double proj = V[0][u] * Atb[0] + V[1][u] * Atb[1] + V[2][u] * Atb[2];
        const double w = proj / (s[u] * s[u]);
        for (int v = 0; v < 3; v++) coef[v] += V[v][u] * w;
    }
}

struct StatsArgs {
    const float* offR;
    const float* offA;
    float* sigmaR;
    float* sigmaA;
    int nR, nA;
    double qvar;  // cullls: quantisation variance (1/NOVER)^2/12 added before the root; 0 for cullst
};

__global__ void cull_stats_kernel(StatsArgs a)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.nR * a.nA) return;
    const int i = k / a.nR, j = k % a.nR;
    const int b = 9;  // cullStats.c:38-39
    const int i1 = i - b / 2 > 0 ? i - b / 2 : 0, i2 = i + b / 2 < a.nA - 1 ? i + b / 2 : a.nA - 1;
    const int j1 = j - b / 2 > 0 ? j - b / 2 : 0, j2 = j + b / 2 < a.nR - 1 ? j + b / 2 : a.nR - 1;
    unsigned ngood = 0;
    double meanA = 0.0, meanR = 0.0;
    for (int ii = i1; ii <= i2; ii++)
        for (int jj = j1; jj <= j2; jj++) {
            const size_t q = (size_t)ii * a.nR + jj;
            if (valid_pt(a.offR[q], a.offA[q])) {
                ngood++;
                meanA += a.offA[q];
                meanR += a.offR[q];
            }
        }
    meanA /= (double)ngood;
    meanR /= (double)ngood;
    double aR[4] = {0, 0, 0, 0}, aA[4] = {0, 0, 0, 0};
    if (ngood > 8) {
        double c[3];
        plane_fit((double)(float)meanR, a.offR, a.offA, a.nR, i1, i2, j1, j2, c);
        aR[1] = c[0] * meanR;
        aR[2] = c[1];
        aR[3] = c[2];
        plane_fit((double)(float)meanA, a.offA, a.offR, a.nR, i1, i2, j1, j2, c);
        aA[1] = c[0] * meanA;
        aA[2] = c[1];
        aA[3] = c[2];
    }
    ngood = 0;
    meanA = meanR = 0.0;
    double varR = 0.0, varA = 0.0;
    for (int ii = i1; ii <= i2; ii++)
        for (int jj = j1; jj <= j2; jj++) {
            const size_t q = (size_t)ii * a.nR + jj;
            if (valid_pt(a.offR[q], a.offA[q])) {
                ngood++;
                float oR = a.offR[q], oA = a.offA[q];
                oR = (float)((double)oR - (aR[1] + aR[2] * (float)ii + aR[3] * (float)jj));
                oA = (float)((double)oA - (aA[1] + aA[2] * (float)ii + aA[3] * (float)jj));
                meanA += oA;
                meanR += oR;
                varA += (double)(oA * oA);
                varR += (double)(oR * oR);
            }
        }
    if (ngood > 8 && a.offR[k] > kValidLim) {
        float sA = (float)(varA / (float)(ngood - 3));
        float sR = (float)(varR / (float)(ngood - 3));
        sA = (float)((double)sA - meanA * meanA / (float)((ngood - 3) * ngood));
        sR = (float)((double)sR - meanR * meanR / (float)((ngood - 3) * ngood));
        sA = (float)(0.00001 > (double)sA ? 0.00001 : (double)sA);
        sR = (float)(0.00001 > (double)sR ? 0.00001 : (double)sR);
        if (a.qvar != 0.0) {  // cullLSStats.c:147-148
            sR = (float)((double)sR + a.qvar);
            sA = (float)((double)sA + a.qvar);
        }
        a.sigmaA[k] = (float)sqrt((double)sA);
        a.sigmaR[k] = (float)sqrt((double)sR);
    } else {
        a.sigmaA[k] = kCulled;
        a.sigmaR[k] = kCulled;
    }
}

// ---------------------------------------------------------------- smooth

struct SmoothArgs {
    const float* offR;
    const float* offA;
    const uint8_t* type;
    float* sigmaR;
    float* sigmaA;
    float* offRS;
    float* offAS;
    int nR, nA, sR, sA;
};

__device__ __forceinline__ float sweight(int m, int s)
{
    const float w2 = (float)((float)s / 2.0 - 0.01);  // cullSmooth.c:10-27
    return (m < -w2 || m > w2) ? 0.5f : 1.0f;
}

__global__ void cull_smooth_kernel(SmoothArgs a)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.nR * a.nA) return;
    const int i = k / a.nR, j = k % a.nR;
    const float nlooks[4] = {0.0f, 1.0f, 0.25f, 0.015f};
    const int i1 = i - a.sA / 2 > 0 ? i - a.sA / 2 : 0, i2 = i + a.sA / 2 < a.nA - 1 ? i + a.sA / 2 : a.nA - 1;
    const int j1 = j - a.sR / 2 > 0 ? j - a.sR / 2 : 0, j2 = j + a.sR / 2 < a.nR - 1 ? j + a.sR / 2 : a.nR - 1;
    double ngood = 0, meanA = 0.0, meanR = 0.0;
    float nLooksEff = 0.0f;
    for (int ii = i1; ii <= i2; ii++) {
        const float wa = sweight(ii - i, a.sA);
        for (int jj = j1; jj <= j2; jj++) {
            const size_t q = (size_t)ii * a.nR + jj;
            if (valid_pt(a.offR[q], a.offA[q])) {
                const double w = (double)(wa * sweight(jj - j, a.sR));
                ngood = __dadd_rn(ngood, w);
                nLooksEff = (float)__dadd_rn((double)nLooksEff, __dmul_rn(w, (double)nlooks[(int)(signed char)a.type[q] & 3]));
                meanA = __dadd_rn(meanA, __dmul_rn(w, (double)a.offA[q]));
                meanR = __dadd_rn(meanR, __dmul_rn(w, (double)a.offR[q]));
            }
        }
    }
    if (((ngood > 1) || (a.sA == 1) || (a.sR == 1)) && a.offR[k] > kValidLim && a.sigmaA[k] > kValidLim) {
        nLooksEff = (float)((double)nLooksEff > 1. ? (double)nLooksEff : 1.);
        a.sigmaA[k] = (float)((double)a.sigmaA[k] / sqrt((double)nLooksEff));
        a.sigmaR[k] = (float)((double)a.sigmaR[k] / sqrt((double)nLooksEff));
        a.offRS[k] = (float)(meanR / (float)ngood);
        a.offAS[k] = (float)(meanA / (float)ngood);
    } else {
        a.offRS[k] = kCulled;
        a.offAS[k] = kCulled;
    }
}

// cullLSSmooth.c:29-70: the unweighted mean over the sA x sR box, one look
// per valid point.
__global__ void cullls_smooth_kernel(SmoothArgs a)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.nR * a.nA) return;
    const int i = k / a.nR, j = k % a.nR;
    const int i1 = i - a.sA / 2 > 0 ? i - a.sA / 2 : 0, i2 = i + a.sA / 2 < a.nA - 1 ? i + a.sA / 2 : a.nA - 1;
    const int j1 = j - a.sR / 2 > 0 ? j - a.sR / 2 : 0, j2 = j + a.sR / 2 < a.nR - 1 ? j + a.sR / 2 : a.nR - 1;
    unsigned ngood = 0;
    float nLooksEff = 0.0f;
    double meanA = 0.0, meanR = 0.0;
    for (int ii = i1; ii <= i2; ii++)
        for (int jj = j1; jj <= j2; jj++) {
            const size_t q = (size_t)ii * a.nR + jj;
            if (valid_pt(a.offR[q], a.offA[q])) {
                ngood++;
                nLooksEff += 1.0f;
                meanA += (double)a.offA[q];
                meanR += (double)a.offR[q];
            }
        }
    if (((ngood > 1) || (a.sA == 1) || (a.sR == 1)) && a.offR[k] > kValidLim && a.sigmaA[k] > kValidLim) {
        nLooksEff = (float)((double)nLooksEff > 1. ? (double)nLooksEff : 1.);
        a.sigmaA[k] = (float)((double)a.sigmaA[k] / sqrt((double)nLooksEff));
        a.sigmaR[k] = (float)((double)a.sigmaR[k] / sqrt((double)nLooksEff));
        a.offRS[k] = (float)(meanR / (float)ngood);
        a.offAS[k] = (float)(meanA / (float)ngood);
    } else {
        a.offRS[k] = kCulled;
        a.offAS[k] = kCulled;
    }
}

// cullLSData.c:36-57 (first pass): valid points and points with data.
__global__ void cullls_count_kernel(const float* offR, const float* offA, const uint8_t* type, unsigned noDataMask,
                                    long long n, unsigned long long* cnt)
{
    unsigned long long nv = 0, nd = 0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        nv += valid_pt(offR[p], offA[p]);
        nd += (type[p] & noDataMask) == 0;
    }
    nv = __reduce_add_sync(0xffffffffu, (unsigned)nv);
    nd = __reduce_add_sync(0xffffffffu, (unsigned)nd);
    if ((threadIdx.x & 31) == 0) {
        if (nv) atomicAdd(&cnt[0], nv);
        if (nd) atomicAdd(&cnt[1], nd);
    }
}

// ---------------------------------------------------------------- sim offsets

__global__ void cull_sim_kernel(float* offR, float* offA, const float* simR, const float* simA, int n, float sign)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    // cullst.c:109-121 with its local LARGEINT = -2e9: offA < 2e9 + 1
    if ((double)offA[k] < (2e9 + 1) && (double)simA[k] < (2e9 + 1)) {
        offA[k] = offA[k] + sign * simA[k];
        offR[k] = offR[k] + sign * simR[k];
    }
}

// ---------------------------------------------------------------- islands

__device__ __forceinline__ int uf_find(int* par, int x)
{
    int p = par[x];
    while (p != x) {
        const int g = par[p];
        if (g < p) par[x] = g;  // path halving (only towards smaller indices)
        x = p;
        p = par[x];
    }
    return x;
}

__device__ void uf_union(int* par, int a, int b)
{
    bool done = false;
    while (!done) {
        a = uf_find(par, a);
        b = uf_find(par, b);
        if (a == b) return;
        if (a < b) {
            const int t = a;
            a = b;
            b = t;
        }
        // link the larger root a under the smaller root b
        const int old = atomicMin(&par[a], b);
        done = (old == a);
        a = old;
    }
}

struct IslandArgs {
    float* offRS;
    float* offAS;
    int* par;
    int* minX;
    int* maxX;
    int* minY;
    int* maxY;
    int* lastRoot;
    unsigned long long* counts;  // [0] islands culled, [1] points culled
    int nR, nA, conn8, thresh;
};

__global__ void isl_init_kernel(IslandArgs a)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.nR * a.nA) return;
    const float minRegion = (float)(-2000000000 + 1000);  // cullIslands.c:62
    a.par[k] = a.offRS[k] >= minRegion ? k : -1;
    a.minX[k] = a.minY[k] = 0x7fffffff;
    a.maxX[k] = a.maxY[k] = -0x7fffffff;
}

__global__ void isl_union_kernel(IslandArgs a)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.nR * a.nA || a.par[k] < 0) return;
    const int i = k / a.nR, j = k % a.nR;
    if (j > 0 && a.par[k - 1] >= 0) uf_union(a.par, k, k - 1);
    if (i > 0 && a.par[k - a.nR] >= 0) uf_union(a.par, k, k - a.nR);
    if (a.conn8 && i > 0) {
        if (j > 0 && a.par[k - a.nR - 1] >= 0) uf_union(a.par, k, k - a.nR - 1);
        if (j < a.nR - 1 && a.par[k - a.nR + 1] >= 0) uf_union(a.par, k, k - a.nR + 1);
    }
}

__global__ void isl_flatten_kernel(IslandArgs a)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.nR * a.nA || a.par[k] < 0) return;
    int r = k;
    while (a.par[r] != r) r = a.par[r];
    a.par[k] = r;
    const int i = k / a.nR, j = k % a.nR;
    atomicMin(&a.minX[r], j);
    atomicMax(&a.maxX[r], j);
    atomicMin(&a.minY[r], i);
    atomicMax(&a.maxY[r], i);
    if (r == k) atomicMax(a.lastRoot, k);  // the component labelled last
}

__global__ void isl_cull_kernel(IslandArgs a)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.nR * a.nA || a.par[k] < 0) return;
    const int r = a.par[k];
    if (r == *a.lastRoot) return;
    if ((a.maxX[r] - a.minX[r]) > a.thresh || (a.maxY[r] - a.minY[r]) > a.thresh) return;
    a.offRS[k] = kCulled;
    if (a.offAS) a.offAS[k] = kCulled;
    atomicAdd(&a.counts[1], 1ull);
    if (r == k) atomicAdd(&a.counts[0], 1ull);
}

}  // namespace sbk

// ======================================================================= C ABI

using namespace sbk;

namespace {

struct CullDev {
    float *offR, *offA, *corr, *simR, *simA, *offRS, *offAS, *sigmaR, *sigmaA;
    uint8_t *type, *mask;
};

// What the passes read, from either entry point (cullst or cullls).
struct CullJob {
    int nR, nA, bR, bA, sR, sA, islandThresh, connectivity;
    StRule rule;          // rule.slowType is set to the device type grid (cullls)
    bool prepass;         // cullst: corr threshold and mask tests before the median pass
    float corrThresh;
    int singleMT;
    double qvar;          // cullls stats: quantisation variance
    bool lsSmooth;        // cullls smoothing
};

CullJob job_of(const sb_cull_params* p)
{
    CullJob j;
    j.nR = p->nR; j.nA = p->nA; j.bR = p->bR; j.bA = p->bA; j.sR = p->sR; j.sA = p->sA;
    j.islandThresh = p->islandThresh; j.connectivity = p->connectivity;
    j.rule.nGood = p->nGood;
    j.rule.maxR = p->maxR; j.rule.maxA = p->maxA;
    j.rule.slowMaxR = p->maxR; j.rule.slowMaxA = p->maxA;
    j.rule.slowType = nullptr;
    j.rule.slowMask = 0;
    j.rule.selfTest = false;
    j.rule.selfLim = 0.0;
    j.prepass = true;
    j.corrThresh = p->corrThresh;
    j.singleMT = p->singleMT;
    j.qvar = 0.0;
    j.lsSmooth = false;
    return j;
}

// cullLSData.c:99-117: limits where every valid neighbour is slow-moving,
// 40 m/yr over deltaT in pixels, at least 0.2; cullLSStats.c:147-148.
CullJob job_of(const sb_cullls_params* p)
{
    CullJob j;
    j.nR = p->nx; j.nA = p->ny; j.bR = p->boxSize; j.bA = p->boxSize; j.sR = p->sX; j.sA = p->sY;
    j.islandThresh = p->islandThresh; j.connectivity = p->connectivity;
    j.rule.nGood = p->nGood;
    j.rule.maxR = p->maxX; j.rule.maxA = p->maxY;
    double mx = 40.0 / 365. * p->deltaT, my = mx;
    mx /= p->dx;
    my /= p->dy;
    j.rule.slowMaxR = mx > 0.2 ? mx : 0.2;
    j.rule.slowMaxA = my > 0.2 ? my : 0.2;
    j.rule.slowType = nullptr;
    j.rule.slowMask = p->slowVelMask;
    j.rule.selfTest = true;
    j.rule.selfLim = p->noDataLimit;
    j.prepass = false;
    j.corrThresh = 0.0f;
    j.singleMT = 0;
    j.qvar = ((1.0 / p->nOver) * (1.0 / p->nOver)) / 12.;
    j.lsSmooth = true;
    return j;
}

int cull_check(sb_context* c, const sb_cull_params* p, const sb_cull_data* d)
{
    if (!c) return SB_ERR_ARG;
    if (!p || !d) return sb_ctx_fail(c, SB_ERR_ARG, "null params or data");
    if (p->nR <= 0 || p->nA <= 0) return sb_ctx_fail(c, SB_ERR_ARG, "empty grid");
    if ((long long)p->nR * p->nA > (1LL << 30)) return sb_ctx_fail(c, SB_ERR_ARG, "grid too large");
    if (!d->offR || !d->offA || !d->corr || !d->type) return sb_ctx_fail(c, SB_ERR_ARG, "null input grid");
    if (p->bR < 0 || p->bA < 0 || (p->bR / 2 * 2 + 1) * (p->bA / 2 * 2 + 1) > 32 * 32)
        return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "cull box larger than 32 x 32");
    if (p->useSim && (!d->simR || !d->simA)) return sb_ctx_fail(c, SB_ERR_ARG, "useSim needs simR/simA");
    return SB_OK;
}

#define CKC(call, what)                                              \
    do {                                                             \
        cudaError_t _e = (call);                                     \
        if (_e != cudaSuccess) return sb_ctx_cuda(c, _e, what);      \
    } while (0)

// Device views of the job's grids (copies host inputs in).
int cull_stage_in(sb_context* c, const sb_cull_params* p, sb_cull_data* d, CullDev* v)
{
    const size_t n = (size_t)p->nR * p->nA, fb = n * sizeof(float);
    cudaError_t e;
    if (d->onDevice) {
        v->offR = d->offR; v->offA = d->offA; v->corr = (float*)d->corr; v->type = d->type;
        v->mask = (uint8_t*)d->mask; v->simR = (float*)d->simR; v->simA = (float*)d->simA;
        v->offRS = d->offRS; v->offAS = d->offAS; v->sigmaR = d->sigmaR; v->sigmaA = d->sigmaA;
        if (!v->offRS) v->offRS = (float*)sb_ctx_buf(c, "c_offRS", fb, &e);
        if (!v->offAS) v->offAS = (float*)sb_ctx_buf(c, "c_offAS", fb, &e);
        if (!v->sigmaR) v->sigmaR = (float*)sb_ctx_buf(c, "c_sigmaR", fb, &e);
        if (!v->sigmaA) v->sigmaA = (float*)sb_ctx_buf(c, "c_sigmaA", fb, &e);
        return SB_OK;
    }
    v->offR = (float*)sb_ctx_buf(c, "c_offR", fb, &e);
    v->offA = (float*)sb_ctx_buf(c, "c_offA", fb, &e);
    v->corr = (float*)sb_ctx_buf(c, "c_corr", fb, &e);
    v->type = (uint8_t*)sb_ctx_buf(c, "c_type", n, &e);
    v->offRS = (float*)sb_ctx_buf(c, "c_offRS", fb, &e);
    v->offAS = (float*)sb_ctx_buf(c, "c_offAS", fb, &e);
    v->sigmaR = (float*)sb_ctx_buf(c, "c_sigmaR", fb, &e);
    v->sigmaA = (float*)sb_ctx_buf(c, "c_sigmaA", fb, &e);
    v->mask = d->mask ? (uint8_t*)sb_ctx_buf(c, "c_mask", n, &e) : nullptr;
    v->simR = p->useSim ? (float*)sb_ctx_buf(c, "c_simR", fb, &e) : nullptr;
    v->simA = p->useSim ? (float*)sb_ctx_buf(c, "c_simA", fb, &e) : nullptr;
    if (!v->offR || !v->offA || !v->corr || !v->type || !v->offRS || !v->offAS || !v->sigmaR || !v->sigmaA ||
        (d->mask && !v->mask) || (p->useSim && (!v->simR || !v->simA)))
        return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
    cudaStream_t s = c->stream;
    CKC(cudaMemcpyAsync(v->offR, d->offR, fb, cudaMemcpyHostToDevice, s), "h2d");
    CKC(cudaMemcpyAsync(v->offA, d->offA, fb, cudaMemcpyHostToDevice, s), "h2d");
    CKC(cudaMemcpyAsync(v->corr, d->corr, fb, cudaMemcpyHostToDevice, s), "h2d");
    CKC(cudaMemcpyAsync(v->type, d->type, n, cudaMemcpyHostToDevice, s), "h2d");
    if (d->mask) CKC(cudaMemcpyAsync(v->mask, d->mask, n, cudaMemcpyHostToDevice, s), "h2d");
    if (p->useSim) {
        CKC(cudaMemcpyAsync(v->simR, d->simR, fb, cudaMemcpyHostToDevice, s), "h2d");
        CKC(cudaMemcpyAsync(v->simA, d->simA, fb, cudaMemcpyHostToDevice, s), "h2d");
    }
    // outputs that a single pass reads (stats -> smooth -> islands)
    if (d->sigmaR) CKC(cudaMemcpyAsync(v->sigmaR, d->sigmaR, fb, cudaMemcpyHostToDevice, s), "h2d");
    if (d->sigmaA) CKC(cudaMemcpyAsync(v->sigmaA, d->sigmaA, fb, cudaMemcpyHostToDevice, s), "h2d");
    if (d->offRS) CKC(cudaMemcpyAsync(v->offRS, d->offRS, fb, cudaMemcpyHostToDevice, s), "h2d");
    if (d->offAS) CKC(cudaMemcpyAsync(v->offAS, d->offAS, fb, cudaMemcpyHostToDevice, s), "h2d");
    return SB_OK;
}

int cull_stage_out(sb_context* c, const sb_cull_params* p, sb_cull_data* d, const CullDev* v)
{
    if (d->onDevice) return SB_OK;
    const size_t n = (size_t)p->nR * p->nA, fb = n * sizeof(float);
    cudaStream_t s = c->stream;
    CKC(cudaMemcpyAsync(d->offR, v->offR, fb, cudaMemcpyDeviceToHost, s), "d2h");
    CKC(cudaMemcpyAsync(d->offA, v->offA, fb, cudaMemcpyDeviceToHost, s), "d2h");
    CKC(cudaMemcpyAsync(d->type, v->type, n, cudaMemcpyDeviceToHost, s), "d2h");
    if (d->offRS) CKC(cudaMemcpyAsync(d->offRS, v->offRS, fb, cudaMemcpyDeviceToHost, s), "d2h");
    if (d->offAS) CKC(cudaMemcpyAsync(d->offAS, v->offAS, fb, cudaMemcpyDeviceToHost, s), "d2h");
    if (d->sigmaR) CKC(cudaMemcpyAsync(d->sigmaR, v->sigmaR, fb, cudaMemcpyDeviceToHost, s), "d2h");
    if (d->sigmaA) CKC(cudaMemcpyAsync(d->sigmaA, v->sigmaA, fb, cudaMemcpyDeviceToHost, s), "d2h");
    return SB_OK;
}

// The median pass as a parallel fixpoint (cull_fix_kernel).  Returns
// SB_ERR_UNSUPPORTED, with offR/offA untouched, when it has not converged
// after kMaxFixSteps steps (or the box is too large for the warp medians):
// the caller then runs the wavefront kernel.
constexpr int kMaxFixSteps = 48;
int run_st_fixpoint(sb_context* c, const CullJob& p, const CullDev* v, int nv, int* ctl, int64_t* nCulledOut)
{
    if (nv > 4) return SB_ERR_UNSUPPORTED;
    const long long n = (long long)p.nR * p.nA;
    cudaError_t e;
    // C (bytes), then int arrays: two revisit lists, the flips, the marks
    uint8_t* C = (uint8_t*)sb_ctx_buf(c, "c_fix", (size_t)n + 16 * sizeof(int) + (size_t)n * 4 * sizeof(int), &e);
    if (!C) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
    int* ibase = (int*)(((uintptr_t)(C + n) + 15) & ~(uintptr_t)15);
    int* R[2] = {ibase, ibase + n};
    int* flipped = ibase + 2 * n;
    int* mark = ibase + 3 * n;
    unsigned* cnt = (unsigned*)sb_ctx_buf(c, "c_fixcnt", 4 * sizeof(unsigned), &e);  // |R0|, |R1|, flips
    if (!cnt) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
    cudaStream_t s = c->stream;
    CKC(cudaMemsetAsync(C, 0, (size_t)n, s), "memset");
    CKC(cudaMemsetAsync(mark, 0, (size_t)n * sizeof(int), s), "memset");
    FixArgs f;
    f.offR = v->offR; f.offA = v->offA;
    f.c = C;
    f.flipped = flipped;
    f.nFlipped = cnt + 2;
    f.nR = p.nR; f.nA = p.nA; f.bR = p.bR; f.bA = p.bA;
    f.rule = p.rule;
    const int threads = 256;
    long long blocks = (n * 32 + threads - 1) / threads;
    if (blocks > (long long)c->numSM * 64) blocks = (long long)c->numSM * 64;
    const int ablocks = c->numSM * 16;
    for (int step = 0; step < kMaxFixSteps; ++step) {
        const int in = step & 1;
        f.list = step == 0 ? nullptr : R[in];
        f.count = cnt + in;
        // the flips and the next list start empty
        CKC(cudaMemsetAsync(cnt + 2, 0, sizeof(unsigned), s), "memset");
        CKC(cudaMemsetAsync(cnt + (in ^ 1), 0, sizeof(unsigned), s), "memset");
        switch (nv) {
        case 1: cull_fix_kernel<1><<<(int)blocks, threads, 0, s>>>(f); break;
        case 2: cull_fix_kernel<2><<<(int)blocks, threads, 0, s>>>(f); break;
        case 3: cull_fix_kernel<3><<<(int)blocks, threads, 0, s>>>(f); break;
        default: cull_fix_kernel<4><<<(int)blocks, threads, 0, s>>>(f); break;
        }
        CKC(cudaGetLastError(), "cull_fix");
        cull_fix_apply_kernel<<<ablocks, 256, 0, s>>>(C, flipped, cnt + 2, R[in ^ 1], cnt + (in ^ 1), mark, step + 1,
                                                      p.nR, p.nA, p.bR, p.bA);  // one warp per flip
        CKC(cudaGetLastError(), "cull_fix_apply");
        c->launches += 2;
        unsigned changed = 0;
        CKC(cudaMemcpyAsync(&changed, cnt + 2, sizeof(changed), cudaMemcpyDeviceToHost, s), "d2h");
        CKC(cudaStreamSynchronize(s), "cull_fix");
        if (changed == 0) {
            unsigned long long* nCulled = (unsigned long long*)(ctl + 4);
            long long ab = (n + 255) / 256;
            if (ab > (long long)c->numSM * 16) ab = (long long)c->numSM * 16;
            cull_apply_kernel<<<(int)ab, 256, 0, s>>>(v->offR, v->offA, C, n, nCulled);
            CKC(cudaGetLastError(), "cull_apply");
            c->launches++;
            unsigned long long culled = 0;
            CKC(cudaMemcpyAsync(&culled, nCulled, sizeof(culled), cudaMemcpyDeviceToHost, s), "d2h");
            CKC(cudaStreamSynchronize(s), "cull_apply");
            *nCulledOut = (int64_t)culled;
            return SB_OK;
        }
    }
    return SB_ERR_UNSUPPORTED;
}

int run_st_data(sb_context* c, const CullJob& p, const CullDev* v, int64_t* nCulledOut)
{
    const int n = p.nR * p.nA;
    cudaError_t e;
    int* ctl = (int*)sb_ctx_buf(c, "c_ctl", sizeof(int) * 4 + sizeof(unsigned long long) * 2, &e);
    int* progress = (int*)sb_ctx_buf(c, "c_progress", sizeof(int) * (size_t)p.nA, &e);
    if (!ctl || !progress) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
    CullArgs a;
    a.offR = v->offR; a.offA = v->offA; a.corr = v->corr; a.type = v->type; a.mask = v->mask;
    a.nR = p.nR; a.nA = p.nA; a.bR = p.bR; a.bA = p.bA;
    a.rule = p.rule;
    a.corrThresh = p.corrThresh; a.singleMT = p.singleMT;
    a.rowCounter = ctl;
    a.errFlag = ctl + 1;
    a.nCulled = (unsigned long long*)(ctl + 4);
    a.progress = progress;
    cudaStream_t s = c->stream;
    CKC(cudaMemsetAsync(ctl, 0, sizeof(int) * 4 + sizeof(unsigned long long) * 2, s), "memset");
    CKC(cudaMemsetAsync(progress, 0, sizeof(int) * (size_t)p.nA, s), "memset");
    if (p.prepass) {
        cull_prepass_kernel<<<(n + 255) / 256, 256, 0, s>>>(a);
        CKC(cudaGetLastError(), "cull_prepass");
        c->launches++;
    }
    const int box = (p.bR / 2 * 2 + 1) * (p.bA / 2 * 2 + 1);
    const int nv = (box + 31) / 32;
    // parallel fixpoint first (exact when it converges), the wavefront if not
    {
        int rc = run_st_fixpoint(c, p, v, nv, ctl, nCulledOut);
        if (rc != SB_ERR_UNSUPPORTED) return rc;
    }
    // one warp per row in flight; enough warps for the wavefront depth
    int warps = c->numSM * 32;
    if (warps > p.nA) warps = p.nA;
    const int threads = 128, blocks = (warps * 32 + threads - 1) / threads;
    const long long spinLimit = c->waitNaps;  // 64 ns naps per wait (sb_set_wait_limit)
    switch (nv) {
    case 1: cull_median_kernel<1><<<blocks, threads, 0, s>>>(a, spinLimit); break;
    case 2: cull_median_kernel<2><<<blocks, threads, 0, s>>>(a, spinLimit); break;
    case 3: cull_median_kernel<3><<<blocks, threads, 0, s>>>(a, spinLimit); break;
    case 4: cull_median_kernel<4><<<blocks, threads, 0, s>>>(a, spinLimit); break;
    case 5: case 6: case 7: case 8: cull_median_kernel<8><<<blocks, threads, 0, s>>>(a, spinLimit); break;
    case 9: case 10: case 11: case 12: case 13: case 14: case 15: case 16:
        cull_median_kernel<16><<<blocks, threads, 0, s>>>(a, spinLimit); break;
    default: cull_median_kernel<32><<<blocks, threads, 0, s>>>(a, spinLimit); break;
    }
    CKC(cudaGetLastError(), "cull_median");
    c->launches++;
    int hostCtl[2];
    unsigned long long culled = 0;
    CKC(cudaMemcpyAsync(hostCtl, ctl, sizeof(int) * 2, cudaMemcpyDeviceToHost, s), "d2h");
    CKC(cudaMemcpyAsync(&culled, ctl + 4, sizeof(culled), cudaMemcpyDeviceToHost, s), "d2h");
    CKC(cudaStreamSynchronize(s), "cull_median");
    if (hostCtl[1]) return sb_ctx_fail(c, SB_ERR_TIMEOUT, "cullSTData wavefront wait timed out");
    *nCulledOut = (int64_t)culled;
    return SB_OK;
}

int run_stats(sb_context* c, const CullJob& p, const CullDev* v)
{
    const int n = p.nR * p.nA;
    StatsArgs a{v->offR, v->offA, v->sigmaR, v->sigmaA, p.nR, p.nA, p.qvar};
    cull_stats_kernel<<<(n + 127) / 128, 128, 0, c->stream>>>(a);
    c->launches++;
    return sb_ctx_cuda(c, cudaGetLastError(), "cull_stats");
}

int run_smooth(sb_context* c, const CullJob& p, const CullDev* v)
{
    const int n = p.nR * p.nA;
    SmoothArgs a{v->offR, v->offA, v->type, v->sigmaR, v->sigmaA, v->offRS, v->offAS, p.nR, p.nA, p.sR, p.sA};
    if (p.lsSmooth)
        cullls_smooth_kernel<<<(n + 127) / 128, 128, 0, c->stream>>>(a);
    else
        cull_smooth_kernel<<<(n + 127) / 128, 128, 0, c->stream>>>(a);
    c->launches++;
    return sb_ctx_cuda(c, cudaGetLastError(), "cull_smooth");
}

int run_islands(sb_context* c, const CullJob& p, const CullDev* v, int64_t* nIslands, int64_t* nIslandPoints)
{
    const int n = p.nR * p.nA;
    cudaError_t e;
    int* ws = (int*)sb_ctx_buf(c, "c_isl", sizeof(int) * (size_t)n * 5 + 64, &e);
    unsigned long long* cntd = (unsigned long long*)sb_ctx_buf(c, "c_isl_cnt", 4 * sizeof(unsigned long long), &e);
    if (!ws || !cntd) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
    IslandArgs a;
    a.offRS = v->offRS;
    a.offAS = v->offAS;
    a.par = ws;
    a.minX = ws + (size_t)n;
    a.maxX = ws + 2 * (size_t)n;
    a.minY = ws + 3 * (size_t)n;
    a.maxY = ws + 4 * (size_t)n;
    a.lastRoot = ws + 5 * (size_t)n;
    a.counts = cntd;
    a.nR = p.nR;
    a.nA = p.nA;
    a.conn8 = p.connectivity != 4;
    a.thresh = p.islandThresh;
    cudaStream_t s = c->stream;
    CKC(cudaMemsetAsync(a.lastRoot, 0xff, sizeof(int), s), "memset");
    CKC(cudaMemsetAsync(a.counts, 0, 2 * sizeof(unsigned long long), s), "memset");
    const int g = (n + 255) / 256;
    isl_init_kernel<<<g, 256, 0, s>>>(a);
    isl_union_kernel<<<g, 256, 0, s>>>(a);
    isl_flatten_kernel<<<g, 256, 0, s>>>(a);
    isl_cull_kernel<<<g, 256, 0, s>>>(a);
    c->launches += 4;
    CKC(cudaGetLastError(), "cull_islands");
    unsigned long long cnt[2];
    CKC(cudaMemcpyAsync(cnt, a.counts, sizeof(cnt), cudaMemcpyDeviceToHost, s), "d2h");
    CKC(cudaStreamSynchronize(s), "cull_islands");
    *nIslands = (int64_t)cnt[0];
    *nIslandPoints = (int64_t)cnt[1];
    return SB_OK;
}

int run_sim(sb_context* c, const CullJob& p, const CullDev* v, float sign)
{
    const int n = p.nR * p.nA;
    cull_sim_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(v->offR, v->offA, v->simR, v->simA, n, sign);
    c->launches++;
    return sb_ctx_cuda(c, cudaGetLastError(), "cull_sim");
}

// Stage in, run the passes, stage out, with the context's four timing events.
template <typename In, typename F, typename Out>
int cull_run(sb_context* c, In stageIn, F body, Out stageOut)
{
    int rc;
    c->err.clear();
    c->launches = 0;
    CKC(cudaSetDevice(c->device), "cudaSetDevice");
    cudaEventRecord(c->ev[0], c->stream);
    CullDev v;
    if ((rc = stageIn(&v)) != SB_OK) return rc;
    cudaEventRecord(c->ev[1], c->stream);
    if ((rc = body(v)) != SB_OK) return rc;
    cudaEventRecord(c->ev[2], c->stream);
    if ((rc = stageOut(&v)) != SB_OK) return rc;
    cudaEventRecord(c->ev[3], c->stream);
    CKC(cudaStreamSynchronize(c->stream), "cull");
    cudaEventElapsedTime(&c->timing[0], c->ev[0], c->ev[3]);
    cudaEventElapsedTime(&c->timing[1], c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&c->timing[2], c->ev[1], c->ev[2]);
    cudaEventElapsedTime(&c->timing[3], c->ev[2], c->ev[3]);
    return SB_OK;
}

template <typename F>
int cull_entry(sb_context* c, const sb_cull_params* p, sb_cull_data* d, F body)
{
    int rc = cull_check(c, p, d);
    if (rc != SB_OK) return rc;
    return cull_run(
        c, [&](CullDev* v) { return cull_stage_in(c, p, d, v); }, body,
        [&](const CullDev* v) { return cull_stage_out(c, p, d, v); });
}

int cullls_check(sb_context* c, const sb_cullls_params* p, const sb_cullls_data* d)
{
    if (!c) return SB_ERR_ARG;
    if (!p || !d) return sb_ctx_fail(c, SB_ERR_ARG, "null params or data");
    if (p->nx <= 0 || p->ny <= 0) return sb_ctx_fail(c, SB_ERR_ARG, "empty grid");
    if ((long long)p->nx * p->ny > (1LL << 30)) return sb_ctx_fail(c, SB_ERR_ARG, "grid too large");
    if (!d->X || !d->Y || !d->type) return sb_ctx_fail(c, SB_ERR_ARG, "null input grid");
    if (p->boxSize < 0 || (p->boxSize / 2 * 2 + 1) * (p->boxSize / 2 * 2 + 1) > 32 * 32)
        return sb_ctx_fail(c, SB_ERR_UNSUPPORTED, "cull box larger than 32 x 32");
    if (!(p->nOver > 0.0)) return sb_ctx_fail(c, SB_ERR_ARG, "nOver (lstrack's NOVER) must be positive");
    if (!(p->dx > 0.0) || !(p->dy > 0.0)) return sb_ctx_fail(c, SB_ERR_ARG, "pixel sizes dx, dy must be positive");
    return SB_OK;
}

int cullls_stage_in(sb_context* c, const sb_cullls_params* p, sb_cullls_data* d, CullDev* v)
{
    const size_t n = (size_t)p->nx * p->ny, fb = n * sizeof(float);
    cudaError_t e;
    *v = CullDev{};
    if (d->onDevice) {
        v->offR = d->X; v->offA = d->Y; v->type = (uint8_t*)d->type;
        v->offRS = d->XS; v->offAS = d->YS; v->sigmaR = d->sigmaX; v->sigmaA = d->sigmaY;
    } else {
        v->offR = (float*)sb_ctx_buf(c, "c_offR", fb, &e);
        v->offA = (float*)sb_ctx_buf(c, "c_offA", fb, &e);
        v->type = (uint8_t*)sb_ctx_buf(c, "c_type", n, &e);
        if (!v->offR || !v->offA || !v->type) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
        CKC(cudaMemcpyAsync(v->offR, d->X, fb, cudaMemcpyHostToDevice, c->stream), "h2d");
        CKC(cudaMemcpyAsync(v->offA, d->Y, fb, cudaMemcpyHostToDevice, c->stream), "h2d");
        CKC(cudaMemcpyAsync(v->type, d->type, n, cudaMemcpyHostToDevice, c->stream), "h2d");
    }
    if (!d->onDevice || !v->offRS) v->offRS = (float*)sb_ctx_buf(c, "c_offRS", fb, &e);
    if (!d->onDevice || !v->offAS) v->offAS = (float*)sb_ctx_buf(c, "c_offAS", fb, &e);
    if (!d->onDevice || !v->sigmaR) v->sigmaR = (float*)sb_ctx_buf(c, "c_sigmaR", fb, &e);
    if (!d->onDevice || !v->sigmaA) v->sigmaA = (float*)sb_ctx_buf(c, "c_sigmaA", fb, &e);
    if (!v->offRS || !v->offAS || !v->sigmaR || !v->sigmaA)
        return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
    return SB_OK;
}

int cullls_stage_out(sb_context* c, const sb_cullls_params* p, sb_cullls_data* d, const CullDev* v)
{
    if (d->onDevice) return SB_OK;
    const size_t fb = (size_t)p->nx * p->ny * sizeof(float);
    cudaStream_t s = c->stream;
    CKC(cudaMemcpyAsync(d->X, v->offR, fb, cudaMemcpyDeviceToHost, s), "d2h");
    CKC(cudaMemcpyAsync(d->Y, v->offA, fb, cudaMemcpyDeviceToHost, s), "d2h");
    if (d->XS) CKC(cudaMemcpyAsync(d->XS, v->offRS, fb, cudaMemcpyDeviceToHost, s), "d2h");
    if (d->YS) CKC(cudaMemcpyAsync(d->YS, v->offAS, fb, cudaMemcpyDeviceToHost, s), "d2h");
    if (d->sigmaX) CKC(cudaMemcpyAsync(d->sigmaX, v->sigmaR, fb, cudaMemcpyDeviceToHost, s), "d2h");
    if (d->sigmaY) CKC(cudaMemcpyAsync(d->sigmaY, v->sigmaA, fb, cudaMemcpyDeviceToHost, s), "d2h");
    return SB_OK;
}

// nAttempt / nMatch of the first cullLSData pass (cullLSData.c:36-57).
int run_ls_counts(sb_context* c, const sb_cullls_params* p, const CullDev* v, sb_cullls_data* d)
{
    const long long n = (long long)p->nx * p->ny;
    cudaError_t e;
    unsigned long long* cnt = (unsigned long long*)sb_ctx_buf(c, "c_lscnt", 2 * sizeof(unsigned long long), &e);
    if (!cnt) return sb_ctx_fail(c, SB_ERR_NOMEM, "device allocation failed");
    cudaStream_t s = c->stream;
    CKC(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned long long), s), "memset");
    long long blocks = (n + 255) / 256;
    if (blocks > (long long)c->numSM * 16) blocks = (long long)c->numSM * 16;
    cullls_count_kernel<<<(int)blocks, 256, 0, s>>>(v->offR, v->offA, v->type, p->noDataMask, n, cnt);
    CKC(cudaGetLastError(), "cullls_count");
    c->launches++;
    unsigned long long h[2];
    CKC(cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, s), "d2h");
    CKC(cudaStreamSynchronize(s), "cullls_count");
    d->nMatch = (int64_t)h[0];
    d->nAttempt = (int64_t)h[1];
    return SB_OK;
}

}  // namespace

extern "C" int sb_cull(sb_context* c, const sb_cull_params* p, sb_cull_data* d)
{
    return cull_entry(c, p, d, [&](const CullDev& v) {
        int rc;
        const CullJob j = job_of(p);
        if (p->useSim && (rc = run_sim(c, j, &v, -1.0f)) != SB_OK) return rc;
        const int passes = p->nCullPasses > 0 ? p->nCullPasses : 3;
        for (int k = 0; k < passes; ++k)
            if ((rc = run_st_data(c, j, &v, &d->nCulled)) != SB_OK) return rc;
        if ((rc = run_stats(c, j, &v)) != SB_OK) return rc;
        if (p->useSim && (rc = run_sim(c, j, &v, 1.0f)) != SB_OK) return rc;
        if ((rc = run_smooth(c, j, &v)) != SB_OK) return rc;
        if (p->islandThresh > 0 && (rc = run_islands(c, j, &v, &d->nIslands, &d->nIslandPoints)) != SB_OK)
            return rc;
        return SB_OK;
    });
}

extern "C" int sb_cull_st_data(sb_context* c, const sb_cull_params* p, sb_cull_data* d)
{
    return cull_entry(c, p, d, [&](const CullDev& v) { return run_st_data(c, job_of(p), &v, &d->nCulled); });
}

extern "C" int sb_cull_stats(sb_context* c, const sb_cull_params* p, sb_cull_data* d)
{
    return cull_entry(c, p, d, [&](const CullDev& v) { return run_stats(c, job_of(p), &v); });
}

extern "C" int sb_cull_smooth(sb_context* c, const sb_cull_params* p, sb_cull_data* d)
{
    return cull_entry(c, p, d, [&](const CullDev& v) { return run_smooth(c, job_of(p), &v); });
}

extern "C" int sb_cull_islands(sb_context* c, const sb_cull_params* p, sb_cull_data* d)
{
    return cull_entry(
        c, p, d, [&](const CullDev& v) { return run_islands(c, job_of(p), &v, &d->nIslands, &d->nIslandPoints); });
}

extern "C" int sb_cullls(sb_context* c, const sb_cullls_params* p, sb_cullls_data* d)
{
    int rc = cullls_check(c, p, d);
    if (rc != SB_OK) return rc;
    return cull_run(
        c, [&](CullDev* v) { return cullls_stage_in(c, p, d, v); },
        [&](const CullDev& v) {
            int r;
            CullJob j = job_of(p);
            j.rule.slowType = v.type;
            if ((r = run_ls_counts(c, p, &v, d)) != SB_OK) return r;
            const int passes = p->nCullPasses > 0 ? p->nCullPasses : 3;
            for (int k = 0; k < passes; ++k)
                if ((r = run_st_data(c, j, &v, &d->nCulled)) != SB_OK) return r;
            if ((r = run_stats(c, j, &v)) != SB_OK) return r;
            if ((r = run_smooth(c, j, &v)) != SB_OK) return r;
            d->nIslands = d->nIslandPoints = 0;
            if (p->islandThresh > 0 && (r = run_islands(c, j, &v, &d->nIslands, &d->nIslandPoints)) != SB_OK)
                return r;
            return SB_OK;
        },
        [&](const CullDev* v) { return cullls_stage_out(c, p, d, v); });
}
