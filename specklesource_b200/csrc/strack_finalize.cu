// strack_finalize.cu -- record initialisation, amplitude-try candidate
// selection, the azShift carry-over fill, and the finalize kernel that writes
// the .dr/.da/.cc/.azd/.mt grids (speckleTrack.c:300-323).
#include <cuda_runtime.h>

#include "strack_finalize.h"

namespace sbk {

__global__ void rec_init_kernel(PointRec* rec, int n)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    PointRec r;
    r.cMax[0] = r.cMax[1] = r.cMax[2] = 0.0;
    r.iMax[0] = r.iMax[1] = r.iMax[2] = 0;
    r.jMax[0] = r.jMax[1] = r.jMax[2] = 0;
    r.azd = 0.0f;  // aZDefocus is never initialised by the reference: pinned to 0
    r.azset = -1;
    r.flags = 0;
    r.azUsed = 0;
    rec[p] = r;
}

// key[p] = 0 for the points whose next missing try is `stage`, else -1 (the
// list is then built in raster order by the ordered partition).
__global__ void select_stage_kernel(const PointPlan* plan, const PointRec* rec, int n, WalkParams w, int stage,
                                    int* key)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const WalkOut o = strack_walk(plan[p], rec[p], w);
    key[p] = o.stage_next == stage ? 0 : -1;
}

// azShift in effect at each point = the last value set at or before it in
// raster order (trackPar->azShift carries over between points; initial 0).
// Single CTA: chunked block scan over the grid.
__global__ void az_fill_kernel(const PointRec* rec, int n, int* azEff)
{
    __shared__ int carry;
    __shared__ int lastIdx[1024];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += blockDim.x) {
        const int p = base + threadIdx.x;
        const int v = (p < n) ? rec[p].azset : -1;
        // inclusive max-scan of "index of the last set element"
        lastIdx[threadIdx.x] = (v >= 0) ? (int)threadIdx.x : -1;
        __syncthreads();
        for (int off = 1; off < (int)blockDim.x; off <<= 1) {
            int t = (threadIdx.x >= (unsigned)off) ? lastIdx[threadIdx.x - off] : -1;
            __syncthreads();
            if (t > lastIdx[threadIdx.x]) lastIdx[threadIdx.x] = t;
            __syncthreads();
        }
        const int li = lastIdx[threadIdx.x];
        if (p < n) azEff[p] = (li >= 0) ? rec[base + li].azset : carry;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) {
            const int lastAll = lastIdx[blockDim.x - 1];
            if (lastAll >= 0 && base + lastAll < n) carry = rec[base + lastAll].azset;
        }
        __syncthreads();
    }
}

__global__ void finalize_kernel(const PointPlan* plan, const PointRec* rec, int n, WalkParams w, int scaleFactor,
                                float* offR, float* offA, float* corr, float* azd, uint8_t* type,
                                unsigned long long* stats, const int* pairOf)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (pairOf) stats += 8 * pairOf[p];  // batched calls: statistics per pair
    const PointPlan pl = plan[p];
    const PointRec r = rec[p];
    const WalkOut o = strack_walk(pl, r, w);
    const int mask = (pl.flags & PF_MASK) != 0;
    float rShift, aShift;
    if (o.good && mask) {
        rShift = (float)(pl.r2 - pl.r1) - o.rShift1;
        aShift = (float)(pl.a2 - pl.a1) - o.aShift1;
    } else {
        rShift = (float)-SB_LARGEINT;
        aShift = (float)-SB_LARGEINT;
    }
    float oR = rShift, oA = aShift;
    if (rShift > -100000) {
        oR *= (float)scaleFactor;
        oA *= (float)scaleFactor;
    }
    offR[p] = oR;
    offA[p] = oA;
    corr[p] = (float)o.cMax;
    if (azd) azd[p] = r.azd;
    type[p] = (uint8_t)o.type;
    // statistics (printLineSummary)
    const int isC = o.good && o.type == SB_CMATCH;
    const int isA = o.good && o.type == SB_AMPMATCH;
    const int isL = o.good && o.type == SB_AMPMATCHLARGE;
    const int fail = !(o.good && mask) && o.haveData;
    if (isC) atomicAdd(&stats[0], 1ull);
    if (isA) atomicAdd(&stats[1], 1ull);
    if (isL) atomicAdd(&stats[2], 1ull);
    if (fail) atomicAdd(&stats[3], 1ull);
    if (o.nSkip) atomicAdd(&stats[4], (unsigned long long)o.nSkip);
}

// Device plan of the grid for a polynomial initial shift, where every point is
// independent: findImage2Pos (speckleTrack.c:810-847, the polyShift branch),
// maskValue (:1951-1965) and boundsCheck (:1822-1828) for the three windows.
// Products and sums are rounded separately (no fused multiply-add), as on the
// host.  key[p] = 0 for complex candidates, else -1.
__global__ void plan_poly_kernel(PlanArgs a, PointPlan* plan, int* key)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.nR * a.nA) return;
    const int i = p / a.nR, j = p % a.nR;
    const int a1 = a.aStart + i * a.deltaA - a.wA / 2;
    const int r1 = a.rStart + j * a.deltaR - a.wR / 2;
    const double sc = (double)a.scaleFactor;
    const double rr = __dmul_rn((double)r1, sc), aa = __dmul_rn((double)a1, sc);
    double rShift = __dadd_rn(__dadd_rn(a.rPoly[0], __dmul_rn(rr, a.rPoly[1])), __dmul_rn(aa, a.rPoly[2]));
    double aShift = __dadd_rn(__dadd_rn(a.aPoly[0], __dmul_rn(rr, a.aPoly[1])), __dmul_rn(aa, a.aPoly[2]));
    rShift = __ddiv_rn(rShift, sc);
    aShift = __ddiv_rn(aShift, sc);
    const int r2 = (rShift >= 0) ? r1 + (int)__dadd_rn(rShift, 0.5) : r1 + (int)__dsub_rn(rShift, 0.5);
    const int a2 = (aShift >= 0) ? a1 + (int)__dadd_rn(aShift, 0.5) : a1 + (int)__dsub_rn(aShift, 0.5);
    int maskVal = 1;
    if (a.mask) {
        const int ia1 = (a1 * a.scaleFactor + a.wA / 2 - a.mA0) / a.mNal;
        const int ir1 = (r1 * a.scaleFactor + a.wR / 2 - a.mR0) / a.mNrl;
        if (ia1 < 0 || ia1 >= a.mNa || ir1 < 0 || ir1 >= a.mNr)
            maskVal = 0;
        else
            maskVal = (int)(signed char)a.mask[(size_t)ia1 * a.mNr + ir1];
        maskVal = maskVal < 1 ? maskVal : 1;
    }
    PointPlan pl;
    pl.r1 = r1;
    pl.a1 = a1;
    pl.r2 = r2;
    pl.a2 = a2;
    pl.flags = maskVal > 0 ? PF_MASK : 0u;
    auto inb = [](int r, int az, int wr, int wa, int sR, int sA) {
        return r > 0 && (r + wr) < sR && az > 0 && (az + wa) < sA;
    };
    if (inb(r1, a1, a.wR, a.wA, a.nr1, a.na1) && inb(r2, a2, a.wR, a.wA, a.nr2, a.na2)) pl.flags |= PF_CBOUND;
    for (int s = 1; s <= 2; ++s) {
        const int a1a = a.aStart + i * a.deltaA - a.wA / 2 * s;
        const int r1a = a.rStart + j * a.deltaR - a.wR / 2 * s;
        const int r2a = r1a + (r2 - r1), a2a = a1a + (a2 - a1);
        if (inb(r1a, a1a, a.wRa * s, a.wAa * s, a.nr1, a.na1) && inb(r2a, a2a, a.wRa * s, a.wAa * s, a.nr2, a.na2))
            pl.flags |= (s == 1 ? PF_SBOUND : PF_LBOUND);
    }
    pl.a1 += a.a1Off;  // bounds are checked in the pair's own coordinates
    pl.a2 += a.a2Off;
    plan[p] = pl;
    int kv = a.keyValue;
    if (a.stripPx > 0) kv = min(max(r1, 0) / a.stripPx, SB_BANDS_MAX - 1);
    key[p] = ((pl.flags & PF_CBOUND) && (pl.flags & PF_MASK) && a.noComplex == 0) ? kv : -1;
    if (a.pairOf) a.pairOf[p] = a.pairId;
}

cudaError_t launch_plan_poly(const PlanArgs& a, PointPlan* plan, int* key, cudaStream_t st)
{
    const int n = a.nR * a.nA;
    plan_poly_kernel<<<(n + 255) / 256, 256, 0, st>>>(a, plan, key);
    return cudaGetLastError();
}

// Band of a complex-list point: the last image band (rows[i] rows each) its
// two W x W windows reach; rows[i] = 0 for an image already on the device.
__device__ __forceinline__ int point_band(const PointPlan& pl, int W, int rows1, int rows2, int nb)
{
    int b = 0;
    if (rows1 > 0) b = max(b, (pl.a1 + W - 1) / rows1);
    if (rows2 > 0) b = max(b, (pl.a2 + W - 1) / rows2);
    return min(max(b, 0), nb - 1);
}

// Band key of every complex-list entry (for the ordered partition by band).
__global__ void band_key_kernel(const PointPlan* plan, const int* list, int n, int W, int rows1, int rows2, int nb,
                                int* bandOf)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) bandOf[i] = point_band(plan[list[i]], W, rows1, rows2, nb);
}

cudaError_t launch_band_key(const PointPlan* plan, const int* list, int n, int W, int rows1, int rows2, int nb,
                            int* bandOf, cudaStream_t st)
{
    if (nb < 1 || nb > SB_BANDS_MAX) return cudaErrorInvalidValue;
    if (n == 0) return cudaSuccess;
    band_key_kernel<<<(n + 255) / 256, 256, 0, st>>>(plan, list, n, W, rows1, rows2, nb, bandOf);
    return cudaGetLastError();
}

cudaError_t launch_rec_init(PointRec* rec, int n, cudaStream_t st)
{
    rec_init_kernel<<<(n + 255) / 256, 256, 0, st>>>(rec, n);
    return cudaGetLastError();
}
cudaError_t launch_select(const PointPlan* plan, const PointRec* rec, int n, const WalkParams& w, int stage,
                          int* key, cudaStream_t st)
{
    select_stage_kernel<<<(n + 255) / 256, 256, 0, st>>>(plan, rec, n, w, stage, key);
    return cudaGetLastError();
}
cudaError_t launch_az_fill(const PointRec* rec, int n, int* azEff, cudaStream_t st)
{
    az_fill_kernel<<<1, 1024, 0, st>>>(rec, n, azEff);
    return cudaGetLastError();
}
cudaError_t launch_finalize(const PointPlan* plan, const PointRec* rec, int n, const WalkParams& w, int scaleFactor,
                            float* offR, float* offA, float* corr, float* azd, uint8_t* type,
                            unsigned long long* stats, cudaStream_t st, const int* pairOf)
{
    if (n <= 0) return cudaSuccess;
    finalize_kernel<<<(n + 255) / 256, 256, 0, st>>>(plan, rec, n, w, scaleFactor, offR, offA, corr, azd, type,
                                                     stats, pairOf);
    return cudaGetLastError();
}

}  // namespace sbk
