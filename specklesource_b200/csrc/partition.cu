// partition.cu -- ordered (stable) partition by key; see partition.h.
#include <cuda_runtime.h>

#include "partition.h"

namespace sbk {

static int part_tiles(int n) { return (n + PART_TILE - 1) / PART_TILE; }

size_t partition_scratch_ints(int n, int K)
{
    // tileCnt[t][k] and tileOff[t][k], then keyOff[K + 1]
    return (size_t)2 * part_tiles(n) * K + K + 1;
}
size_t partition_keyoff_at(int n, int K) { return (size_t)2 * part_tiles(n) * K; }

__global__ void __launch_bounds__(PART_TILE) part_count_kernel(const int* __restrict__ key, int n, int K,
                                                               int* __restrict__ tileCnt)
{
    __shared__ int h[PART_KMAX];
    if (threadIdx.x < PART_KMAX) h[threadIdx.x] = 0;
    __syncthreads();
    const int i = blockIdx.x * PART_TILE + threadIdx.x;
    const int k = i < n ? key[i] : -1;
    if (k >= 0 && k < K) atomicAdd(&h[k], 1);
    __syncthreads();
    if (threadIdx.x < K) tileCnt[(size_t)blockIdx.x * K + threadIdx.x] = h[threadIdx.x];
}

// One CTA of 1024 threads: exclusive scan over tiles, key by key.
__global__ void __launch_bounds__(1024) part_scan_kernel(const int* __restrict__ tileCnt, int nTiles, int K,
                                                         int* __restrict__ tileOff, int* __restrict__ keyOff)
{
    __shared__ int ws[32];
    __shared__ int total;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int base = 0;  // running first position of the current key
    for (int k = 0; k < K; ++k) {
        if (tid == 0) keyOff[k] = base;
        int run = 0;
        for (int t0 = 0; t0 < nTiles; t0 += 1024) {
            const int t = t0 + tid;
            const int v = t < nTiles ? tileCnt[(size_t)t * K + k] : 0;
            int x = v;  // inclusive warp scan
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (lane == 31) ws[warp] = x;
            __syncthreads();
            if (warp == 0) {
                int s = ws[lane];
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, s, o);
                    if (lane >= o) s += y;
                }
                ws[lane] = s;  // inclusive over warps
                if (lane == 31) total = s;
            }
            __syncthreads();
            const int excl = x - v + (warp > 0 ? ws[warp - 1] : 0);
            if (t < nTiles) tileOff[(size_t)t * K + k] = run + excl;
            run += total;
            __syncthreads();
        }
        base += run;
    }
    if (tid == 0) keyOff[K] = base;
}

__global__ void __launch_bounds__(PART_TILE) part_write_kernel(const int* __restrict__ key,
                                                               const int* __restrict__ val, int n, int K,
                                                               const int* __restrict__ tileOff,
                                                               const int* __restrict__ keyOff, int* __restrict__ out)
{
    __shared__ int wc[PART_KMAX][32];  // [key][warp]: count, then exclusive prefix over warps
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int e = tid; e < PART_KMAX * 32; e += PART_TILE) wc[e / 32][e % 32] = 0;
    __syncthreads();
    const int i = blockIdx.x * PART_TILE + tid;
    int k = i < n ? key[i] : -1;
    if (k >= K) k = -1;
    const unsigned same = __match_any_sync(0xffffffffu, k);
    const int rank = __popc(same & ((1u << lane) - 1u));
    if (k >= 0 && rank == 0) wc[k][warp] = __popc(same);
    __syncthreads();
    if (warp < K) {  // warp kk scans the 32 warp counts of key kk
        const int v = wc[warp][lane];
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        wc[warp][lane] = x - v;
    }
    __syncthreads();
    if (k >= 0) {
        const int pos = keyOff[k] + tileOff[(size_t)blockIdx.x * K + k] + wc[k][warp] + rank;
        out[pos] = val ? val[i] : i;
    }
}

cudaError_t launch_partition(const int* key, const int* val, int n, int K, int* out, int* scratch, cudaStream_t st)
{
    if (K < 1 || K > PART_KMAX || n < 0) return cudaErrorInvalidValue;
    const int nt = part_tiles(n);
    int* tileCnt = scratch;
    int* tileOff = scratch + (size_t)nt * K;
    int* keyOff = scratch + partition_keyoff_at(n, K);
    if (nt == 0) return cudaMemsetAsync(keyOff, 0, sizeof(int) * (K + 1), st);
    part_count_kernel<<<nt, PART_TILE, 0, st>>>(key, n, K, tileCnt);
    part_scan_kernel<<<1, 1024, 0, st>>>(tileCnt, nt, K, tileOff, keyOff);
    part_write_kernel<<<nt, PART_TILE, 0, st>>>(key, val, n, K, tileOff, keyOff, out);
    return cudaGetLastError();
}

}  // namespace sbk
