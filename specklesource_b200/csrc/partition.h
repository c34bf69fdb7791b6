// partition.h -- ordered (stable) partition of a list by a small integer key.
//
// Items i in [0, n) with key[i] in [0, K) are written to out[] grouped by key
// (key 0 first) and in increasing i within a key; items with key < 0 are
// dropped.  out[pos] = val[i], or i when val is null.  Three launches: per-tile
// key counts, one-CTA scan of the counts, and the scatter (ranks from warp
// match masks).  The order is deterministic, so a raster-ordered input stays
// raster-ordered, which keeps the window sweep of the matching kernels inside
// L2.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

namespace sbk {

constexpr int PART_TILE = 1024;  // items per tile (one per thread)
constexpr int PART_KMAX = 32;    // largest number of keys (one warp of part_write_kernel per key)

// ints of device scratch launch_partition needs for n items and K keys
size_t partition_scratch_ints(int n, int K);
// Offset (in ints) into the scratch of keyOff[0..K]: keyOff[k] = first output
// position of key k, keyOff[K] = number of items kept.
size_t partition_keyoff_at(int n, int K);

cudaError_t launch_partition(const int* key, const int* val, int n, int K, int* out, int* scratch,
                             cudaStream_t st);

}  // namespace sbk
