// xb_partition.cuh -- edge-balanced partition of a vertex frontier.
//
// For frontier-driven kernels whose per-vertex work is its adjacency (the
// multi-source SSSP relax rounds, the matching forest expansion): an
// exclusive scan of the frontier's degrees gives every frontier entry its
// first edge in the round's edge order (eoff) and its column-index position
// minus that (ebase); the round's edges are then cut into chunks of kChunk
// consecutive edges, and chunk_first[c] names the entry that owns the first
// edge of chunk c.  A consumer takes one chunk per warp: lane l of step it
// handles chunk edge 32 * it + l (consecutive column-index reads), and the
// owner of an edge is the number of entries that start at or before it --
// a popcount over a 256-bit mask of entry starts.  Every frontier entry must
// have at least one edge, so a chunk spans at most kChunk + 1 entries.
#pragma once

#include <cstdint>

namespace xbp {
namespace {

constexpr int kThreads = 256;                 // scan blocks
constexpr int kItems = 8;                     // per thread
constexpr int kTile = kThreads * kItems;      // frontier entries per scan tile
constexpr int kChunk = 32 * kItems;           // frontier edges per consumer chunk (one warp)


// Block-wide exclusive scan of one int64 per thread (blockDim.x == kThreads
// or 1024); the block total goes to *total.
__device__ __forceinline__ int64_t block_scan_i64(int64_t x, int64_t* total) {
  __shared__ int64_t s_w[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  int64_t incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_w[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int64_t t = lane < nwarps ? s_w[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < nwarps) s_w[lane] = t;
  }
  __syncthreads();
  const int64_t excl = (warp > 0 ? s_w[warp - 1] : 0) + incl - x;
  *total = s_w[nwarps - 1];
  __syncthreads();  // s_w is reused by the next call
  return excl;
}

// Scan phase 1: the degree sum of each tile of kTile frontier entries.
template <typename OffT>
__global__ void __launch_bounds__(kThreads) k_lb_tile_sums(const int32_t* __restrict__ list,
                                                           const int32_t* __restrict__ cnt_p,
                                                           const OffT* __restrict__ ro, int64_t* tsum) {
  const int32_t cnt = *cnt_p;
  if ((int64_t)blockIdx.x * kTile >= cnt) return;  // grids may be sized for the largest frontier
  const int64_t i0 = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kItems;
  int64_t sum = 0;
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    const int64_t i = i0 + j;
    if (i < cnt) {
      const int32_t u = list[i];
      sum += (int64_t)(ro[u + 1] - ro[u]);
    }
  }
  int64_t total;
  block_scan_i64(sum, &total);
  if (threadIdx.x == 0) tsum[blockIdx.x] = total;
}

// Scan phase 2 (one block of 1024): tile offsets in place, the round's edge
// total and chunk count.
__global__ void __launch_bounds__(1024) k_lb_tile_scan(int64_t* tsum, const int32_t* __restrict__ cnt_p,
                                                       int64_t* edges, int64_t* nchunks,
                                                       unsigned long long* relaxed) {
  const int32_t ntiles = (*cnt_p + kTile - 1) / kTile;
  int64_t carry = 0;
  for (int32_t b0 = 0; b0 < ntiles; b0 += blockDim.x) {
    const int32_t b = b0 + threadIdx.x;
    const int64_t x = b < ntiles ? tsum[b] : 0;
    int64_t total;
    const int64_t ex = block_scan_i64(x, &total);
    if (b < ntiles) tsum[b] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) {
    *edges = carry;
    *nchunks = (carry + kChunk - 1) / kChunk;
    *relaxed += (unsigned long long)carry;
  }
}

// Scan phase 3: per frontier entry its first edge in the round's edge order
// (eoff) and its column-index position minus that (ebase); for every chunk
// boundary inside its edges, the owner's index (chunk_first).
template <typename OffT>
__global__ void __launch_bounds__(kThreads) k_lb_offsets(const int32_t* __restrict__ list,
                                                         const int32_t* __restrict__ cnt_p,
                                                         const OffT* __restrict__ ro,
                                                         const int64_t* __restrict__ tsum, int64_t* eoff,
                                                         int64_t* ebase, int32_t* chunk_first) {
  const int32_t cnt = *cnt_p;
  if ((int64_t)blockIdx.x * kTile >= cnt) return;
  const int64_t i0 = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kItems;
  int64_t deg[kItems], beg[kItems];
  int64_t sum = 0;
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    const int64_t i = i0 + j;
    deg[j] = beg[j] = 0;
    if (i < cnt) {
      const int32_t u = list[i];
      beg[j] = (int64_t)ro[u];
      deg[j] = (int64_t)ro[u + 1] - beg[j];
    }
    sum += deg[j];
  }
  int64_t total;
  int64_t off = block_scan_i64(sum, &total) + tsum[blockIdx.x];
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    const int64_t i = i0 + j;
    if (i < cnt) {
      eoff[i] = off;
      ebase[i] = beg[j] - off;
      for (int64_t c = (off + kChunk - 1) / kChunk; c * kChunk < off + deg[j]; c++) chunk_first[c] = (int32_t)i;
    }
    off += deg[j];
  }
}

// All three phases in one block (kThreads threads) for a frontier of at
// most kTile entries: the common case of a round's first and last levels,
// where launches, not bytes, are the cost.
template <typename OffT>
__global__ void __launch_bounds__(kThreads) k_lb_single(const int32_t* __restrict__ list,
                                                        const int32_t* __restrict__ cnt_p,
                                                        const OffT* __restrict__ ro, int64_t* eoff, int64_t* ebase,
                                                        int32_t* chunk_first, int64_t* edges, int64_t* nchunks,
                                                        unsigned long long* relaxed) {
  const int32_t cnt = *cnt_p;
  const int64_t i0 = (int64_t)threadIdx.x * kItems;
  int64_t deg[kItems], beg[kItems];
  int64_t sum = 0;
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    const int64_t i = i0 + j;
    deg[j] = beg[j] = 0;
    if (i < cnt) {
      const int32_t u = list[i];
      beg[j] = (int64_t)ro[u];
      deg[j] = (int64_t)ro[u + 1] - beg[j];
    }
    sum += deg[j];
  }
  int64_t total;
  int64_t off = block_scan_i64(sum, &total);
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    const int64_t i = i0 + j;
    if (i < cnt) {
      eoff[i] = off;
      ebase[i] = beg[j] - off;
      for (int64_t c = (off + kChunk - 1) / kChunk; c * kChunk < off + deg[j]; c++) chunk_first[c] = (int32_t)i;
    }
    off += deg[j];
  }
  if (threadIdx.x == 0) {
    *edges = total;
    *nchunks = (total + kChunk - 1) / kChunk;
    *relaxed += (unsigned long long)total;
  }
}

}  // namespace
}  // namespace xbp
