// xb_kernels.cuh -- sm_100a device code of the multi-source traversal.
//
// Data layout in HBM (one traversal pass = NW words of B bits per vertex,
// B*NW sources traversed together):
//   seen[v*NW+i]      bits of the sources that have reached v
//   F[v*NW+i]         bits newly reached at the current level (the frontier)
//   N[v*NW+i]         bits reached at the next level (all zero between levels
//                     except at next-frontier vertices)
//   plane[j][v*NW+i]  bit j of the level of (source, v), bit-sliced: the level
//                     of source s at v is sum_j bit_s(plane[j][v]) << j
//   FL/NL             frontier vertex lists, split by degree (light / heavy)
//
// One level step (level L -> L+1) is either
//   push:  every frontier vertex v ORs F[v] & ~seen[w] into N[w] for each
//          neighbour w (atomicOr), the first toucher of w appends it to a list,
//          then a finalize pass folds N into seen/planes and buckets the list;
//   pull:  every vertex w with unseen live bits ORs F[u] over its neighbours u
//          (no atomics; edge-flat warp tiles with a segmented OR scan), writes
//          N[w], seen, planes and appends w by warp-ballot compaction.
// Both are the expand step of the reference's alternating-forest engine
// (ExpandAlternatingForest, apps/xb/src/xblsm_gpu/xblossom_gpu_engine_10.cu:270-359;
// parExpand_pro_all apps/xb/src/xblsm_cpu/par_pro_pernode.cu:178-234) with the
// claim replaced by an order-free bit OR, so levels are exact regardless of
// schedule.
//
// Parents are resolved after the search by the table pass: for vertex v at
// level L for source s, parent = smallest-id neighbour u with level L-1.  Two
// adjacent reached vertices differ in level by at most one, so level mod 4
// (planes 0 and 1) decides "u is one level up"; the bit-sliced compare does
// it for all B sources of a word at once.  The pass transposes a 32-vertex x
// B-source tile in shared memory and writes whole 128-byte rows of the
// source-major level and parent tables with streaming stores.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace xbk {

template <typename W>
struct WB;
template <>
struct WB<unsigned int> {
  static constexpr int bits = 32;
};
template <>
struct WB<unsigned long long> {
  static constexpr int bits = 64;
};

__device__ __forceinline__ int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }
__device__ __forceinline__ int popc(unsigned int x) { return __popc(x); }
__device__ __forceinline__ int popc(unsigned long long x) { return __popcll(x); }
__device__ __forceinline__ int ffs0(unsigned int x) { return __ffs(x) - 1; }
__device__ __forceinline__ int ffs0(unsigned long long x) { return __ffsll(x) - 1; }

template <typename W>
__device__ __forceinline__ W shfl_up(W x, int d) {
  return __shfl_up_sync(0xffffffffu, x, d);
}
template <typename W>
__device__ __forceinline__ W shfl_down(W x, int d) {
  return __shfl_down_sync(0xffffffffu, x, d);
}
template <typename W>
__device__ __forceinline__ W shfl_idx(W x, int l) {
  return __shfl_sync(0xffffffffu, x, l);
}

// Counters of one level (device).  live[i] = OR of the frontier words.
struct LevelCtr {
  int32_t n_light;
  int32_t n_heavy;
  int32_t n_touched;
  int32_t pad;
  unsigned long long edges;  // sum of degrees of the frontier
  unsigned long long live[4];
};

// Counters of one batch (device).
struct BatchCtr {
  unsigned long long reached;
  unsigned long long edges_traversed;
  unsigned long long edges_scanned;
  unsigned long long vertices_scanned;
  unsigned long long vertices_swept;
  unsigned long long parent_edges;
  long long m_unfinished;  // sum of degrees of vertices not reached by every source
  int32_t err;
  int32_t pad;
};

struct Ctrs {
  LevelCtr lv[2];
  BatchCtr b;
};

template <typename W, int NW>
struct Masks {
  W w[NW];
};

// Lists of one frontier: light (deg <= heavy) and heavy vertices.
struct Lists {
  int32_t* light;
  int32_t* heavy;
};

template <typename OffT>
__device__ __forceinline__ int64_t deg_of(const OffT* ro, int32_t v) {
  return (int64_t)ro[v + 1] - (int64_t)ro[v];
}

// Warp-aggregated append of `flag` lanes' values to list[*count].  All 32
// lanes must call it.
__device__ __forceinline__ void warp_append(bool flag, int32_t value, int32_t* list, int32_t* count) {
  const unsigned bal = __ballot_sync(0xffffffffu, flag);
  if (bal == 0) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(bal) - 1;
  int32_t base = 0;
  if (lane == leader) base = atomicAdd(count, __popc(bal));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (flag) list[base + __popc(bal & ((1u << lane) - 1u))] = value;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long x) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
  return x;
}
__device__ __forceinline__ long long warp_sum_i64(long long x) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
  return x;
}
template <typename W>
__device__ __forceinline__ W warp_or(W x) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) x |= __shfl_xor_sync(0xffffffffu, x, d);
  return x;
}

// Records a newly reached vertex (all lanes call; `has` marks lanes that own
// one): folds new bits into seen and the level planes, updates the counters
// and appends the vertex to the next frontier's light/heavy list.
template <typename W, int NW, typename OffT>
__device__ __forceinline__ void commit_new(bool has, int32_t w, const W (&nw)[NW], const W (&sw)[NW],
                                           int64_t dg, int level, W* seen, W* planes, int64_t plane_stride,
                                           const Masks<W, NW>& active, int heavy, Lists nl, LevelCtr* nctr,
                                           BatchCtr* bc) {
  int cnt = 0;
  bool fin_now = false;
  if (has) {
    bool full = true;
#pragma unroll
    for (int i = 0; i < NW; i++) {
      const W s2 = sw[i] | nw[i];
      if (nw[i]) {
        seen[(int64_t)w * NW + i] = s2;
        for (int j = 0; (level >> j) != 0; j++)
          if ((level >> j) & 1) planes[j * plane_stride + (int64_t)w * NW + i] |= nw[i];
      }
      cnt += popc(nw[i]);
      full = full && (s2 == active.w[i]);
    }
    fin_now = full;
  }
  const bool light = has && dg <= heavy;
  const bool hv = has && dg > heavy;
  warp_append(light, w, nl.light, &nctr->n_light);
  warp_append(hv, w, nl.heavy, &nctr->n_heavy);
  unsigned long long e_tr = has ? (unsigned long long)dg * (unsigned long long)cnt : 0ull;
  unsigned long long rch = (unsigned long long)cnt;
  unsigned long long fe = has ? (unsigned long long)dg : 0ull;
  long long fin = fin_now ? -(long long)dg : 0ll;
  e_tr = warp_sum_u64(e_tr);
  rch = warp_sum_u64(rch);
  fe = warp_sum_u64(fe);
  fin = warp_sum_i64(fin);
  W lv[NW];
#pragma unroll
  for (int i = 0; i < NW; i++) lv[i] = warp_or<W>(has ? nw[i] : (W)0);
  if ((threadIdx.x & 31) == 0) {
    if (rch) {
      atomicAdd(&bc->reached, rch);
      atomicAdd(&bc->edges_traversed, e_tr);
      atomicAdd(&nctr->edges, fe);
#pragma unroll
      for (int i = 0; i < NW; i++)
        if (lv[i]) atomicOr(&nctr->live[i], (unsigned long long)lv[i]);
    }
    if (fin) atomicAdd((unsigned long long*)&bc->m_unfinished, (unsigned long long)fin);
  }
}

// ---------------------------------------------------------------------------
// Batch initialisation: one block; thread t owns source slot t.
template <typename W, int NW, typename OffT>
__global__ void k_init_batch(const int32_t* __restrict__ src, int kb, const OffT* __restrict__ ro, W* F,
                             W* seen, Masks<W, NW> active, int heavy, Lists fl, Ctrs* ctr) {
  constexpr int B = WB<W>::bits;
  const int t = threadIdx.x;
  int32_t v = -1;
  if (t < kb) {
    v = src[t];
    const W bit = (W)1 << (t % B);
    atomicOr(&F[(int64_t)v * NW + t / B], bit);
    atomicOr(&seen[(int64_t)v * NW + t / B], bit);
  }
  __syncthreads();
  bool first = t < kb;
  if (first)
    for (int t2 = 0; t2 < t; t2++)
      if (src[t2] == v) {
        first = false;
        break;
      }
  W nw[NW], sw[NW];
#pragma unroll
  for (int i = 0; i < NW; i++) {
    nw[i] = first ? F[(int64_t)v * NW + i] : (W)0;
    sw[i] = 0;  // seen already holds the bits; commit_new must not add planes (level 0)
  }
  const int64_t dg = first ? deg_of(ro, v) : 0;
  // level 0: no plane bits; commit_new with level 0 only counts and appends.
  // seen was set above, so pass seen-before = 0 and a dummy seen pointer write
  // of the same value is harmless.
  commit_new<W, NW, OffT>(first, v, nw, sw, dg, 0, seen, seen, 0, active, heavy, fl, &ctr->lv[0],
                          &ctr->b);
}

// ---------------------------------------------------------------------------
// Push, light frontier vertices: one warp per vertex.
// NW == 1: the lane whose atomicOr turns N[w] from 0 to non-zero appends w.
// NW > 1: first toucher decided by an epoch stamp per vertex.
template <typename W, int NW, typename OffT>
__global__ void k_push_light(const int32_t* __restrict__ list, const int32_t* __restrict__ count,
                             const OffT* __restrict__ ro, const int32_t* __restrict__ ci, W* F,
                             const W* __restrict__ seen, W* N, int32_t* stamp, int32_t epoch,
                             int32_t* touched, Ctrs* ctr, int cur) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int32_t cnt = *count;
  LevelCtr* nctr = &ctr->lv[cur ^ 1];
  unsigned long long scanned = 0, vcount = 0;
  for (int64_t idx = warp; idx < cnt; idx += nwarps) {
    const int32_t v = list[idx];
    vcount++;
    W f[NW];
#pragma unroll
    for (int i = 0; i < NW; i++) f[i] = F[(int64_t)v * NW + i];
    __syncwarp();
    if (lane < NW) F[(int64_t)v * NW + lane] = 0;
    const int64_t beg = ro[v], end = ro[v + 1];
    scanned += (unsigned long long)(end - beg);
    for (int64_t base = beg; base < end; base += 32) {
      const int64_t e = base + lane;
      bool app = false;
      int32_t w = 0;
      if (e < end) {
        w = __ldg(&ci[e]);
        bool added = false;
#pragma unroll
        for (int i = 0; i < NW; i++) {
          const W m = f[i] & ~seen[(int64_t)w * NW + i];
          if (m) {
            const W cur_n = N[(int64_t)w * NW + i];
            if ((cur_n & m) != m) {
              const W old = atomicOr(&N[(int64_t)w * NW + i], m);
              if (NW == 1) {
                app = (old == 0);
              } else if ((old & m) != m) {
                added = true;
              }
            }
          }
        }
        if (NW > 1 && added) app = atomicExch(&stamp[w], epoch) != epoch;
      }
      warp_append(app, w, touched, &nctr->n_touched);
    }
  }
  if (lane == 0 && vcount) {
    atomicAdd(&ctr->b.edges_scanned, scanned);
    atomicAdd(&ctr->b.vertices_scanned, vcount);
  }
}

// Push, heavy frontier vertices: one block per vertex.
template <typename W, int NW, typename OffT>
__global__ void k_push_heavy(const int32_t* __restrict__ list, const int32_t* __restrict__ count,
                             const OffT* __restrict__ ro, const int32_t* __restrict__ ci, W* F,
                             const W* __restrict__ seen, W* N, int32_t* stamp, int32_t epoch,
                             int32_t* touched, Ctrs* ctr, int cur) {
  const int32_t cnt = *count;
  LevelCtr* nctr = &ctr->lv[cur ^ 1];
  for (int64_t idx = blockIdx.x; idx < cnt; idx += gridDim.x) {
    const int32_t v = list[idx];
    W f[NW];
#pragma unroll
    for (int i = 0; i < NW; i++) f[i] = F[(int64_t)v * NW + i];
    __syncthreads();
    if (threadIdx.x < NW) F[(int64_t)v * NW + threadIdx.x] = 0;
    const int64_t beg = ro[v], end = ro[v + 1];
    if (threadIdx.x == 0) {
      atomicAdd(&ctr->b.edges_scanned, (unsigned long long)(end - beg));
      atomicAdd(&ctr->b.vertices_scanned, 1ull);
    }
    for (int64_t base = beg; base < end; base += blockDim.x) {
      const int64_t e = base + threadIdx.x;
      bool app = false;
      int32_t w = 0;
      if (e < end) {
        w = __ldg(&ci[e]);
        bool added = false;
#pragma unroll
        for (int i = 0; i < NW; i++) {
          const W m = f[i] & ~seen[(int64_t)w * NW + i];
          if (m) {
            const W cur_n = N[(int64_t)w * NW + i];
            if ((cur_n & m) != m) {
              const W old = atomicOr(&N[(int64_t)w * NW + i], m);
              if (NW == 1) {
                app = (old == 0);
              } else if ((old & m) != m) {
                added = true;
              }
            }
          }
        }
        if (NW > 1 && added) app = atomicExch(&stamp[w], epoch) != epoch;
      }
      warp_append(app, w, touched, &nctr->n_touched);
    }
    __syncthreads();
  }
}

// After a push: fold N into seen/planes for every touched vertex, bucket the
// next frontier.
template <typename W, int NW, typename OffT>
__global__ void k_push_finalize(const int32_t* __restrict__ touched, const OffT* __restrict__ ro, const W* N,
                                W* seen, W* planes, int64_t plane_stride, int level, Masks<W, NW> active,
                                int heavy, Lists nl, Ctrs* ctr, int cur) {
  LevelCtr* nctr = &ctr->lv[cur ^ 1];
  const int32_t cnt = nctr->n_touched;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < cnt; base += stride) {
    const int64_t idx = base + threadIdx.x;
    const bool has = idx < cnt;
    int32_t w = 0;
    W nw[NW], sw[NW];
    int64_t dg = 0;
    if (has) {
      w = touched[idx];
#pragma unroll
      for (int i = 0; i < NW; i++) {
        nw[i] = N[(int64_t)w * NW + i];
        sw[i] = seen[(int64_t)w * NW + i];
      }
      dg = deg_of(ro, w);
    } else {
#pragma unroll
      for (int i = 0; i < NW; i++) nw[i] = sw[i] = 0;
    }
    commit_new<W, NW, OffT>(has, w, nw, sw, dg, level, seen, planes, plane_stride, active, heavy, nl, nctr,
                            &ctr->b);
  }
}

// Segmented inclusive OR scan over a warp, segments = equal consecutive keys.
template <typename W>
__device__ __forceinline__ W seg_or_scan(W x, int key) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const W y = shfl_up<W>(x, d);
    const int k2 = __shfl_up_sync(0xffffffffu, key, d);
    if (lane >= d && k2 == key) x |= y;
  }
  return x;
}

// ---------------------------------------------------------------------------
// Pull, light vertices: one warp per tile of 32 consecutive vertices.  The
// tile's wanted adjacency ranges are flattened and read edge-parallel
// (coalesced colIndices), F is gathered per edge, a segmented OR scan folds
// the words per owner vertex into shared memory.
template <typename W, int NW, typename OffT, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_pull_tiles(int64_t n, const OffT* __restrict__ ro,
                                                           const int32_t* __restrict__ ci, const W* __restrict__ F,
                                                           W* seen, W* N, W* planes, int64_t plane_stride, int level,
                                                           Masks<W, NW> active, int heavy, Lists nl, Ctrs* ctr,
                                                           int cur) {
  __shared__ int32_t s_off[WARPS][33];
  __shared__ int64_t s_beg[WARPS][32];
  __shared__ W s_acc[WARPS][32][NW];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int64_t ntiles = (n + 31) >> 5;
  const int64_t warp = (int64_t)blockIdx.x * WARPS + wib;
  const int64_t nwarps = (int64_t)gridDim.x * WARPS;
  LevelCtr* cctr = &ctr->lv[cur];
  LevelCtr* nctr = &ctr->lv[cur ^ 1];
  W live[NW];
#pragma unroll
  for (int i = 0; i < NW; i++) live[i] = (W)cctr->live[i] & active.w[i];
  unsigned long long e_scan = 0, v_scan = 0, v_sweep = 0;
  for (int64_t tile = warp; tile < ntiles; tile += nwarps) {
    const int64_t v = tile * 32 + lane;
    const bool valid = v < n;
    W sw[NW], want[NW];
    bool any = false;
    int64_t beg = 0, dg = 0;
    if (valid) {
      beg = ro[v];
      dg = (int64_t)ro[v + 1] - beg;
#pragma unroll
      for (int i = 0; i < NW; i++) {
        sw[i] = seen[v * NW + i];
        want[i] = live[i] & ~sw[i];
        any = any || want[i] != 0;
      }
    } else {
#pragma unroll
      for (int i = 0; i < NW; i++) sw[i] = want[i] = 0;
    }
    v_sweep += valid ? 1 : 0;
    const bool scan_me = any && dg > 0 && dg <= heavy;
    v_scan += scan_me ? 1 : 0;
    int32_t d = scan_me ? (int32_t)dg : 0;
    // exclusive scan of d over the warp
    int32_t inc = d;
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, inc, s);
      if (lane >= s) inc += y;
    }
    const int32_t total = __shfl_sync(0xffffffffu, inc, 31);
    s_off[wib][lane] = inc - d;
    if (lane == 31) s_off[wib][32] = inc;
    s_beg[wib][lane] = beg;
#pragma unroll
    for (int i = 0; i < NW; i++) s_acc[wib][lane][i] = 0;
    __syncwarp();
    e_scan += (unsigned long long)(lane == 0 ? total : 0);
    for (int32_t base = 0; base < total; base += 32) {
      const int32_t e = base + lane;
      int key = 32 + lane;  // unique key for idle lanes
      W f[NW];
#pragma unroll
      for (int i = 0; i < NW; i++) f[i] = 0;
      if (e < total) {
        // owner: last j with s_off[j] <= e (binary search over 33 offsets)
        int lo = 0, hi = 31;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (s_off[wib][mid] <= e)
            lo = mid;
          else
            hi = mid - 1;
        }
        key = lo;
        const int32_t u = __ldg(&ci[s_beg[wib][lo] + (e - s_off[wib][lo])]);
        if (NW == 1) {
          f[0] = __ldg(&F[u]);
        } else {
#pragma unroll
          for (int i = 0; i < NW; i++) f[i] = __ldg(&F[(int64_t)u * NW + i]);
        }
      }
      const int next_key = __shfl_down_sync(0xffffffffu, key, 1);
      const bool tail = (lane == 31) || (next_key != key);
#pragma unroll
      for (int i = 0; i < NW; i++) {
        const W r = seg_or_scan<W>(f[i], key);
        if (tail && key < 32) s_acc[wib][key][i] |= r;
      }
      __syncwarp();
    }
    W nw[NW];
    bool has = false;
#pragma unroll
    for (int i = 0; i < NW; i++) {
      nw[i] = scan_me ? (s_acc[wib][lane][i] & want[i]) : (W)0;
      has = has || nw[i] != 0;
    }
    if (has) {
#pragma unroll
      for (int i = 0; i < NW; i++) N[v * NW + i] = nw[i];
    }
    commit_new<W, NW, OffT>(has, (int32_t)v, nw, sw, dg, level, seen, planes, plane_stride, active, heavy, nl,
                            nctr, &ctr->b);
    __syncwarp();
  }
  e_scan = warp_sum_u64(e_scan);
  v_scan = warp_sum_u64(v_scan);
  v_sweep = warp_sum_u64(v_sweep);
  if (lane == 0) {
    if (e_scan) atomicAdd(&ctr->b.edges_scanned, e_scan);
    if (v_scan) atomicAdd(&ctr->b.vertices_scanned, v_scan);
    if (v_sweep) atomicAdd(&ctr->b.vertices_swept, v_sweep);
  }
}

// Block-wide OR reduce (all threads get the result).  s_red: W[32][NW].
template <typename W, int NW>
__device__ __forceinline__ void block_or(W (&x)[NW], W (*s_red)[NW]) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < NW; i++) x[i] = warp_or<W>(x[i]);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < NW; i++) s_red[wid][i] = x[i];
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NW; i++) {
    W r = 0;
    for (int k = 0; k < nw; k++) r |= s_red[k][i];
    x[i] = r;
  }
}

// Pull, heavy vertices (degree > heavy): one block per vertex, early exit
// once every wanted bit is found.
template <typename W, int NW, typename OffT>
__global__ void k_pull_heavy(const int32_t* __restrict__ hlist, int32_t nh, const OffT* __restrict__ ro,
                             const int32_t* __restrict__ ci, const W* __restrict__ F, W* seen, W* N, W* planes,
                             int64_t plane_stride, int level, Masks<W, NW> active, int heavy, Lists nl, Ctrs* ctr,
                             int cur) {
  __shared__ W s_red[32][NW];
  LevelCtr* cctr = &ctr->lv[cur];
  LevelCtr* nctr = &ctr->lv[cur ^ 1];
  for (int64_t idx = blockIdx.x; idx < nh; idx += gridDim.x) {
    const int32_t v = hlist[idx];
    W sw[NW], want[NW];
    bool any = false;
#pragma unroll
    for (int i = 0; i < NW; i++) {
      sw[i] = seen[(int64_t)v * NW + i];
      want[i] = ((W)cctr->live[i] & active.w[i]) & ~sw[i];
      any = any || want[i] != 0;
    }
    if (!any) continue;  // uniform across the block
    const int64_t beg = ro[v], end = ro[v + 1];
    W acc[NW];
#pragma unroll
    for (int i = 0; i < NW; i++) acc[i] = 0;
    int64_t scanned = 0;
    for (int64_t base = beg; base < end; base += blockDim.x) {
      const int64_t e = base + threadIdx.x;
      if (e < end) {
        const int32_t u = __ldg(&ci[e]);
#pragma unroll
        for (int i = 0; i < NW; i++) acc[i] |= __ldg(&F[(int64_t)u * NW + i]);
      }
      scanned += imin64((int64_t)blockDim.x, end - base);
      block_or<W, NW>(acc, s_red);
      bool done = true;
#pragma unroll
      for (int i = 0; i < NW; i++) done = done && ((acc[i] & want[i]) == want[i]);
      if (done) break;
    }
    if (threadIdx.x < 32) {
      W nw[NW];
      bool has = false;
#pragma unroll
      for (int i = 0; i < NW; i++) {
        nw[i] = threadIdx.x == 0 ? (acc[i] & want[i]) : (W)0;
        has = has || nw[i] != 0;
      }
      if (has) {
#pragma unroll
        for (int i = 0; i < NW; i++) N[(int64_t)v * NW + i] = nw[i];
      }
      W s0[NW];
#pragma unroll
      for (int i = 0; i < NW; i++) s0[i] = sw[i];
      commit_new<W, NW, OffT>(has, v, nw, s0, end - beg, level, seen, planes, plane_stride, active, heavy, nl,
                              nctr, &ctr->b);
      if (threadIdx.x == 0) {
        atomicAdd(&ctr->b.edges_scanned, (unsigned long long)scanned);
        atomicAdd(&ctr->b.vertices_scanned, 1ull);
      }
    }
    __syncthreads();
  }
}

// Zeroes F at the vertices of a frontier list.
template <typename W, int NW>
__global__ void k_clear_list(const int32_t* __restrict__ list, const int32_t* __restrict__ count, W* F) {
  const int32_t cnt = *count;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)cnt * NW;
       i += (int64_t)gridDim.x * blockDim.x)
    F[(int64_t)list[i / NW] * NW + (i % NW)] = 0;
}

// ---------------------------------------------------------------------------
// Table pass.  Word wi of the pass (sources word_base .. word_base+kbw-1).
// One warp per 32-vertex tile; level[s*n + v] and parent[s*n + v].
template <typename W, int NW>
__device__ __forceinline__ W plane_at(const W* planes, int64_t plane_stride, int j, int64_t v, int wi) {
  return planes[j * plane_stride + v * NW + wi];
}

template <typename W, int NW, typename OffT, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_tables(int64_t n, const OffT* __restrict__ ro,
                                                       const int32_t* __restrict__ ci, const W* __restrict__ seen,
                                                       const W* __restrict__ planes, int64_t plane_stride, int nplanes,
                                                       int wi, int kbw, int heavy, int32_t* __restrict__ level_out,
                                                       int32_t* __restrict__ parent_out, Ctrs* ctr) {
  constexpr int B = WB<W>::bits;
  __shared__ int32_t s_par[WARPS][B][32];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int64_t ntiles = (n + 31) >> 5;
  const int64_t warp = (int64_t)blockIdx.x * WARPS + wib;
  const int64_t nwarps = (int64_t)gridDim.x * WARPS;
  unsigned long long pe = 0;
  for (int64_t tile = warp; tile < ntiles; tile += nwarps) {
    const int64_t v = tile * 32 + lane;
    const bool valid = v < n;
    W sv = 0, p0 = 0, p1 = 0, anyp = 0;
    int64_t beg = 0, dg = 0;
    if (valid) {
      sv = seen[v * NW + wi];
      p0 = plane_at<W, NW>(planes, plane_stride, 0, v, wi);
      p1 = plane_at<W, NW>(planes, plane_stride, 1, v, wi);
      anyp = p0 | p1;
      for (int j = 2; j < nplanes; j++) anyp |= plane_at<W, NW>(planes, plane_stride, j, v, wi);
      beg = ro[v];
      dg = (int64_t)ro[v + 1] - beg;
    }
    const W root = sv & ~anyp;
    const W need = sv & ~root;
    const W t0 = ~p0, t1 = ~(p0 ^ p1);  // bit-sliced (level - 1) mod 4
    const bool is_heavy = dg > heavy;
    // light: lane-private scan with early exit
    W found = 0;
    if (valid && need && !is_heavy && dg <= 32) {
      for (int64_t e = beg; e < beg + dg; e++) {
        const int32_t u = __ldg(&ci[e]);
        pe++;
        const W su = seen[(int64_t)u * NW + wi];
        const W q0 = plane_at<W, NW>(planes, plane_stride, 0, u, wi);
        const W q1 = plane_at<W, NW>(planes, plane_stride, 1, u, wi);
        W eq = su & ~(q0 ^ t0) & ~(q1 ^ t1) & need & ~found;
        found |= eq;
        while (eq) {
          const int b = ffs0(eq);
          s_par[wib][b][lane] = u;
          eq &= eq - 1;
        }
        if (found == need) break;
      }
    }
    // medium: warp-cooperative scan, one vertex at a time
    unsigned med = __ballot_sync(0xffffffffu, valid && need && !is_heavy && dg > 32);
    while (med) {
      const int j = __ffs(med) - 1;
      med &= med - 1;
      const W nd = shfl_idx<W>(need, j);
      const W a0 = shfl_idx<W>(t0, j), a1 = shfl_idx<W>(t1, j);
      const int64_t b0 = __shfl_sync(0xffffffffu, beg, j);
      const int64_t d0 = __shfl_sync(0xffffffffu, dg, j);
      W fnd = 0;
      for (int64_t base = 0; base < d0; base += 32) {
        const int64_t e = base + lane;
        W eq = 0;
        int32_t u = 0;
        if (e < d0) {
          u = __ldg(&ci[b0 + e]);
          const W su = seen[(int64_t)u * NW + wi];
          const W q0 = plane_at<W, NW>(planes, plane_stride, 0, u, wi);
          const W q1 = plane_at<W, NW>(planes, plane_stride, 1, u, wi);
          eq = su & ~(q0 ^ a0) & ~(q1 ^ a1) & nd & ~fnd;
        }
        // exclusive prefix OR in lane (= neighbour) order: the lowest lane wins
        W inc = eq;
#pragma unroll
        for (int s = 1; s < 32; s <<= 1) {
          const W y = shfl_up<W>(inc, s);
          if (lane >= s) inc |= y;
        }
        W excl = shfl_up<W>(inc, 1);
        if (lane == 0) excl = 0;
        W mine = eq & ~excl;
        while (mine) {
          const int b = ffs0(mine);
          s_par[wib][b][j] = u;
          mine &= mine - 1;
        }
        fnd |= shfl_idx<W>(inc, 31);
        if (lane == 0) pe += (unsigned long long)imin64(32, d0 - base);
        if (fnd == nd) break;
      }
    }
    __syncwarp();
    // write rows: level and parent of sources 0..kbw-1 at vertices tile*32 + lane
    if (valid && !is_heavy) {
      constexpr int RP = 8;  // planes held in registers; deeper levels read on demand
      W pl[RP];
#pragma unroll
      for (int j = 0; j < RP; j++) pl[j] = j < nplanes ? plane_at<W, NW>(planes, plane_stride, j, v, wi) : (W)0;
      for (int s = 0; s < kbw; s++) {
        int32_t lv = -1, pr = -1;
        if ((sv >> s) & 1) {
          lv = 0;
#pragma unroll
          for (int j = 0; j < RP; j++) lv |= (int32_t)((pl[j] >> s) & 1) << j;
          for (int j = RP; j < nplanes; j++)
            lv |= (int32_t)((plane_at<W, NW>(planes, plane_stride, j, v, wi) >> s) & 1) << j;
          pr = ((root >> s) & 1) ? (int32_t)v : s_par[wib][s][lane];
        }
        __stcs(&level_out[(int64_t)s * n + v], lv);
        __stcs(&parent_out[(int64_t)s * n + v], pr);
      }
    }
    __syncwarp();
  }
  pe = warp_sum_u64(pe);
  if (lane == 0 && pe) atomicAdd(&ctr->b.parent_edges, pe);
}

// Table pass for heavy vertices: one block per vertex, block-wide ordered
// scan of the adjacency with early exit.
template <typename W, int NW, typename OffT>
__global__ void k_tables_heavy(const int32_t* __restrict__ hlist, int32_t nh, int64_t n, const OffT* __restrict__ ro,
                               const int32_t* __restrict__ ci, const W* __restrict__ seen, const W* __restrict__ planes,
                               int64_t plane_stride, int nplanes, int wi, int kbw, int32_t* __restrict__ level_out,
                               int32_t* __restrict__ parent_out, Ctrs* ctr) {
  __shared__ W s_wor[32];
  __shared__ W s_found;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwb = blockDim.x >> 5;
  for (int64_t idx = blockIdx.x; idx < nh; idx += gridDim.x) {
    const int64_t v = hlist[idx];
    const W sv = seen[v * NW + wi];
    const W p0 = plane_at<W, NW>(planes, plane_stride, 0, v, wi);
    const W p1 = plane_at<W, NW>(planes, plane_stride, 1, v, wi);
    W anyp = p0 | p1;
    for (int j = 2; j < nplanes; j++) anyp |= plane_at<W, NW>(planes, plane_stride, j, v, wi);
    const W root = sv & ~anyp;
    const W need = sv & ~root;
    const W t0 = ~p0, t1 = ~(p0 ^ p1);
    const int64_t beg = ro[v], end = ro[v + 1];
    W fnd = 0;
    unsigned long long pe = 0;
    if (need) {
      for (int64_t base = beg; base < end; base += blockDim.x) {
        const int64_t e = base + threadIdx.x;
        W eq = 0;
        int32_t u = 0;
        if (e < end) {
          u = __ldg(&ci[e]);
          const W su = seen[(int64_t)u * NW + wi];
          const W q0 = plane_at<W, NW>(planes, plane_stride, 0, u, wi);
          const W q1 = plane_at<W, NW>(planes, plane_stride, 1, u, wi);
          eq = su & ~(q0 ^ t0) & ~(q1 ^ t1) & need & ~fnd;
        }
        // block-wide exclusive prefix OR in thread order
        W inc = eq;
#pragma unroll
        for (int s = 1; s < 32; s <<= 1) {
          const W y = shfl_up<W>(inc, s);
          if (lane >= s) inc |= y;
        }
        if (lane == 31) s_wor[wid] = inc;
        __syncthreads();
        W before = 0;
        for (int k = 0; k < wid; k++) before |= s_wor[k];
        W all = 0;
        for (int k = 0; k < nwb; k++) all |= s_wor[k];
        const W lane_excl = shfl_up<W>(inc, 1);
        const W excl = before | (lane ? lane_excl : (W)0);
        W mine = eq & ~excl;
        while (mine) {
          const int b = ffs0(mine);
          parent_out[(int64_t)b * n + v] = u;
          mine &= mine - 1;
        }
        pe += (unsigned long long)imin64((int64_t)blockDim.x, end - base);
        fnd |= all;
        __syncthreads();
        if (fnd == need) break;
      }
    }
    if (threadIdx.x == 0) {
      s_found = fnd;
      if (pe) atomicAdd(&ctr->b.parent_edges, pe);
    }
    for (int s = threadIdx.x; s < kbw; s += blockDim.x) {
      int32_t lv = -1;
      if ((sv >> s) & 1) {
        lv = 0;
        for (int j = 0; j < nplanes; j++) lv |= (int32_t)((plane_at<W, NW>(planes, plane_stride, j, v, wi) >> s) & 1) << j;
        if ((root >> s) & 1) parent_out[(int64_t)s * n + v] = (int32_t)v;
      } else {
        parent_out[(int64_t)s * n + v] = -1;
      }
      level_out[(int64_t)s * n + v] = lv;
    }
    __syncthreads();
  }
}

}  // namespace xbk
