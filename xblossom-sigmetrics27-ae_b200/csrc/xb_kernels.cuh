// xb_kernels.cuh -- sm_100a device code of the multi-source traversal.
//
// Data layout in HBM (one traversal pass = NW words of B bits per vertex,
// B*NW sources traversed together; word i of vertex v at index v*NW+i):
//   seen[v*NW+i]      bits of the sources that have reached v
//   F[v*NW+i]         bits newly reached at the current level (the frontier)
//   N[v*NW+i]         bits reached at the next level (all zero between levels
//                     except at next-frontier vertices)
//   level planes      the level bit-sliced: bit j of the level of every source
//                     at v.  Planes 0 and 1 are interleaved per word
//                     (p01[2*(v*NW+i)] = plane 0, +1 = plane 1) so one
//                     16-byte load returns "level mod 4" of 64 sources; planes
//                     j >= 2 are separate arrays ph[(j-2)*stride + v*NW+i].
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
// adjacent reached vertices differ in level by at most one, and every
// neighbour of a vertex reached by s is reached by s, so "level(u) == L-1"
// reduces to a bit-sliced compare of level mod 4 (planes 0 and 1), done for
// all B sources of a word at once.  The pass walks each 32-vertex tile's
// adjacency edge-parallel in ascending order (per-vertex early exit once every
// needed bit has a parent), transposes the 32-vertex x B-source tile in shared
// memory and writes whole 128-byte rows of the source-major tables with
// streaming stores.
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

// Vertices of degree <= this keep their pull-step parents as one-byte
// adjacency positions (0..255).
constexpr int kP8MaxDegree = 256;

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
  int32_t work;   // chunks handed out by the step that builds this frontier (k_pull_lanes)
  int32_t work2;  // heavy vertices handed out by the same step (k_pull_heavy)
  int32_t n_hwant;  // heavy vertices with wanted bits, listed by the same step (k_heavy_want)
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
  int32_t level;        // level discovered by the current step (0 after init)
  int32_t nplanes;      // level planes in use (all levels < 2^nplanes)
  int32_t zero_plane;   // plane the current step must clear first (-1: none)
  int32_t dir;          // current step: 0 push, 1 pull, 2 none (frontier empty)
  int32_t pushed_deep;  // a push step reached level >= 2
  int32_t push_levels;
  int32_t pull_levels;
  int32_t step_calls;  // k_step_begin calls of the pass ("done" included)
};

struct Ctrs {
  LevelCtr lv[2];
  BatchCtr b;
  int32_t epoch;  // stamp of the current step; grows across passes and calls
  int32_t pad;
};

template <typename W, int NW>
struct Masks {
  W w[NW];
};

// Lists of one frontier: light (deg <= heavy) and heavy vertices, and
// (when bits is set) one bit per vertex marking the frontier's vertices, so
// the pull steps of a sparse frontier skip the gathers of neighbours outside
// it.  The bitmap must be all zero before the step that builds the frontier.
struct Lists {
  int32_t* light;
  int32_t* heavy;
  uint32_t* bits;
};

// A pull step reads the frontier bitmap before each frontier-word gather when
// the frontier holds fewer than n / kSparseDiv vertices: then most gathers
// would return zero words, and the bit (a 4-byte word of a bitmap 1/256 the
// size of the frontier words, mostly cache-resident) saves their HBM sectors.
constexpr int kSparseDiv = 8;

// Bitmap of the current frontier for a pull step, or null when the frontier
// is dense (the check would only add latency).
__device__ __forceinline__ const uint32_t* sparse_bits(const uint32_t* bits, const LevelCtr* cctr, int64_t n) {
  return (bits != nullptr && ((long long)cctr->n_light + cctr->n_heavy) * kSparseDiv < n) ? bits : nullptr;
}

// Whether vertex u is in the frontier (always, without a bitmap).
__device__ __forceinline__ bool in_frontier(const uint32_t* __restrict__ bits, int32_t u) {
  return bits == nullptr || ((__ldg(&bits[u >> 5]) >> (u & 31)) & 1u);
}

// Vector types for loading NW consecutive words / a plane pair at once.
template <typename W, int K>
struct Vec;
template <>
struct Vec<unsigned long long, 1> {
  using T = unsigned long long;
};
template <>
struct Vec<unsigned long long, 2> {
  using T = ulonglong2;
};
template <>
struct Vec<unsigned int, 1> {
  using T = unsigned int;
};
template <>
struct Vec<unsigned int, 2> {
  using T = uint2;
};
template <>
struct Vec<unsigned int, 4> {
  using T = uint4;
};

// Loads K consecutive words starting at p (p aligned to K words, read-only
// for the rest of the kernel or written only by the loading thread).
template <typename W, int K>
__device__ __forceinline__ void load_words(const W* __restrict__ p, W (&out)[K]) {
  if constexpr (K == 1) {
    out[0] = __ldg(p);
  } else if constexpr (sizeof(W) == 8 && K == 2) {
    const ulonglong2 x = __ldg(reinterpret_cast<const ulonglong2*>(p));
    out[0] = x.x;
    out[1] = x.y;
  } else if constexpr (sizeof(W) == 8 && K == 4) {
    // one 32-byte load (sm_100): a whole sector per lane in one instruction,
    // half the L1 wavefronts of two 16-byte loads
    unsigned long long a, b, c, d;
    asm("ld.global.nc.v4.u64 {%0, %1, %2, %3}, [%4];" : "=l"(a), "=l"(b), "=l"(c), "=l"(d) : "l"(p));
    out[0] = a;
    out[1] = b;
    out[2] = c;
    out[3] = d;
  } else if constexpr (sizeof(W) == 4 && K == 2) {
    const uint2 x = __ldg(reinterpret_cast<const uint2*>(p));
    out[0] = x.x;
    out[1] = x.y;
  } else {
    static_assert(sizeof(W) == 4 && K == 4, "unsupported word vector");
    const uint4 x = __ldg(reinterpret_cast<const uint4*>(p));
    out[0] = x.x;
    out[1] = x.y;
    out[2] = x.z;
    out[3] = x.w;
  }
}

// Level planes of one traversal pass.
template <typename W, int NW>
struct Planes {
  W* p01;          // planes 0 and 1, interleaved per word
  W* ph;           // planes 2.. : ph[(j-2)*stride + v*NW + i]
  int64_t stride;  // words per plane array

  __device__ __forceinline__ W get(int j, int64_t v, int i) const {
    return j < 2 ? p01[((v * NW + i) << 1) + j] : ph[(int64_t)(j - 2) * stride + v * NW + i];
  }
  // ORs `bits` into the planes of the bits set in `level`.
  __device__ __forceinline__ void add(int level, int64_t v, int i, W bits) const {
    const int64_t q = (v * NW + i) << 1;
    if (level & 1) p01[q] |= bits;
    if (level & 2) p01[q + 1] |= bits;
    for (int j = 2; (level >> j) != 0; j++)
      if ((level >> j) & 1) ph[(int64_t)(j - 2) * stride + v * NW + i] |= bits;
  }
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

// Zeroes the position-plane row of (v, word i).  Rows are not cleared per
// pass: each is zeroed (or written whole) when its vertex first gets bits of
// that word -- here for sources and pushed vertices, by the pull otherwise --
// and rows of words a vertex never reaches are never read.
template <typename W>
__device__ __forceinline__ void ppos_zero_row(W* ppos, int64_t v, int nw, int i) {
  W* r = ppos + (v * nw + i) * 8;
#pragma unroll
  for (int k = 0; k < 8; k++) r[k] = 0;
}

// Per-lane counter increments, kept in registers until the kernel ends.
template <typename W, int NW>
struct StatAcc {
  unsigned long long e_tr = 0, rch = 0, fe = 0;
  long long fin = 0;
  W live[NW] = {};
};

// Records a newly reached vertex (all lanes call; `has` marks lanes that own
// one): folds new bits into seen and the level planes, accumulates the
// counters and appends the vertex to the next frontier's light/heavy list.
template <typename W, int NW, typename OffT>
__device__ __forceinline__ void commit_new(bool has, int32_t w, const W (&nw)[NW], const W (&sw)[NW],
                                           int64_t dg, int level, W* seen, const Planes<W, NW>& pl,
                                           const Masks<W, NW>& active, int heavy, Lists nl, LevelCtr* nctr,
                                           StatAcc<W, NW>& acc) {
  if (has) {
    bool full = true;
    int cnt = 0;
#pragma unroll
    for (int i = 0; i < NW; i++) {
      const W s2 = sw[i] | nw[i];
      if (nw[i]) {
        seen[(int64_t)w * NW + i] = s2;
        pl.add(level, w, i, nw[i]);
      }
      cnt += popc(nw[i]);
      full = full && (s2 == active.w[i]);
      acc.live[i] |= nw[i];
    }
    acc.rch += (unsigned long long)cnt;
    acc.e_tr += (unsigned long long)dg * (unsigned long long)cnt;
    acc.fe += (unsigned long long)dg;
    if (full) acc.fin -= dg;
  }
  if (has && nl.bits) atomicOr(&nl.bits[w >> 5], 1u << (w & 31));
  const bool light = has && dg <= heavy;
  const bool hv = has && dg > heavy;
  warp_append(light, w, nl.light, &nctr->n_light);
  warp_append(hv, w, nl.heavy, &nctr->n_heavy);
}

// Folds a warp's accumulated counters into the level / batch counters: one
// set of atomics per warp per kernel instead of per committed tile (all 32
// lanes must call it).
template <typename W, int NW>
__device__ __forceinline__ void flush_stats(StatAcc<W, NW>& acc, LevelCtr* nctr, BatchCtr* bc) {
  const unsigned long long e_tr = warp_sum_u64(acc.e_tr);
  const unsigned long long rch = warp_sum_u64(acc.rch);
  const unsigned long long fe = warp_sum_u64(acc.fe);
  const long long fin = warp_sum_i64(acc.fin);
  W lv[NW];
#pragma unroll
  for (int i = 0; i < NW; i++) lv[i] = warp_or<W>(acc.live[i]);
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
                             W* seen, Planes<W, NW> pl, Masks<W, NW> active, int heavy, Lists fl, Ctrs* ctr,
                             W* ppos = nullptr) {
  constexpr int B = WB<W>::bits;
  const int t = threadIdx.x;
  int32_t v = -1;
  if (t < kb) {
    v = src[t];
    const W bit = (W)1 << (t % B);
    atomicOr(&F[(int64_t)v * NW + t / B], bit);
    atomicOr(&seen[(int64_t)v * NW + t / B], bit);
    if (ppos) ppos_zero_row<W>(ppos, v, NW, t / B);  // sources sharing a row write the same zeros
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
    sw[i] = 0;
  }
  const int64_t dg = first ? deg_of(ro, v) : 0;
  // level 0 sets no plane bits; seen already holds the bits and commit_new
  // rewrites the same value.
  StatAcc<W, NW> acc;
  commit_new<W, NW, OffT>(first, v, nw, sw, dg, 0, seen, pl, active, heavy, fl, &ctr->lv[0], acc);
  flush_stats<W, NW>(acc, &ctr->lv[0], &ctr->b);
}

// Push body for one edge (v -> w) with frontier words f.  Returns true when
// this thread is the first toucher of w in this level.
template <typename W, int NW>
__device__ __forceinline__ bool push_edge(int32_t w, const W (&f)[NW], const W* __restrict__ seen, W* N,
                                          int32_t* stamp, int32_t epoch) {
  bool app = false, added = false;
  W sw[NW];
  load_words<W, NW>(seen + (int64_t)w * NW, sw);
#pragma unroll
  for (int i = 0; i < NW; i++) {
    const W m = f[i] & ~sw[i];
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
  return app;
}

// ---------------------------------------------------------------------------
// Push, light frontier vertices: one warp per vertex.
// NW == 1: the lane whose atomicOr turns N[w] from 0 to non-zero appends w.
// NW > 1: first toucher decided by an epoch stamp per vertex.
template <typename W, int NW, typename OffT>
__global__ void k_push_light(const int32_t* __restrict__ list, const int32_t* __restrict__ count,
                             const OffT* __restrict__ ro, const int32_t* __restrict__ ci, W* F,
                             const W* __restrict__ seen, W* N, int32_t* stamp, int32_t* touched, Ctrs* ctr,
                             int cur) {
  const int32_t epoch = ctr->epoch;
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
        w = __ldcs(&ci[e]);
        app = push_edge<W, NW>(w, f, seen, N, stamp, epoch);
      }
      warp_append(app, w, touched, &nctr->n_touched);
    }
  }
  if (lane == 0 && vcount) {
    atomicAdd(&ctr->b.edges_scanned, scanned);
    atomicAdd(&ctr->b.vertices_scanned, vcount);
  }
}

// Push, heavy frontier vertices: blockIdx.y walks the heavy list, blockIdx.x
// splits each adjacency into chunks of `chunk` edges so a hub spreads over
// many SMs.  F of heavy vertices is cleared afterwards by k_clear_list.
template <typename W, int NW, typename OffT>
__global__ void k_push_heavy(const int32_t* __restrict__ list, const int32_t* __restrict__ count,
                             const OffT* __restrict__ ro, const int32_t* __restrict__ ci, const W* __restrict__ F,
                             const W* __restrict__ seen, W* N, int32_t* stamp, int32_t* touched, Ctrs* ctr,
                             int cur, int chunk) {
  const int32_t epoch = ctr->epoch;
  const int32_t cnt = *count;
  LevelCtr* nctr = &ctr->lv[cur ^ 1];
  for (int64_t idx = blockIdx.y; idx < cnt; idx += gridDim.y) {
    const int32_t v = list[idx];
    W f[NW];
#pragma unroll
    for (int i = 0; i < NW; i++) f[i] = F[(int64_t)v * NW + i];
    const int64_t beg = ro[v], end = ro[v + 1];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      atomicAdd(&ctr->b.edges_scanned, (unsigned long long)(end - beg));
      atomicAdd(&ctr->b.vertices_scanned, 1ull);
    }
    for (int64_t cb = beg + (int64_t)blockIdx.x * chunk; cb < end; cb += (int64_t)gridDim.x * chunk) {
      const int64_t ce = imin64(end, cb + chunk);
      for (int64_t base = cb; base < ce; base += blockDim.x) {
        const int64_t e = base + threadIdx.x;
        bool app = false;
        int32_t w = 0;
        if (e < ce) {
          w = __ldcs(&ci[e]);
          app = push_edge<W, NW>(w, f, seen, N, stamp, epoch);
        }
        warp_append(app, w, touched, &nctr->n_touched);
      }
    }
  }
}

// After a push: fold N into seen/planes for every touched vertex, bucket the
// next frontier.
template <typename W, int NW, typename OffT>
__global__ void k_push_finalize(const int32_t* __restrict__ touched, const OffT* __restrict__ ro, const W* N,
                                W* seen, Planes<W, NW> pl, Masks<W, NW> active, int heavy, Lists nl, Ctrs* ctr,
                                int cur, W* pushed, uint32_t* consumed_bits, int64_t bit_words,
                                W* ppos = nullptr) {
  const int level = ctr->b.level;
  LevelCtr* nctr = &ctr->lv[cur ^ 1];
  const int32_t cnt = nctr->n_touched;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  if (consumed_bits)  // the pushed frontier's bitmap (nothing reads it any more)
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < bit_words; i += stride) consumed_bits[i] = 0;
  StatAcc<W, NW> acc;
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
        // bits reached by a push step have no recorded parent index: the
        // table pass searches their parents
        pushed[(int64_t)w * NW + i] |= nw[i];
        if (ppos && nw[i] && !sw[i]) ppos_zero_row<W>(ppos, w, NW, i);  // first bits of this word
      }
      dg = deg_of(ro, w);
    } else {
#pragma unroll
      for (int i = 0; i < NW; i++) nw[i] = sw[i] = 0;
    }
    commit_new<W, NW, OffT>(has, w, nw, sw, dg, level, seen, pl, active, heavy, nl, nctr, acc);
  }
  flush_stats<W, NW>(acc, nctr, &ctr->b);
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

// Owner lane of flat edge e: last j in [0,31] with off[j] <= e.
__device__ __forceinline__ int flat_owner(const int32_t* __restrict__ off, int32_t e) {
  int lo = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1)
    if (off[lo + step] <= e) lo += step;
  return lo;
}

// Flat-window bookkeeping of a warp tile: lane j owns a run of d_j edges at
// flat offsets [off_j, off_j + d_j).  For the 32 flat positions starting at
// wb, returns the owner lane of this lane's position and the lane index of the
// first position of that owner's run inside the window (-1 when the run began
// in an earlier window).  Lanes past the end get owner -1.
struct WinOwner {
  int owner;
  int head;
};
__device__ __forceinline__ WinOwner window_owner(int32_t off, int32_t d, int32_t wb, int32_t total,
                                                 const int8_t* __restrict__ r2l) {
  const int lane = threadIdx.x & 31;
  const bool in_win = d > 0 && off >= wb && off < wb + 32;
  const unsigned starts = __reduce_or_sync(0xffffffffu, in_win ? (1u << (off - wb)) : 0u);
  const int before = __popc(__ballot_sync(0xffffffffu, d > 0 && off < wb));
  WinOwner r{-1, -1};
  if (wb + lane < total) {
    const unsigned upto = starts & (0xffffffffu >> (31 - lane));  // starts at positions <= lane
    const int cnt = before + __popc(upto);
    r.owner = r2l[cnt - 1];
    r.head = upto ? 31 - __clz(upto) : -1;
  }
  return r;
}

// ---------------------------------------------------------------------------
// Pull, light vertices: one warp per tile of 32 consecutive vertices.  The
// tile's wanted adjacency ranges are flattened and read edge-parallel
// (coalesced colIndices), U x 32 edges per round with all loads issued before
// any is consumed; F is gathered per edge and a segmented OR scan (head flags
// from one warp reduction per window) folds the words per owner vertex into
// shared memory.  The same scan gives, for every newly reached bit, its first
// frontier neighbour in ascending (= smallest-id) order: that neighbour's
// position in the owner's adjacency (< 256 for vertices of degree <=
// kP8MaxDegree) is recorded bit-sliced in ppos (8 words per vertex and word:
// word k holds bit k of every source's position), so one claim of any number
// of sources costs at most 8 ORs and the table pass reads parents instead of
// searching for them.  ppos must be zero at the start of the pass.
template <typename W, int NW, typename OffT, int WARPS, int U>
__global__ void __launch_bounds__(WARPS * 32, 32 / WARPS) k_pull_tiles(int64_t n, const OffT* __restrict__ ro,
                                                           const int32_t* __restrict__ ci, const W* __restrict__ F,
                                                           W* seen, W* N, Planes<W, NW> pl, Masks<W, NW> active,
                                                           int heavy, Lists nl, Ctrs* ctr, int cur,
                                                           W* __restrict__ ppos) {
  const int level = ctr->b.level;
  __shared__ int64_t s_base[WARPS][32];  // colIndices index of flat position 0 of each lane's run
  __shared__ int32_t s_off[WARPS][32];
  __shared__ int8_t s_r2l[WARPS][32];    // rank among non-empty runs -> lane
  __shared__ W s_acc[WARPS][32][NW];
  __shared__ W s_want[WARPS][32][NW];
  __shared__ W s_pp[WARPS][32][NW][8];   // bit-sliced positions of this level's claims
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
  StatAcc<W, NW> acc;
  for (int64_t tile = warp; tile < ntiles; tile += nwarps) {
    const int64_t v = tile * 32 + lane;
    const bool valid = v < n;
    W sw[NW], want[NW];
    bool any = false;
    int64_t beg = 0, dg = 0;
    if (valid) {
      beg = ro[v];
      dg = (int64_t)ro[v + 1] - beg;
      load_words<W, NW>(seen + v * NW, sw);
#pragma unroll
      for (int i = 0; i < NW; i++) {
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
    const int32_t d = scan_me ? (int32_t)dg : 0;
    int32_t inc = d;
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, inc, s);
      if (lane >= s) inc += y;
    }
    const int32_t total = __shfl_sync(0xffffffffu, inc, 31);
    const int32_t off = inc - d;
    const unsigned nz = __ballot_sync(0xffffffffu, d > 0);
    if (d > 0) s_r2l[wib][__popc(nz & ((1u << lane) - 1u))] = (int8_t)lane;
    s_off[wib][lane] = off;
    s_base[wib][lane] = beg - off;
#pragma unroll
    for (int i = 0; i < NW; i++) {
      s_acc[wib][lane][i] = 0;
      s_want[wib][lane][i] = want[i];
#pragma unroll
      for (int k = 0; k < 8; k++) s_pp[wib][lane][i][k] = 0;
    }
    __syncwarp();
    e_scan += (unsigned long long)(lane == 0 ? total : 0);
    for (int32_t base = 0; base < total; base += 32 * U) {
      WinOwner wo[U];
      int32_t col[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int32_t wb = base + u * 32;
        wo[u] = window_owner(off, d, wb, total, s_r2l[wib]);
        col[u] = wo[u].owner >= 0 ? __ldcs(&ci[s_base[wib][wo[u].owner] + wb + lane]) : -1;
      }
      W f[U][NW];
#pragma unroll
      for (int u = 0; u < U; u++) {
        if (col[u] >= 0) {
          load_words<W, NW>(F + (int64_t)col[u] * NW, f[u]);
        } else {
#pragma unroll
          for (int i = 0; i < NW; i++) f[u][i] = 0;
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int o = wo[u].owner, h = wo[u].head;
        const int32_t e = base + u * 32 + lane;
        // tail = last position of its run in this window
        const int o_next = __shfl_down_sync(0xffffffffu, o, 1);
        const bool tail = o >= 0 && (lane == 31 || o_next != o);
        const int32_t pos = o >= 0 ? e - s_off[wib][o] : 0;  // position in the owner's adjacency
#pragma unroll
        for (int i = 0; i < NW; i++) {
          // candidates: wanted bits of the owner this edge brings that no
          // earlier window had; a window without any changes nothing
          const W c = o >= 0 ? (f[u][i] & s_want[wib][o][i] & ~s_acc[wib][o][i]) : (W)0;
          if (!__any_sync(0xffffffffu, c != 0)) continue;
          W x = c;
#pragma unroll
          for (int s = 1; s < 32; s <<= 1) {
            const W y = shfl_up<W>(x, s);
            if (lane - s >= h && lane >= s) x |= y;
          }
          W ex = shfl_up<W>(x, 1);
          if (!(lane >= 1 && lane - 1 >= h)) ex = 0;
          if (o >= 0) {
            const W claim = c & ~ex;
            if (claim && pos < kP8MaxDegree) {
              // bit k of this position goes to plane k of every claimed source
#pragma unroll
              for (int k = 0; k < 8; k++)
                if ((pos >> k) & 1) atomicOr(&s_pp[wib][o][i][k], claim);
            }
          }
          __syncwarp();
          if (tail) s_acc[wib][o][i] |= x;
          __syncwarp();
        }
      }
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
      // fold this level's claimed positions into the vertex's position planes
      if (dg <= kP8MaxDegree) {
#pragma unroll
        for (int i = 0; i < NW; i++) {
          if (!nw[i]) continue;
          W* prow = ppos + (v * NW + i) * 8;
#pragma unroll
          for (int k = 0; k < 8; k++) {
            const W add = s_pp[wib][lane][i][k];
            if (add) prow[k] |= add;
          }
        }
      }
    }
    commit_new<W, NW, OffT>(has, (int32_t)v, nw, sw, dg, level, seen, pl, active, heavy, nl, nctr, acc);
    __syncwarp();
  }
  flush_stats<W, NW>(acc, nctr, &ctr->b);
  e_scan = warp_sum_u64(e_scan);
  v_scan = warp_sum_u64(v_scan);
  v_sweep = warp_sum_u64(v_sweep);
  if (lane == 0) {
    if (e_scan) atomicAdd(&ctr->b.edges_scanned, e_scan);
    if (v_scan) atomicAdd(&ctr->b.vertices_scanned, v_scan);
    if (v_sweep) atomicAdd(&ctr->b.vertices_swept, v_sweep);
  }
}

// colIndices are read once per step and are larger than L2: their loads use
// the streaming (evict-first) path so the frontier and seen words the edges
// gather stay resident in L2.
//
// Pull, light vertices (degree 1..heavy), one vertex per lane.  The graph's
// light vertices are listed by falling degree (lorder), so the 32 lanes of a
// warp walk adjacencies of nearly equal length; warps take chunks of the list
// (lchunk: at most kLaneChunk vertices and about kLaneChunkEdges edges each)
// from a counter, longest first, and queue the wanted vertices in shared
// memory, so every processed group of 32 is full.  Each
// lane scans its adjacency in ascending order with 16-byte colIndices loads and
// one frontier-word gather per edge, and stops once every wanted bit is found:
// the edge where a bit first appears is its smallest-id parent, recorded
// bit-sliced in ppos (position < kP8MaxDegree) as in k_pull_tiles.  nctr->work
// must be zero at launch (k_step_begin clears the next level's counters).
constexpr int kLaneChunk = 256;
constexpr int kLaneChunkEdges = 2048;

template <typename W, int NW, typename OffT>
__device__ __forceinline__ void pull_lane_vertex(bool act, int32_t v, const W (&sw)[NW], const W (&live)[NW],
                                                 const OffT* __restrict__ ro, const int32_t* __restrict__ ci,
                                                 const W* __restrict__ F, W* seen, W* N, const Planes<W, NW>& pl,
                                                 const Masks<W, NW>& active, int heavy, int level, Lists nl,
                                                 LevelCtr* nctr, W* __restrict__ ppos, StatAcc<W, NW>& sacc,
                                                 unsigned long long& e_scan, W* spp,
                                                 const uint32_t* __restrict__ fb) {
  // position planes of this lane's claims: registers for one word, the
  // lane's shared-memory column for more (plane-major, 32 lanes apart, so a
  // warp's accesses hit distinct banks; they change only on a claim)
  constexpr bool kRegPP = NW == 1;
  W want[NW], acc[NW], rpp[kRegPP ? 8 : 1];
  auto pp = [&](int i, int k) -> W& { return kRegPP ? rpp[k] : spp[(i * 8 + k) * 32]; };
  int64_t beg = 0, end = 0;
  if (act) {
    beg = ro[v];
    end = ro[v + 1];
  }
#pragma unroll
  for (int i = 0; i < NW; i++) {
    want[i] = act ? (live[i] & ~sw[i]) : (W)0;
    acc[i] = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) pp(i, k) = 0;
  }
  const bool rec = end - beg <= kP8MaxDegree;
  // aligned groups of G entries (G/4 16-byte loads; G = 8 for one word per
  // vertex, 4 for more, so the gathered words fit in registers); entries
  // outside [beg, end) are masked off.  The next group's colIndices are
  // loaded before this group's frontier words are gathered, so the two
  // latencies overlap.
  constexpr int G = NW == 1 ? 8 : 4;
  constexpr int Q = G / 4;
  int64_t j0 = beg & ~(int64_t)3;
  int4 q[Q];
#pragma unroll
  for (int h = 0; h < Q; h++) q[h] = make_int4(0, 0, 0, 0);
  if (j0 < end) {
#pragma unroll
    for (int h = 0; h < Q; h++) q[h] = __ldcs(reinterpret_cast<const int4*>(ci + j0 + 4 * h));
  }
  for (; j0 < end; j0 += G) {
    int32_t cols[G];
#pragma unroll
    for (int h = 0; h < Q; h++) {
      cols[4 * h] = q[h].x;
      cols[4 * h + 1] = q[h].y;
      cols[4 * h + 2] = q[h].z;
      cols[4 * h + 3] = q[h].w;
    }
    if (j0 + G < end) {
#pragma unroll
      for (int h = 0; h < Q; h++) q[h] = __ldcs(reinterpret_cast<const int4*>(ci + j0 + G + 4 * h));
    }
    W f[G][NW];
#pragma unroll
    for (int t = 0; t < G; t++) {
      const int64_t j = j0 + t;
      if (j >= beg && j < end && in_frontier(fb, cols[t])) {
        load_words<W, NW>(F + (int64_t)cols[t] * NW, f[t]);
      } else {
#pragma unroll
        for (int i = 0; i < NW; i++) f[t][i] = 0;
      }
    }
    bool done = true;
#pragma unroll
    for (int t = 0; t < G; t++) {
      const int pos = (int)(j0 + t - beg);
#pragma unroll
      for (int i = 0; i < NW; i++) {
        const W c = f[t][i] & want[i] & ~acc[i];
        if (c) {
          acc[i] |= c;
          if (rec) {
#pragma unroll
            for (int k = 0; k < 8; k++)
              if ((pos >> k) & 1) pp(i, k) |= c;
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < NW; i++) done = done && acc[i] == want[i];
    if (done) {
      j0 += G;
      break;
    }
  }
  if (act) e_scan += (unsigned long long)(imin64(j0, end) - beg);
  bool has = false;
#pragma unroll
  for (int i = 0; i < NW; i++) has = has || acc[i] != 0;
  if (has) {
#pragma unroll
    for (int i = 0; i < NW; i++) {
      N[(int64_t)v * NW + i] = acc[i];
      if (rec && acc[i]) {
        W* prow = ppos + ((int64_t)v * NW + i) * 8;
        if (sw[i] == 0) {
          // the vertex's first bits of this word: the row is written whole
#pragma unroll
          for (int k = 0; k < 8; k++) prow[k] = pp(i, k);
        } else {
#pragma unroll
          for (int k = 0; k < 8; k++)
            if (pp(i, k)) prow[k] |= pp(i, k);
        }
      }
    }
  }
  commit_new<W, NW, OffT>(has, v, acc, sw, end - beg, level, seen, pl, active, heavy, nl, nctr, sacc);
}

template <typename W, int NW, typename OffT, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, WARPS == 4 ? 4 : 3) k_pull_lanes(int32_t nchunks, const int32_t* __restrict__ lchunk,
                                                           const int32_t* __restrict__ lorder,
                                                           const OffT* __restrict__ ro,
                                                           const int32_t* __restrict__ ci, const W* __restrict__ F,
                                                           W* seen, W* N, Planes<W, NW> pl, Masks<W, NW> active,
                                                           int heavy, Lists nl, Ctrs* ctr, int cur,
                                                           W* __restrict__ ppos, int64_t n,
                                                           const uint32_t* __restrict__ fbits,
                                                           uint8_t* __restrict__ cdone) {
  const int level = ctr->b.level;
  __shared__ int32_t s_qv[WARPS][64];
  __shared__ W s_qs[WARPS][64][NW];
  __shared__ W s_pp[NW > 1 ? WARPS : 1][NW > 1 ? NW * 8 : 1][32];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  LevelCtr* cctr = &ctr->lv[cur];
  LevelCtr* nctr = &ctr->lv[cur ^ 1];
  W live[NW];
#pragma unroll
  for (int i = 0; i < NW; i++) live[i] = (W)cctr->live[i] & active.w[i];
  unsigned long long e_scan = 0, v_scan = 0, v_sweep = 0;
  StatAcc<W, NW> sacc;
  int qn = 0;  // queued vertices (warp-uniform)
  W* spp = NW > 1 ? &s_pp[NW > 1 ? wib : 0][0][lane] : nullptr;
  const uint32_t* fb = sparse_bits(fbits, cctr, n);
  for (;;) {
    int chunk = 0;
    if (lane == 0) chunk = atomicAdd(&nctr->work, 1);
    chunk = __shfl_sync(0xffffffffu, chunk, 0);
    const bool last = chunk >= nchunks;
    if (!last) {
      // a chunk none of whose vertices wanted a live bit keeps wanting none:
      // live bits only shrink over a pass and seen bits only grow
      if (cdone[chunk]) continue;
      bool chunk_want = false;
      const int64_t c0 = lchunk[chunk], c1 = lchunk[chunk + 1];
      for (int64_t t = c0; t < c1; t += 32) {
        const int64_t idx = t + lane;
        int32_t v = 0;
        W sw[NW];
        bool want = false;
#pragma unroll
        for (int i = 0; i < NW; i++) sw[i] = 0;
        if (idx < c1) {
          v = lorder[idx];
          load_words<W, NW>(seen + (int64_t)v * NW, sw);
#pragma unroll
          for (int i = 0; i < NW; i++) want = want || (live[i] & ~sw[i]) != 0;
          v_sweep++;
        }
        const unsigned wm = __ballot_sync(0xffffffffu, want);
        chunk_want = chunk_want || wm != 0;
        if (want) {
          const int slot = qn + __popc(wm & ((1u << lane) - 1u));
          s_qv[wib][slot] = v;
#pragma unroll
          for (int i = 0; i < NW; i++) s_qs[wib][slot][i] = sw[i];
        }
        qn += __popc(wm);
        __syncwarp();
        if (qn >= 32) {
          W qs[NW];
#pragma unroll
          for (int i = 0; i < NW; i++) qs[i] = s_qs[wib][lane][i];
          const int32_t qv = s_qv[wib][lane];
          // move the overflow (< 32 entries) to the front
          const int rest = qn - 32;
          int32_t mv = 0;
          W ms[NW];
          if (lane < rest) {
            mv = s_qv[wib][32 + lane];
#pragma unroll
            for (int i = 0; i < NW; i++) ms[i] = s_qs[wib][32 + lane][i];
          }
          __syncwarp();
          if (lane < rest) {
            s_qv[wib][lane] = mv;
#pragma unroll
            for (int i = 0; i < NW; i++) s_qs[wib][lane][i] = ms[i];
          }
          qn = rest;
          __syncwarp();
          v_scan++;
          pull_lane_vertex<W, NW, OffT>(true, qv, qs, live, ro, ci, F, seen, N, pl, active, heavy, level, nl, nctr,
                                        ppos, sacc, e_scan, spp, fb);
        }
      }
      if (!chunk_want && lane == 0) cdone[chunk] = 1;
    }
    if (last) {
      // the list is exhausted: drain the partial queue
      if (qn > 0) {
        const bool act = lane < qn;
        W qs[NW];
        int32_t qv = 0;
#pragma unroll
        for (int i = 0; i < NW; i++) qs[i] = act ? s_qs[wib][lane][i] : (W)0;
        if (act) qv = s_qv[wib][lane];
        v_scan += act ? 1 : 0;
        pull_lane_vertex<W, NW, OffT>(act, qv, qs, live, ro, ci, F, seen, N, pl, active, heavy, level, nl, nctr,
                                      ppos, sacc, e_scan, spp, fb);
      }
      break;
    }
  }
  flush_stats<W, NW>(sacc, nctr, &ctr->b);
  e_scan = warp_sum_u64(e_scan);
  v_scan = warp_sum_u64(v_scan);
  v_sweep = warp_sum_u64(v_sweep);
  if (lane == 0) {
    if (e_scan) atomicAdd(&ctr->b.edges_scanned, e_scan);
    if (v_scan) atomicAdd(&ctr->b.vertices_scanned, v_scan);
    if (v_sweep) atomicAdd(&ctr->b.vertices_swept, v_sweep);
  }
}

// First occurrence inside a warp group of 32 consecutive edges (lane order =
// edge order): returns the bits of f that no earlier lane and no earlier group
// (`before`) has; *grp receives the OR of the whole group.
template <typename W>
__device__ __forceinline__ W first_bits(W f, W before, W* grp) {
  const int lane = threadIdx.x & 31;
  W x = f;
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    const W y = shfl_up<W>(x, s);
    if (lane >= s) x |= y;
  }
  W ex = shfl_up<W>(x, 1);
  if (lane == 0) ex = 0;
  *grp = shfl_idx<W>(x, 31);
  return f & ~ex & ~before;
}

// Pull, heavy vertices of degree <= hub: one warp per vertex, U x 32 edges per
// round in ascending order with all loads issued up front, early exit once
// every wanted bit is found.  The first frontier neighbour of each newly
// reached bit is its min-id parent; it is stored in hpar[idx*ROW + bit] (ROW =
// B*NW) for the table pass.  Hubs (degree > hub) are left to k_pull_hubs.
//
// The heavy vertices a step must scan are listed first (k_heavy_want: one
// thread per heavy vertex, warp-ballot compaction of their heavy indices), so
// the warps of k_pull_heavy take only vertices with work from the counter.
template <typename W, int NW, typename OffT>
__global__ void __launch_bounds__(256) k_heavy_want(const int32_t* __restrict__ hlist, int32_t nh,
                                                    const OffT* __restrict__ ro, const W* __restrict__ seen,
                                                    Masks<W, NW> active, int hub, Ctrs* ctr, int cur,
                                                    int32_t* __restrict__ wlist) {
  const LevelCtr* cctr = &ctr->lv[cur];
  LevelCtr* nctr = &ctr->lv[cur ^ 1];
  W live[NW];
#pragma unroll
  for (int i = 0; i < NW; i++) live[i] = (W)cctr->live[i] & active.w[i];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < nh; base += stride) {
    const int64_t idx = base + threadIdx.x;
    bool want = false;
    if (idx < nh) {
      const int32_t v = hlist[idx];
      if (deg_of(ro, v) <= hub) {
        W sw[NW];
        load_words<W, NW>(seen + (int64_t)v * NW, sw);
#pragma unroll
        for (int i = 0; i < NW; i++) want = want || (live[i] & ~sw[i]) != 0;
      }
    }
    warp_append(want, (int32_t)idx, wlist, &nctr->n_hwant);
  }
}

template <typename W, int NW, typename OffT, int U>
__global__ void __launch_bounds__(256, (NW == 4 && U == 1) ? 3 : (NW == 4 ? 2 : 1)) k_pull_heavy(const int32_t* __restrict__ hlist,
                             const int32_t* __restrict__ wlist, const OffT* __restrict__ ro,
                             const int32_t* __restrict__ ci, const W* __restrict__ F, W* seen, W* N,
                             Planes<W, NW> pl, Masks<W, NW> active, int heavy, int hub, Lists nl, Ctrs* ctr,
                             int cur, int32_t* __restrict__ hpar, int64_t n, const uint32_t* __restrict__ fbits) {
  const int level = ctr->b.level;
  constexpr int B = WB<W>::bits;
  constexpr int ROW = B * NW;
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  LevelCtr* cctr = &ctr->lv[cur];
  LevelCtr* nctr = &ctr->lv[cur ^ 1];
  W live[NW];
#pragma unroll
  for (int i = 0; i < NW; i++) live[i] = (W)cctr->live[i] & active.w[i];
  StatAcc<W, NW> sacc;
  unsigned long long scanned = 0, vcount = 0;
  (void)warp;
  (void)nwarps;
  (void)hub;
  const int32_t nwant = nctr->n_hwant;  // listed by k_heavy_want before this kernel
  const uint32_t* fb = sparse_bits(fbits, cctr, n);
  for (;;) {
    // the list keeps the heavy list's falling-degree order: warps take
    // vertices from a counter, the longest adjacencies first
    int32_t t = 0;
    if (lane == 0) t = atomicAdd(&nctr->work2, 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= nwant) break;
    const int32_t idx = wlist[t];
    const int32_t v = hlist[idx];
    const int64_t beg = ro[v], end = ro[v + 1];
    W sw[NW], want[NW];
    load_words<W, NW>(seen + (int64_t)v * NW, sw);
    bool any = false;
#pragma unroll
    for (int i = 0; i < NW; i++) {
      want[i] = live[i] & ~sw[i];
      any = any || want[i] != 0;
    }
    if (!any) continue;  // warp-uniform
    vcount++;
    W acc[NW];
#pragma unroll
    for (int i = 0; i < NW; i++) acc[i] = 0;
    // colIndices of the next round are loaded before this round's gathers
    int32_t coln[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int64_t e = beg + u * 32 + lane;
      coln[u] = e < end ? __ldcs(&ci[e]) : -1;
    }
    for (int64_t base = beg; base < end; base += 32 * U) {
      int32_t col[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        col[u] = coln[u];
        const int64_t e = base + 32 * U + u * 32 + lane;
        coln[u] = e < end ? __ldcs(&ci[e]) : -1;
      }
      W f[U][NW];
#pragma unroll
      for (int u = 0; u < U; u++) {
        if (col[u] >= 0 && in_frontier(fb, col[u])) {
          load_words<W, NW>(F + (int64_t)col[u] * NW, f[u]);
        } else {
#pragma unroll
          for (int i = 0; i < NW; i++) f[u][i] = 0;
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
#pragma unroll
        for (int i = 0; i < NW; i++) {
          // candidates: wanted bits this edge brings that no earlier round had;
          // most rounds have none, and then nothing changes
          const W c = f[u][i] & want[i] & ~acc[i];
          if (!__any_sync(0xffffffffu, c != 0)) continue;
          W grp;
          W claim = first_bits<W>(c, 0, &grp);
          if (hpar == nullptr) claim = 0;  // caller searches these parents later
          while (claim) {
            const int b = ffs0(claim);
            hpar[idx * ROW + i * B + b] = col[u];
            claim &= claim - 1;
          }
          acc[i] |= grp;
        }
      }
      scanned += (unsigned long long)imin64(32 * U, end - base);
      bool done = true;
#pragma unroll
      for (int i = 0; i < NW; i++) done = done && ((acc[i] & want[i]) == want[i]);
      if (done) break;
    }
    W nw[NW];
    bool has = false;
#pragma unroll
    for (int i = 0; i < NW; i++) {
      nw[i] = lane == 0 ? (acc[i] & want[i]) : (W)0;
      has = has || nw[i] != 0;
    }
    if (has) {
#pragma unroll
      for (int i = 0; i < NW; i++) N[(int64_t)v * NW + i] = nw[i];
    }
    commit_new<W, NW, OffT>(has, v, nw, sw, end - beg, level, seen, pl, active, heavy, nl, nctr, sacc);
  }
  flush_stats<W, NW>(sacc, nctr, &ctr->b);
  if (lane == 0 && vcount) {
    atomicAdd(&ctr->b.edges_scanned, scanned);
    atomicAdd(&ctr->b.vertices_scanned, vcount);
  }
}

// Pull, hubs (degree > hub): one warp per (heavy index, chunk) item, no early
// exit; found bits go to N[v] with atomicOr and each bit's first neighbour in
// the chunk to hpar with atomicMin (hpar rows start at INT32_MAX), so the
// smallest id over all chunks wins.  k_pull_hub_commit then records them.
template <typename W, int NW, typename OffT, int U>
__global__ void k_pull_hubs(const int32_t* __restrict__ hlist, const int2* __restrict__ items, int64_t nitems,
                            const OffT* __restrict__ ro, const int32_t* __restrict__ ci, const W* __restrict__ F,
                            const W* __restrict__ seen, W* N, Masks<W, NW> active, Ctrs* ctr, int cur, int chunk,
                            int32_t* __restrict__ hpar, int64_t n, const uint32_t* __restrict__ fbits) {
  constexpr int B = WB<W>::bits;
  constexpr int ROW = B * NW;
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  LevelCtr* cctr = &ctr->lv[cur];
  W live[NW];
#pragma unroll
  for (int i = 0; i < NW; i++) live[i] = (W)cctr->live[i] & active.w[i];
  unsigned long long scanned = 0;
  const uint32_t* fb = sparse_bits(fbits, cctr, n);
  for (int64_t it = warp; it < nitems; it += nwarps) {
    const int2 item = items[it];
    const int64_t idx = item.x;
    const int32_t v = hlist[idx];
    W sw[NW], want[NW];
    load_words<W, NW>(seen + (int64_t)v * NW, sw);
    bool any = false;
#pragma unroll
    for (int i = 0; i < NW; i++) {
      want[i] = live[i] & ~sw[i];
      any = any || want[i] != 0;
    }
    if (!any) continue;  // warp-uniform
    const int64_t end = ro[v + 1];
    const int64_t cb = (int64_t)ro[v] + (int64_t)item.y * chunk;
    const int64_t ce = imin64(end, cb + chunk);
    W acc[NW];
#pragma unroll
    for (int i = 0; i < NW; i++) acc[i] = 0;
    for (int64_t base = cb; base < ce; base += 32 * U) {
      int32_t col[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int64_t e = base + u * 32 + lane;
        col[u] = e < ce ? __ldcs(&ci[e]) : -1;
      }
      W f[U][NW];
#pragma unroll
      for (int u = 0; u < U; u++) {
        if (col[u] >= 0 && in_frontier(fb, col[u])) {
          load_words<W, NW>(F + (int64_t)col[u] * NW, f[u]);
        } else {
#pragma unroll
          for (int i = 0; i < NW; i++) f[u][i] = 0;
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
#pragma unroll
        for (int i = 0; i < NW; i++) {
          const W c = f[u][i] & want[i] & ~acc[i];
          if (!__any_sync(0xffffffffu, c != 0)) continue;
          W grp;
          W claim = first_bits<W>(c, 0, &grp);
          while (claim) {
            const int b = ffs0(claim);
            atomicMin(&hpar[idx * ROW + i * B + b], col[u]);
            claim &= claim - 1;
          }
          acc[i] |= grp;
        }
      }
      scanned += (unsigned long long)imin64(32 * U, ce - base);
    }
    if (lane == 0) {
#pragma unroll
      for (int i = 0; i < NW; i++) {
        const W found = acc[i] & want[i];
        if (found) atomicOr(&N[(int64_t)v * NW + i], found);
      }
    }
  }
  if (lane == 0 && scanned) atomicAdd(&ctr->b.edges_scanned, scanned);
}

// Records the level's new bits of the hubs (after k_pull_hubs).
template <typename W, int NW, typename OffT>
__global__ void k_pull_hub_commit(const int32_t* __restrict__ hlist, int32_t nh, const OffT* __restrict__ ro,
                                  W* seen, const W* N, Planes<W, NW> pl, Masks<W, NW> active, int heavy,
                                  int hub, Lists nl, Ctrs* ctr, int cur) {
  const int level = ctr->b.level;
  LevelCtr* nctr = &ctr->lv[cur ^ 1];
  StatAcc<W, NW> sacc;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < nh; base += stride) {
    const int64_t idx = base + threadIdx.x;
    int32_t v = 0;
    int64_t dg = 0;
    bool has = false;
    W nw[NW], sw[NW];
#pragma unroll
    for (int i = 0; i < NW; i++) nw[i] = sw[i] = 0;
    if (idx < nh) {
      v = hlist[idx];
      dg = deg_of(ro, v);
      if (dg > hub) {
#pragma unroll
        for (int i = 0; i < NW; i++) {
          nw[i] = N[(int64_t)v * NW + i];
          sw[i] = seen[(int64_t)v * NW + i];
          has = has || nw[i] != 0;
        }
      }
    }
    commit_new<W, NW, OffT>(has, v, nw, sw, dg, level, seen, pl, active, heavy, nl, nctr, sacc);
  }
  flush_stats<W, NW>(sacc, nctr, &ctr->b);
}

// Zeroes F at the vertices of a frontier list.
template <typename W, int NW>
__global__ void k_clear_list(const int32_t* __restrict__ list, const int32_t* __restrict__ count, W* F) {
  const int32_t cnt = *count;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)cnt * NW;
       i += (int64_t)gridDim.x * blockDim.x)
    F[(int64_t)list[i / NW] * NW + (i % NW)] = 0;
}

template <typename T>
__global__ void k_fill(T* p, int64_t count, T value) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = value;
}

// ---------------------------------------------------------------------------
// Table pass of a pass of kb sources (wsrc[0..kb)), all its words.  For word
// wi, rows[wi*2B + s] and rows[wi*2B + B + s] are the level and parent rows (n
// int32 each) of its source s, so the sources of one word may belong to
// different queries and output buffers.
//
// The vertex's own level classes: root = the vertex is the source (level 0 is
// the only level with every plane bit clear); lvl1 = level exactly 1, whose
// only possible parent is the source itself.
// Neighbours per vertex the table pass keeps in shared memory for the
// recorded-position lookups.
constexpr int kCiCache = 8;

// 8x8 bit-matrix transpose (Hacker's Delight, 2nd ed., section 7-3): bit
// 8r + c moves to bit 8c + r.
__device__ __forceinline__ unsigned long long transpose8(unsigned long long x) {
  unsigned long long t;
  t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
  x ^= t ^ (t << 7);
  t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
  x ^= t ^ (t << 14);
  t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
  x ^= t ^ (t << 28);
  return x;
}

// Half h (0 = low) of a word, as 32 bits.
template <typename W>
__device__ __forceinline__ uint32_t half32(W x, int h) {
  if constexpr (sizeof(W) == 4) {
    return (uint32_t)x;
  } else {
    return (uint32_t)(h ? (x >> 32) : x);
  }
}

// Byte bb of each of a, b, c, d in bytes 0..3; sel = bb | (bb + 4) << 4.
__device__ __forceinline__ uint32_t gather4(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t sel) {
  return __byte_perm(__byte_perm(a, b, sel), __byte_perm(c, d, sel), 0x5410);
}

// transpose8 on the 64-bit value hi:lo, in 32-bit operations.
__device__ __forceinline__ void transpose8x8(uint32_t& lo, uint32_t& hi) {
  uint32_t t;
  t = (lo ^ (lo >> 7)) & 0x00AA00AAu;
  lo ^= t ^ (t << 7);
  t = (hi ^ (hi >> 7)) & 0x00AA00AAu;
  hi ^= t ^ (t << 7);
  t = (lo ^ (lo >> 14)) & 0x0000CCCCu;
  lo ^= t ^ (t << 14);
  t = (hi ^ (hi >> 14)) & 0x0000CCCCu;
  hi ^= t ^ (t << 14);
  t = (lo ^ ((lo >> 28) | (hi << 4))) & 0xF0F0F0F0u;
  lo ^= t ^ (t << 28);
  hi ^= t >> 4;
}

// Byte b of each of 8 words, word r landing in byte r.
template <typename W>
__device__ __forceinline__ unsigned long long gather_bytes8(const W (&p)[8], int b) {
  unsigned long long x = 0;
#pragma unroll
  for (int r = 0; r < 8; r++) x |= (unsigned long long)((p[r] >> (8 * b)) & 0xFF) << (8 * r);
  return x;
}

template <typename W, int NW>
__device__ __forceinline__ void vertex_levels(const W* __restrict__ seen, const Planes<W, NW>& pl, int nplanes,
                                              int64_t v, int wi, W& sv, W& p0, W& p1, W& root, W& lvl1) {
  sv = seen[v * NW + wi];
  W pr[2];
  load_words<W, 2>(pl.p01 + ((v * NW + wi) << 1), pr);
  p0 = pr[0];
  p1 = pr[1];
  W hi = 0;
  for (int j = 2; j < nplanes; j++) hi |= pl.get(j, v, wi);
  root = sv & ~(p0 | p1 | hi);
  lvl1 = sv & p0 & ~p1 & ~hi;
}

// Per-source digest of a traversal row (serving results without tables).
struct RowDigest {
  unsigned long long reached;    // vertices with level >= 0
  unsigned long long level_sum;  // sum of their levels
  unsigned long long row_hash;   // sum of row_entry_hash over them (mod 2^64)
  unsigned int depth;            // largest level
  unsigned int pad;
};

// Hash of one (vertex, level, parent) entry: the splitmix64 finalizer
// (Steele, Lea, Flood 2014) of the vertex id times the golden-ratio constant
// XOR the (level, parent) pair packed into 64 bits.
__host__ __device__ __forceinline__ unsigned long long row_entry_hash(int64_t v, int32_t level, int32_t parent) {
  unsigned long long z = (unsigned long long)v * 0x9E3779B97F4A7C15ull;
  z ^= ((unsigned long long)(uint32_t)level << 32) | (unsigned long long)(uint32_t)parent;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// One warp per 32-vertex tile.  Parents of bits reached by a pull step come
// from the recorded p8 index (ci[ro[v] + p8[v][s]]).
//
// DIG: every row of the pass is digest-only and nothing is stored (the row
// pointers are not used).  Each (vertex, source) entry adds to its source's
// RowDigest instead: warp reductions over the tile's 32 vertices per source,
// entries whose parent is searched added by the search itself, block totals
// in shared memory, one set of global atomics per block and source (dig[row]
// must be zero at launch).  The sums equal k_row_digest's over the rows the
// plain variant would have written.  Bits reached by a push
// step (and every bit of a vertex whose degree exceeds 256) are searched:
// rounds over the flattened, still-needed adjacency (ascending within each
// vertex), U x 32 edges per round, loads issued up front; a segmented
// exclusive prefix OR in edge order hands each needed bit to its first
// (= smallest-id) matching neighbour.
template <typename W, int NW, typename OffT, int WARPS, int U, bool DIG = false>
__global__ void __launch_bounds__(WARPS * 32, (DIG ? 20 : 24) / WARPS) k_tables(int64_t n, const OffT* __restrict__ ro,
                                                       const int32_t* __restrict__ ci, const W* __restrict__ seen,
                                                       Planes<W, NW> pl, int kb, int heavy,
                                                       int32_t* const* __restrict__ rows, Ctrs* ctr,
                                                       const W* __restrict__ ppos, const W* __restrict__ pushed,
                                                       const int32_t* __restrict__ wsrc,
                                                       const int32_t* __restrict__ hidx_of,
                                                       const int32_t* __restrict__ hpar,
                                                       RowDigest* __restrict__ dig = nullptr) {
  constexpr int B = WB<W>::bits;
  constexpr int ROW = B * NW;
  const int nplanes = ctr->b.nplanes;
  __shared__ int32_t s_src[NW][B];
  __shared__ int32_t* s_row[NW][2][B];
  // DIG: block totals per source (reached, level sum, hash sum; depth)
  __shared__ unsigned long long s_dsum[DIG ? NW * B : 1][3];
  __shared__ unsigned int s_ddep[DIG ? NW * B : 1];
  for (int j = threadIdx.x; j < NW * B; j += blockDim.x) {
    const int w = j / B, s = j % B;
    s_src[w][s] = j < kb ? wsrc[j] : -1;
    s_row[w][0][s] = j < kb ? rows[w * 2 * B + s] : nullptr;
    s_row[w][1][s] = j < kb ? rows[w * 2 * B + B + s] : nullptr;
    if constexpr (DIG) {
      s_dsum[j][0] = s_dsum[j][1] = s_dsum[j][2] = 0;
      s_ddep[j] = 0;
    }
  }
  __syncthreads();
  const int nwords = (kb + B - 1) / B;
  __shared__ int32_t s_off[WARPS][33];
  __shared__ int64_t s_pos[WARPS][32];
  __shared__ W s_need[WARPS][32];
  __shared__ W s_t0[WARPS][32];
  __shared__ W s_t1[WARPS][32];
  __shared__ W s_found[WARPS][32];
  __shared__ int32_t s_ci[WARPS][32][kCiCache + 1];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int64_t ntiles = (n + 31) >> 5;
  const int64_t warp = (int64_t)blockIdx.x * WARPS + wib;
  const int64_t nwarps = (int64_t)gridDim.x * WARPS;
  unsigned long long pe = 0;
  for (int64_t tile = warp; tile < ntiles; tile += nwarps) {
   // the words of a tile back to back: their vertex words share sectors
   for (int wi = 0; wi < nwords; wi++) {
    const int kbw = min(B, kb - wi * B);
    const int64_t v = tile * 32 + lane;
    const bool valid = v < n;
    // a tile no source of this word reached (isolated vertices, small
    // components): every entry is -1, nothing else to read; in other tiles
    // an unreached lane skips its loads the same way
    const bool reached = valid && seen[v * NW + wi] != 0;
    if (!__any_sync(0xffffffffu, reached)) {
      if constexpr (!DIG) {
        if (valid) {
#pragma unroll 4
          for (int s = 0; s < kbw; s++) {
            __stcs(&s_row[wi][0][s][v], -1);
            __stcs(&s_row[wi][1][s][v], -1);
          }
        }
      }
      continue;
    }
    W sv = 0, p0 = 0, p1 = 0, root = 0, lvl1 = 0;
    int64_t beg = 0, dg = 0;
    if (reached) {
      vertex_levels<W, NW>(seen, pl, nplanes, v, wi, sv, p0, p1, root, lvl1);
      beg = ro[v];
      dg = (int64_t)ro[v + 1] - beg;
    }
    const bool is_heavy = dg > heavy;
    const bool has_p8 = dg <= kP8MaxDegree;
    W pw = 0;
    if (reached && !is_heavy && has_p8) pw = pushed[v * NW + wi];
    // bits whose parent must be searched (level-1 bits: the source itself)
    const W need = (valid && !is_heavy) ? (sv & ~root & ~lvl1 & (has_p8 ? pw : ~(W)0)) : (W)0;
    s_need[wib][lane] = need;
    s_t0[wib][lane] = ~p0;         // bit-sliced (level - 1) mod 4, plane 0
    s_t1[wib][lane] = ~(p0 ^ p1);  // plane 1
    s_found[wib][lane] = 0;
    int64_t pos = beg;
    const int64_t end = beg + dg;
    __syncwarp();
    for (;;) {
      const W fnd = s_found[wib][lane];
      const int32_t r = (need & ~fnd) ? (int32_t)(end - pos) : 0;
      int32_t inc = r;
#pragma unroll
      for (int s = 1; s < 32; s <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, inc, s);
        if (lane >= s) inc += y;
      }
      const int32_t total = __shfl_sync(0xffffffffu, inc, 31);
      if (total == 0) break;
      const int32_t off = inc - r;
      s_off[wib][lane] = off;
      if (lane == 31) s_off[wib][32] = inc;
      s_pos[wib][lane] = pos;
      __syncwarp();
      const int32_t take = total < 32 * U ? total : 32 * U;
      int key[U];
      int32_t col[U];
      W q0[U], q1[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int32_t e = u * 32 + lane;
        key[u] = 32 + lane;
        col[u] = -1;
        if (e < take) {
          const int o = flat_owner(s_off[wib], e);
          key[u] = o;
          col[u] = __ldcs(&ci[s_pos[wib][o] + (e - s_off[wib][o])]);
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        q0[u] = q1[u] = 0;
        if (col[u] >= 0) {
          W pr[2];
          load_words<W, 2>(pl.p01 + (((int64_t)col[u] * NW + wi) << 1), pr);
          q0[u] = pr[0];
          q1[u] = pr[1];
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int k = key[u];
        const bool act = k < 32;
        W eq = 0;
        if (act) eq = ~(q0[u] ^ s_t0[wib][k]) & ~(q1[u] ^ s_t1[wib][k]) & s_need[wib][k];
        W incl = eq;
#pragma unroll
        for (int s = 1; s < 32; s <<= 1) {
          const W y = shfl_up<W>(incl, s);
          const int k2 = __shfl_up_sync(0xffffffffu, k, s);
          if (lane >= s && k2 == k) incl |= y;
        }
        const W prev = shfl_up<W>(incl, 1);
        const int kprev = __shfl_up_sync(0xffffffffu, k, 1);
        const W excl = (lane > 0 && kprev == k) ? prev : (W)0;
        const int knext = __shfl_down_sync(0xffffffffu, k, 1);
        const bool tail = (lane == 31) || (knext != k);
        if (act) {
          // first match of each needed bit: the parent goes straight to its
          // row (the row pass below leaves these entries alone)
          W mine = eq & ~excl & ~s_found[wib][k];
          while (mine) {
            const int b = ffs0(mine);
            if constexpr (DIG) {
              // digest-only rows: this entry's digest terms, its level read
              // from the owner's planes (the row pass below skips it)
              const int64_t vk = tile * 32 + k;
              int32_t lvl = 0;
              for (int j = 0; j < nplanes; j++) lvl |= (int32_t)((pl.get(j, vk, wi) >> b) & 1) << j;
              const int jrow = wi * B + b;
              atomicAdd(&s_dsum[jrow][0], 1ull);
              atomicAdd(&s_dsum[jrow][1], (unsigned long long)lvl);
              atomicAdd(&s_dsum[jrow][2], row_entry_hash(vk, lvl, col[u]));
              atomicMax(&s_ddep[jrow], (unsigned)lvl);
            } else {
              __stcs(&s_row[wi][1][b][tile * 32 + k], col[u]);
            }
            mine &= mine - 1;
          }
        }
        __syncwarp();
        if (act && tail) s_found[wib][k] |= incl;
        __syncwarp();
      }
      // advance this lane's vertex by the edges the round consumed
      int32_t used = take - off;
      used = used < 0 ? 0 : (used > r ? r : used);
      pos += used;
      if (lane == 0) pe += (unsigned long long)take;
      __syncwarp();
    }
    // write rows: level and parent of sources 0..kbw-1 at vertices tile*32 + lane.
    // Every lane runs the decode (it holds a warp vote); lanes past n load and
    // store nothing.
    {
      constexpr int RP = 8;  // planes decoded by transposes; deeper levels read on demand
      // parent sources: recorded position (light, pulled; bit-sliced in 8
      // planes), recorded id (heavy), searched (written above), the source
      // itself (levels 0 and 1)
      const bool use_pp = reached && !is_heavy && has_p8;
      const W* prow = ppos + (v * NW + wi) * 8;
      const int32_t* hrow = is_heavy ? hpar + (int64_t)hidx_of[v] * ROW + wi * B : nullptr;
      // the first kCiCache neighbours of the vertex: most recorded positions
      // point there (the first frontier neighbour of a large frontier)
      int32_t* cic = s_ci[wib][lane];
      if (use_pp) {
#pragma unroll
        for (int j = 0; j < kCiCache; j++) cic[j] = j < dg ? __ldg(&ci[beg + j]) : -1;
      }
      // Eight sources at a time, per 32-bit half of the words: the level bytes
      // and position bytes of sources 8b..8b+7 come from byte permutes of the
      // 8 plane halves and an 8x8 bit transpose; the parent is the cached
      // neighbour at the recorded position.  Rarer classes (the source itself,
      // level 1, heavy rows, positions beyond the cache) are patched only when
      // some lane of the warp has one.  Searched bits (need) already hold
      // their parent.
      const bool deep = nplanes > RP;
      constexpr int HALVES = (int)sizeof(W) / 4;
#pragma unroll 1
      for (int h = 0; h < HALVES; h++) {
        if (h * 32 >= kbw) break;
        // 32-bit halves of the level planes and position planes
        uint32_t L[8], P[8];
        L[0] = half32<W>(p0, h);
        L[1] = half32<W>(p1, h);
#pragma unroll
        for (int j = 2; j < RP; j++)
          L[j] = (reached && j < nplanes)
                     ? reinterpret_cast<const uint32_t*>(pl.ph + (int64_t)(j - 2) * pl.stride + v * NW + wi)[h]
                     : 0u;
#pragma unroll
        for (int r = 0; r < 8; r++) P[r] = use_pp ? reinterpret_cast<const uint32_t*>(prow + r)[h] : 0u;
        const uint32_t sv32 = half32<W>(sv, h), rt32 = half32<W>(root, h), l132 = half32<W>(lvl1, h);
        const uint32_t nd32 = half32<W>(need, h);
        // recorded positions >= kCiCache (a bit in position planes 3..7)
        const uint32_t far32 = (P[3] | P[4] | P[5] | P[6] | P[7]) & sv32 & ~(nd32 | rt32 | l132);
        const bool rare = __any_sync(0xffffffffu, (rt32 | l132 | far32) != 0 || hrow != nullptr);
#pragma unroll 1
        for (int bb = 0; bb < 4; bb++) {
          const int sb = h * 32 + bb * 8;
          if (sb >= kbw) break;
          const uint32_t sel = (uint32_t)bb | ((uint32_t)(bb + 4) << 4);
          uint32_t llo = gather4(L[0], L[1], L[2], L[3], sel), lhi = gather4(L[4], L[5], L[6], L[7], sel);
          transpose8x8(llo, lhi);
          uint32_t plo = 0, phi = 0;
          if (use_pp) {
            plo = gather4(P[0], P[1], P[2], P[3], sel);
            phi = gather4(P[4], P[5], P[6], P[7], sel);
            transpose8x8(plo, phi);
          }
          const uint32_t svb = (sv32 >> (8 * bb)) & 0xFFu, ndb = (nd32 >> (8 * bb)) & 0xFFu;
          int32_t lv[8], pr[8];
#pragma unroll
          for (int i = 0; i < 8; i++) {
            const uint32_t lw = i < 4 ? llo : lhi, pw = i < 4 ? plo : phi;
            lv[i] = (int32_t)((lw >> (8 * (i & 3))) & 0xFFu);
            pr[i] = cic[(pw >> (8 * (i & 3))) & (kCiCache - 1)];
          }
          if (rare) {
            const uint32_t rtb = (rt32 >> (8 * bb)) & 0xFFu, l1b = (l132 >> (8 * bb)) & 0xFFu;
            const uint32_t farb = (far32 >> (8 * bb)) & 0xFFu;
#pragma unroll
            for (int i = 0; i < 8; i++) {
              const uint32_t pw = i < 4 ? plo : phi;
              if (((farb >> i) & 1) && !hrow) pr[i] = __ldg(&ci[beg + ((pw >> (8 * (i & 3))) & 0xFFu)]);
              if (hrow && sb + i < kbw) pr[i] = hrow[sb + i];
              if ((l1b >> i) & 1) pr[i] = s_src[wi][sb + i];
              if ((rtb >> i) & 1) pr[i] = (int32_t)v;
            }
          }
          if (deep) {
#pragma unroll
            for (int i = 0; i < 8; i++)
              if ((svb >> i) & 1)
                for (int j = RP; j < nplanes; j++) lv[i] |= (int32_t)((pl.get(j, v, wi) >> (sb + i)) & 1) << j;
          }
          if constexpr (DIG) {
#pragma unroll
            for (int i = 0; i < 8; i++) {
              const int s = sb + i;
              // searched entries were added by the search above
              const bool hit = s < kbw && valid && ((svb >> i) & 1) && !((ndb >> i) & 1);
              const unsigned long long hsh = hit ? row_entry_hash(v, lv[i], pr[i]) : 0ull;
              const unsigned lvu = hit ? (unsigned)lv[i] : 0u;
              // 32-bit warp reductions; the 64-bit sums are rebuilt from
              // pieces that cannot overflow over 32 lanes
              const unsigned cnt = __popc(__ballot_sync(0xffffffffu, hit));
              const unsigned l0 = __reduce_add_sync(0xffffffffu, lvu & 0xFFFFu);
              const unsigned l1 = __reduce_add_sync(0xffffffffu, lvu >> 16);
              const unsigned dm = __reduce_max_sync(0xffffffffu, lvu);
              const unsigned h0 = __reduce_add_sync(0xffffffffu, (unsigned)(hsh & 0xFFFFu));
              const unsigned h1 = __reduce_add_sync(0xffffffffu, (unsigned)((hsh >> 16) & 0xFFFFu));
              const unsigned h2 = __reduce_add_sync(0xffffffffu, (unsigned)(hsh >> 32));
              if (lane == i && cnt) {
                const int j = wi * B + s;
                atomicAdd(&s_dsum[j][0], (unsigned long long)cnt);
                atomicAdd(&s_dsum[j][1], (unsigned long long)l0 + ((unsigned long long)l1 << 16));
                atomicAdd(&s_dsum[j][2], (unsigned long long)h0 + ((unsigned long long)h1 << 16) +
                                             ((unsigned long long)h2 << 32));
                atomicMax(&s_ddep[j], dm);
              }
            }
          } else {
#pragma unroll
            for (int i = 0; i < 8; i++) {
              const int s = sb + i;
              if (s < kbw && valid) {
                const bool hit = (svb >> i) & 1;
                __stcs(&s_row[wi][0][s][v], hit ? lv[i] : -1);
                if (!((ndb >> i) & 1)) __stcs(&s_row[wi][1][s][v], hit ? pr[i] : -1);
              }
            }
          }
        }
      }
    }
    __syncwarp();
   }
  }
  pe = warp_sum_u64(pe);
  if (lane == 0 && pe) atomicAdd(&ctr->b.parent_edges, pe);
  if constexpr (DIG) {
    __syncthreads();
    for (int j = threadIdx.x; j < kb; j += blockDim.x) {
      if (s_dsum[j][0] == 0) continue;
      atomicAdd(&dig[j].reached, s_dsum[j][0]);
      atomicAdd(&dig[j].level_sum, s_dsum[j][1]);
      atomicAdd(&dig[j].row_hash, s_dsum[j][2]);
      atomicMax(&dig[j].depth, s_ddep[j]);
    }
  }
}

// Table pass for heavy vertices, scan step, for the bits a push step reached
// at level >= 2 (the pull steps recorded every other parent in hpar): the
// blocks walk a per-graph list of (heavy index, chunk) items, each chunk
// `chunk` edges of one adjacency.  Each block hands every needed bit to the
// first matching neighbour of its chunk (block-wide exclusive prefix OR in
// edge order) and folds it into hpar[idx*ROW + wi*B + bit] with atomicMin, so
// the smallest id over all chunks wins regardless of schedule.  Those hpar
// slots still hold the INT32_MAX written at the start of the pass.
template <typename W, int NW, typename OffT>
__global__ void __launch_bounds__(256) k_tables_heavy_scan(const int32_t* __restrict__ hlist,
                                                           const int2* __restrict__ items, int64_t nitems,
                                                           const OffT* __restrict__ ro, const int32_t* __restrict__ ci,
                                                           const W* __restrict__ seen, Planes<W, NW> pl, int wi,
                                                           int chunk, int32_t* hpar, Ctrs* ctr,
                                                           const W* __restrict__ pushed) {
  constexpr int B = WB<W>::bits;
  constexpr int ROW = B * NW;
  if (!ctr->b.pushed_deep) return;  // no push step reached level >= 2: nothing to search
  const int nplanes = ctr->b.nplanes;
  __shared__ W s_wor[8];
  __shared__ W s_claimed;
  __shared__ int32_t s_items[32];
  __shared__ int s_nitems;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  // groups of 32 items: the first warp checks them for needed bits at once,
  // the block then walks only the items that have some (after a push step
  // only few items have any, and a walk pays a dependent-load latency per
  // item); groups small enough that every block gets some
  for (int64_t gbase = (int64_t)blockIdx.x * 32; gbase < nitems; gbase += (int64_t)gridDim.x * 32) {
   {
    if (threadIdx.x == 0) s_nitems = 0;
    __syncthreads();
    const int64_t it = gbase + threadIdx.x;
    bool has = false;
    if (threadIdx.x < 32 && it < nitems) {
      const int64_t v = hlist[items[it].x];
      W sv, p0, p1, root, lvl1;
      vertex_levels<W, NW>(seen, pl, nplanes, v, wi, sv, p0, p1, root, lvl1);
      has = (sv & ~root & ~lvl1 & pushed[v * NW + wi]) != 0;
    }
    if (has) s_items[atomicAdd(&s_nitems, 1)] = (int32_t)threadIdx.x;
    __syncthreads();
   }
   const int nlisted = s_nitems;
   for (int li = 0; li < nlisted; li++) {
    const int2 item = items[gbase + s_items[li]];
    const int64_t idx = item.x;
    const int64_t v = hlist[idx];
    W sv, p0, p1, root, lvl1;
    vertex_levels<W, NW>(seen, pl, nplanes, v, wi, sv, p0, p1, root, lvl1);
    const W need = sv & ~root & ~lvl1 & pushed[v * NW + wi];
    const W t0 = ~p0, t1 = ~(p0 ^ p1);
    const int64_t beg = ro[v], end = ro[v + 1];
    const int64_t c0 = beg + (int64_t)item.y * chunk;
    for (int64_t cb = c0; cb < end && cb < c0 + chunk; cb += chunk) {  // one chunk
      const int64_t ce = imin64(end, cb + chunk);
      if (threadIdx.x == 0) s_claimed = 0;
      __syncthreads();
      unsigned long long pe = 0;
      for (int64_t base = cb; base < ce; base += 4 * 256) {
        int32_t col[4];
        W q0[4], q1[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int64_t e = base + u * 256 + threadIdx.x;
          col[u] = e < ce ? __ldcs(&ci[e]) : -1;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          q0[u] = q1[u] = 0;
          if (col[u] >= 0) {
            W pr[2];
            load_words<W, 2>(pl.p01 + (((int64_t)col[u] * NW + wi) << 1), pr);
            q0[u] = pr[0];
            q1[u] = pr[1];
          }
        }
        bool all_done = false;
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const W claimed = s_claimed;
          const W eq = col[u] >= 0 ? (~(q0[u] ^ t0) & ~(q1[u] ^ t1) & need & ~claimed) : (W)0;
          W incl = eq;
#pragma unroll
          for (int s = 1; s < 32; s <<= 1) {
            const W y = shfl_up<W>(incl, s);
            if (lane >= s) incl |= y;
          }
          if (lane == 31) s_wor[wid] = incl;
          __syncthreads();
          W before = 0, all = 0;
#pragma unroll
          for (int k = 0; k < 8; k++) {
            const W x = s_wor[k];
            if (k < wid) before |= x;
            all |= x;
          }
          W lp = shfl_up<W>(incl, 1);
          const W excl = before | (lane ? lp : (W)0);
          W mine = eq & ~excl;
          while (mine) {
            const int b = ffs0(mine);
            atomicMin(&hpar[idx * ROW + wi * B + b], col[u]);
            mine &= mine - 1;
          }
          __syncthreads();
          if (threadIdx.x == 0) s_claimed = claimed | all;
          __syncthreads();
          all_done = ((claimed | all) & need) == need;
        }
        pe += (unsigned long long)imin64(4 * 256, ce - base);
        if (all_done) break;  // later edges of this chunk have larger ids
      }
      if (threadIdx.x == 0) atomicAdd(&ctr->b.parent_edges, pe);
      __syncthreads();
    }
   }
   __syncthreads();  // s_items / s_nitems are rewritten by the next group
  }
}

// ---------------------------------------------------------------------------
// Level-loop control.  The same single-thread kernels drive the host loop of
// xb_traverse (which reads the decision back) and the device loop of
// xb_traverse_batched (which feeds it to conditional nodes of a CUDA graph).

// Resets the counters of a pass; the unfinished-edge estimate starts at m.
static __global__ void k_pass_init(Ctrs* ctr, long long m) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  LevelCtr z{};
  ctr->lv[0] = z;
  ctr->lv[1] = z;
  BatchCtr b{};
  b.m_unfinished = m;
  b.nplanes = 3;  // planes 0-2 are cleared with the pass
  b.zero_plane = -1;
  ctr->b = b;
}

// Decides the next step from the current frontier's counters lv[cur]:
// dir = 0 push, 1 pull (frontier edges * alpha > unfinished edges), 2 done.
// After a pull step, a frontier of fewer than push_below vertices is pushed
// (0 = never): the tail of a traversal, where a pull would still sweep every
// light vertex for a handful of frontier vertices.
// Advances the level, picks the level plane to clear, bumps the stamp epoch
// and zeroes the next frontier's counters.  A frontier still alive at
// level_bound stops the loop with the error flag set.
static __global__ void k_step_begin(Ctrs* ctr, int cur, float alpha, int nplanes_alloc, int level_bound,
                                    int graph_mode, cudaGraphConditionalHandle hswitch, long long push_below = 0) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  BatchCtr& b = ctr->b;
  const LevelCtr& lc = ctr->lv[cur];
  int dir = 2;
  b.step_calls += 1;
  b.zero_plane = -1;  // k_zero_plane runs after every decision in a graph, "done" included
  // a traversal has at most n <= 2^nplanes_alloc levels; a frontier still alive
  // beyond that (or beyond a lower bound the caller set) means corrupted
  // state: stop the loop and flag it
  const bool alive = (long long)lc.n_light + lc.n_heavy > 0;
  if (b.dir != 2 && b.err == 0 && alive && b.level >= level_bound) b.err = 2;
  if (b.dir != 2 && b.err == 0 && alive) {
    dir = ((double)lc.edges * (double)alpha > (double)b.m_unfinished) ? 1 : 0;
    if (dir == 1 && b.dir == 1 && (long long)lc.n_light + lc.n_heavy < push_below) dir = 0;
    b.level += 1;
    if (b.nplanes < nplanes_alloc && (1 << b.nplanes) <= b.level) {
      b.zero_plane = b.nplanes;
      b.nplanes += 1;
    }
    if (dir == 0) {
      b.push_levels += 1;
      if (b.level >= 2) b.pushed_deep = 1;
    } else {
      b.pull_levels += 1;
    }
    ctr->epoch += 1;
    LevelCtr z{};
    ctr->lv[cur ^ 1] = z;
  }
  b.dir = dir;
  if (graph_mode) cudaGraphSetConditional(hswitch, (unsigned)dir);
}

// Clears the level plane k_step_begin picked (planes >= 3 live in ph).
template <typename W>
__global__ void k_zero_plane(W* ph, int64_t stride, int64_t words, const Ctrs* ctr) {
  const int zp = ctr->b.zero_plane;
  if (zp < 3) return;
  W* p = ph + (int64_t)(zp - 2) * stride;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = 0;
}

// Zeroes the consumed frontier after a pull step: the listed vertices when
// the frontier is small, the whole array otherwise.
template <typename W, int NW>
__global__ void k_clear_frontier(W* F, int64_t n, Lists fl, const Ctrs* ctr, int cur) {
  const int32_t nlight = ctr->lv[cur].n_light, nheavy = ctr->lv[cur].n_heavy;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (fl.bits)
    for (int64_t i = tid; i < (n + 31) / 32; i += stride) fl.bits[i] = 0;
  if (((int64_t)nlight + nheavy) * 16 < n) {
    for (int64_t i = tid; i < ((int64_t)nlight + nheavy) * NW; i += stride) {
      const int64_t j = i / NW;
      const int32_t v = j < nlight ? fl.light[j] : fl.heavy[j - nlight];
      F[(int64_t)v * NW + (i % NW)] = 0;
    }
  } else {
    for (int64_t i = tid; i < n * NW; i += stride) F[i] = 0;
  }
}

// After the second step of a loop body: keep looping while the traversal has
// a frontier.
static __global__ void k_loop_end(const Ctrs* ctr, int cur_next, cudaGraphConditionalHandle hwhile) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const bool more = ctr->b.dir != 2 && ctr->b.err == 0 &&
                    (long long)ctr->lv[cur_next].n_light + ctr->lv[cur_next].n_heavy > 0;
  cudaGraphSetConditional(hwhile, more ? 1u : 0u);
}

// Algorithmic bytes of a pass's level steps: the row-offset pair (R bytes) of
// every scanned vertex, colIndices + the gathered frontier words of every
// scanned edge, and a three-word sweep (seen read, seen and next-frontier
// write) of every swept vertex.  wsz = bytes per word, nw = words per vertex.
__host__ __device__ inline long long level_bytes_of(const BatchCtr& b, int R, int wsz, int nw) {
  const long long wb = (long long)wsz * nw;
  return (long long)R * (long long)b.vertices_scanned + (4 + wb) * (long long)b.edges_scanned +
         3 * wb * (long long)b.vertices_swept;
}

// Algorithmic bytes of a pass's table pass: per vertex its row offsets, seen,
// level planes and parent-position planes (per word), the colIndices entry of
// every recorded parent, colIndices + gathered plane pair of every searched
// edge, and the two written tables (kb rows of n int32 each).
__host__ __device__ inline long long table_bytes_of(const BatchCtr& b, long long n, int kb, int R, int wsz, int nw) {
  return (long long)nw * n * (R + (long long)wsz * (1 + b.nplanes + 8)) + 4 * (long long)b.reached +
         (4 + 2 * (long long)wsz) * (long long)b.parent_edges + 8 * (long long)kb * n;
}

// Per-call totals over passes (device).
struct PassSum {
  unsigned long long edges_traversed, reached, edges_scanned, vertices_scanned, vertices_swept, parent_edges;
  unsigned long long level_bytes, table_bytes;
  unsigned long long launches;  // kernels the passes ran (graph mode)
  int32_t max_level, push_levels, pull_levels, passes;
  int32_t errors;  // passes that ended with BatchCtr::err set
  int32_t pad;
};

// Folds a finished pass (n vertices, kb sources; R, wsz, nw as in
// level_bytes_of) into the totals.  Kernel count of a pass run by a graph:
// fixed_k outside the level loop (this one included), two per step decision
// (k_step_begin, k_zero_plane), one k_loop_end per two decisions, and push_k /
// pull_k per push / pull step.
static __global__ void k_pass_accum(const Ctrs* ctr, PassSum* sum, long long n, int kb, int R, int wsz, int nw,
                                    int fixed_k, int push_k, int pull_k) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const BatchCtr& b = ctr->b;
  sum->launches += (unsigned long long)(fixed_k + 2 * b.step_calls + b.step_calls / 2 + push_k * b.push_levels +
                                        pull_k * b.pull_levels);
  sum->level_bytes += (unsigned long long)level_bytes_of(b, R, wsz, nw);
  sum->table_bytes += (unsigned long long)table_bytes_of(b, n, kb, R, wsz, nw);
  sum->edges_traversed += b.edges_traversed;
  sum->reached += b.reached;
  sum->edges_scanned += b.edges_scanned;
  sum->vertices_scanned += b.vertices_scanned;
  sum->vertices_swept += b.vertices_swept;
  sum->parent_edges += b.parent_edges;
  if (b.level > sum->max_level) sum->max_level = b.level;  // levels with a non-empty frontier
  sum->push_levels += b.push_levels;
  sum->pull_levels += b.pull_levels;
  sum->passes += 1;
  if (b.err) sum->errors += 1;
}

// ---------------------------------------------------------------------------
// FIFO parents: the parent rule of a sequential FIFO breadth-first search
// (xblossom::Graph::findShortestPath, apps/xb/src/include/graph/xgraph.h:155-191):
// a vertex's parent is the first dequeued vertex adjacent to it, and a
// level's queue is ordered by (place of the parent in its own level's queue,
// place in the parent's adjacency).  Computed after the traversal from the
// finished level row, one block per source, level by level:
//   keys    every frontier vertex (queue rank r; one warp per vertex) offers r
//           to its next-level neighbours with atomicMin, in the parent row
//   counts  children of rank r = next-level neighbours whose key is r
//   scan    block-wide exclusive scan of the counts: first child's rank
//   queue   each frontier vertex writes its children in adjacency order
//           (warp ballots); then the keys become parent ids
// The adjacency must hold no duplicate entries.  work: 3*n int32 per block
// (two queues and the counts).

// Exclusive prefix sum of a[0..len) in place over the whole block; returns
// the total to every thread.
__device__ __forceinline__ int64_t block_exclusive_scan(int32_t* a, int64_t len) {
  __shared__ int32_t s_w[32];
  __shared__ int64_t s_carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < len; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    const int32_t x = i < len ? a[i] : 0;
    int32_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      int32_t t = lane < nwarps ? s_w[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += y;
      }
      if (lane < nwarps) s_w[lane] = t;
    }
    __syncthreads();
    const int64_t carry = s_carry;
    if (i < len) a[i] = (int32_t)(carry + (warp > 0 ? s_w[warp - 1] : 0) + incl - x);
    __syncthreads();
    if (threadIdx.x == 0) s_carry = carry + s_w[nwarps - 1];
    __syncthreads();
  }
  return s_carry;
}

// Block b handles source j = j0 + b of the pass (rows in the table pass
// layout: word j/B, level row rows[wi*2B + j%B], parent row rows[wi*2B + B +
// j%B]).  The parent row holds the traversal's parents on entry (the source
// its own parent, -1 unreached); levels >= 1 are rewritten.
template <typename OffT>
__global__ void __launch_bounds__(1024) k_fifo_parents(int64_t n, const OffT* __restrict__ ro,
                                                       const int32_t* __restrict__ ci, int32_t* const* __restrict__ rows,
                                                       int B, int j0, int kb, const int32_t* __restrict__ src,
                                                       int32_t* work, int64_t wstride) {
  const int j = j0 + (int)blockIdx.x;
  if (j >= kb) return;  // block-uniform
  const int wi = j / B, b = j % B;
  const int32_t* lv = rows[wi * 2 * B + b];
  int32_t* pr = rows[wi * 2 * B + B + b];
  int32_t* q0 = work + (int64_t)blockIdx.x * wstride;
  int32_t* q1 = q0 + n;
  int32_t* cnt = q1 + n;
  __shared__ int64_t s_qn;
  for (int64_t v = threadIdx.x; v < n; v += blockDim.x)
    if (lv[v] >= 1) pr[v] = INT32_MAX;
  if (threadIdx.x == 0) {
    q0[0] = src[j];
    s_qn = 1;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int32_t d = 0;; d++) {
    const int64_t qn = s_qn;
    if (qn == 0) break;  // block-uniform
    for (int64_t r = warp; r < qn; r += nwarps) {  // keys
      const int32_t u = q0[r];
      const int64_t end = ro[u + 1];
      for (int64_t e = (int64_t)ro[u] + lane; e < end; e += 32) {
        const int32_t w = ci[e];
        if (lv[w] == d + 1) atomicMin(&pr[w], (int32_t)r);
      }
    }
    __syncthreads();
    for (int64_t r = warp; r < qn; r += nwarps) {  // counts
      const int32_t u = q0[r];
      const int64_t end = ro[u + 1];
      int32_t c = 0;
      for (int64_t e = (int64_t)ro[u] + lane; e < end; e += 32) {
        const int32_t w = ci[e];
        c += (lv[w] == d + 1 && pr[w] == (int32_t)r) ? 1 : 0;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
      if (lane == 0) cnt[r] = c;
    }
    __syncthreads();
    const int64_t total = block_exclusive_scan(cnt, qn);
    for (int64_t r = warp; r < qn; r += nwarps) {  // next queue, children in adjacency order
      const int32_t u = q0[r];
      const int64_t beg = ro[u], end = ro[u + 1];
      int64_t pos = cnt[r];
      for (int64_t e0 = beg; e0 < end; e0 += 32) {
        const int64_t e = e0 + lane;
        int32_t w = 0;
        bool hit = false;
        if (e < end) {
          w = ci[e];
          hit = lv[w] == d + 1 && pr[w] == (int32_t)r;
        }
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (hit) q1[pos + __popc(m & ((1u << lane) - 1u))] = w;
        pos += __popc(m);
      }
    }
    __syncthreads();
    for (int64_t i = threadIdx.x; i < total; i += blockDim.x) {  // keys -> parent ids
      const int32_t w = q1[i];
      pr[w] = q0[pr[w]];
    }
    __syncthreads();
    int32_t* t = q0;
    q0 = q1;
    q1 = t;
    if (threadIdx.x == 0) s_qn = total;
    __syncthreads();
  }
}

// Digest of one table row pair (level row, parent row of a source): the
// summary a serving client gets instead of the full tables.  row_hash is
// position-sensitive: the wrapping sum over reached vertices v of
// row_entry_hash(v, level[v], parent[v]), so moving a parent or a level from
// one vertex to another changes it, while the sum keeps it independent of the
// order the GPU visits the vertices in.
// Digests of the pass rows the flags mark; rows are in the table pass layout
// (word wi: level rows at rows[wi*2B + b], parent rows at rows[wi*2B + B + b]).
// blockIdx.y = row within the pass; out[row] must be zero beforehand.
static __global__ void __launch_bounds__(256) k_row_digest(int32_t* const* __restrict__ rows,
                                                          const int32_t* __restrict__ flags, int kb, int B,
                                                          int64_t n, RowDigest* out) {
  const int r = blockIdx.y;
  if (r >= kb || !flags[r]) return;
  const int wi = r / B, b = r % B;
  const int32_t* lv = rows[wi * 2 * B + b];
  const int32_t* pr = rows[wi * 2 * B + B + b];
  unsigned long long cnt = 0, ls = 0, hs = 0;
  unsigned int dep = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t l = __ldcs(&lv[i]);
    if (l >= 0) {
      cnt++;
      ls += (unsigned long long)l;
      hs += row_entry_hash(i, l, __ldcs(&pr[i]));
      dep = max(dep, (unsigned int)l);
    }
  }
  cnt = warp_sum_u64(cnt);
  ls = warp_sum_u64(ls);
  hs = warp_sum_u64(hs);
  for (int o = 16; o > 0; o >>= 1) dep = max(dep, __shfl_xor_sync(0xffffffffu, dep, o));
  if ((threadIdx.x & 31) == 0 && cnt) {
    atomicAdd(&out[r].reached, cnt);
    atomicAdd(&out[r].level_sum, ls);
    atomicAdd(&out[r].row_hash, hs);
    atomicMax(&out[r].depth, dep);
  }
}

// Per vertex v, the sum of its neighbours' degrees (the CSR entries a
// traversal from v reads at its second level): the tie-break of the pass
// grouping by source degree.  Warp per vertex; the loop bound is uniform
// over the warp, so the shuffle reduction runs with every lane.
template <typename OffT>
__global__ void k_reach2(int64_t n, const OffT* __restrict__ ro, const int32_t* __restrict__ ci,
                         long long* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
    const int64_t b = (int64_t)ro[v], e = (int64_t)ro[v + 1];
    long long s = 0;
    for (int64_t i = b + lane; i < e; i += 32) {
      const int32_t u = ci[i];
      s += (long long)(ro[u + 1] - ro[u]);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) out[v] = s;
  }
}

}  // namespace xbk
