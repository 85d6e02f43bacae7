// xb_match.cu -- maximum-cardinality matching on a resident graph: the
// traversal core in alternating mode (xb_max_match).
//
// The reference's search phase (apps/xb/src/xblsm_gpu/xblossom_gpu_engine_10.cu:72-80
// and the CPU engine apps/xb/src/xblsm_cpu/par_pro_pernode.cu:42-90) grows an
// alternating forest from all exposed vertices at once, flips the
// vertex-disjoint augmenting paths it finds between trees, handles blossoms
// inside a tree, and repeats until a search finds no augmenting path.  This
// file does the same with Edmonds' blossom rule (J. Edmonds, "Paths, trees,
// and flowers", 1965) in a forest:
//
//  - the first phase starts a fresh forest (every exposed vertex an outer
//    root); a later phase keeps the trees that flipped nothing and restarts
//    from all their outer vertices (the reference engines reuse trees the
//    same way, xblossom_gpu_engine_10.cu:83-166);
//  - a level expands all outer frontier vertices (edge-balanced chunks of
//    the frontier's adjacency, xb_partition.cuh):
//      * a matched pair (w, mate w) not in any tree is claimed by one CAS on
//        the state word of min(w, mate w): w becomes inner (pred = v), its
//        mate outer and part of the next frontier;
//      * an outer neighbour in another tree closes an augmenting path: the
//        two trees are locked (two exchanges, released on failure -- no
//        waiting) and the edge recorded, so recorded paths are vertex
//        disjoint;
//      * an outer neighbour of the same tree in another blossom is a
//        blossom candidate, linked into a per-tree list;
//  - after a level with augmenting paths, every recorded path is flipped
//    (thread per path); the flipped trees keep their locks and drop out, the
//    other trees keep growing in the same phase (so a phase gathers a large
//    set of disjoint paths, as a Hopcroft-Karp phase does);
//  - the candidates of the live trees are contracted, one thread per tree
//    walking its list: the cycle's top is the first common blossom base on the two
//    paths to the root, `pred` of the outer vertices on the cycle is
//    rerouted across it (so a later augmenting path can be read back
//    through the blossom), the bases are merged into the top (union-find),
//    and the inner vertices on the cycle become outer frontier vertices;
//  - a phase whose frontier runs empty without any two trees meeting proves
//    the matching maximum (no lock was tried, so no edge was skipped).
//
// State word per vertex: -1 outside the forest, else root * 4 + label
// (1 outer, 2 inner), written in one store so a reader sees a whole state.
// A reader that finds a pair half claimed skips it: if the vertex is outer
// it will scan the edge itself on the next level.  Every walk over tree or
// blossom pointers is bounded by n steps and reports XB_ERR_STATE on
// overrun instead of looping.
#include "xb_engine_common.cuh"
#include "xb_partition.cuh"

using xbi::fail;

namespace {

constexpr int32_t kOuter = 1, kInner = 2;

__device__ __forceinline__ int32_t mm_state(int32_t root, int32_t label) { return root * 4 + label; }

// Blossom base of x with path halving (only the owning tree's thread writes).
__device__ __forceinline__ int32_t mm_find(int32_t* base, int32_t x, int64_t n, int32_t* err) {
  for (int64_t i = 0; i <= n; i++) {
    const int32_t b = base[x];
    if (b == x) return x;
    const int32_t bb = base[b];
    base[x] = bb;
    x = bb;
  }
  atomicExch(err, 1);
  return x;
}

// Read-only base lookup for the expand kernel (bases do not change there).
__device__ __forceinline__ int32_t mm_find_ro(const int32_t* base, int32_t x, int64_t n) {
  for (int64_t i = 0; i <= n; i++) {
    const int32_t b = base[x];
    if (b == x) return x;
    x = b;
  }
  return -1;
}

template <typename OffT>
__global__ void k_mm_check(int64_t n, const OffT* __restrict__ ro, const int32_t* __restrict__ ci,
                           const int32_t* __restrict__ mate, int32_t* bad) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t m = mate[v];
    if (m == -1) continue;
    if (m < 0 || m >= n || m == v || mate[m] != v) {
      atomicAdd(bad, 1);
      continue;
    }
    int64_t lo = ro[v], hi = ro[v + 1];  // sorted adjacency: is m a neighbour?
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (ci[mid] < m) lo = mid + 1;
      else hi = mid;
    }
    if (lo == (int64_t)ro[v + 1] || ci[lo] != m) atomicAdd(bad, 1);
  }
}

template <typename OffT>
__global__ void k_mm_init(int64_t n, const OffT* __restrict__ ro, const int32_t* __restrict__ mate, int32_t* st,
                          int32_t* pred, int32_t* base, int32_t* lock, int32_t* head, int32_t* front,
                          int32_t* fcount) {
  // warp-uniform rounds, so the frontier appends go out one atomic per warp
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t b0 = (int64_t)blockIdx.x * blockDim.x; b0 < n; b0 += stride) {
    const int64_t v = b0 + threadIdx.x;
    bool app = false;
    if (v < n) {
      const bool has_edge = ro[v + 1] > ro[v];
      const bool exposed = mate[v] < 0;
      st[v] = exposed ? mm_state((int32_t)v, kOuter) : -1;
      pred[v] = -1;
      base[v] = (int32_t)v;
      lock[v] = 0;
      head[v] = -1;
      app = exposed && has_edge;  // isolated roots grow nothing
    }
    xbk::warp_append(app, (int32_t)v, front, fcount);
  }
}

// Next phase from the current forest: the trees whose augmenting paths were
// flipped (locked roots) dissolve -- their vertices, all matched now, leave
// the forest -- and every other tree stays as it is (labels, pred, blossom
// bases); all outer vertices of the kept trees form the first frontier, so
// the search re-examines every edge of the forest against the vertices that
// just became free.  The locks are cleared afterwards (separate memset).
template <typename OffT>
__global__ void k_mm_reinit(int64_t n, const OffT* __restrict__ ro, int32_t* st, int32_t* pred, int32_t* base,
                            const int32_t* __restrict__ lock, int32_t* head, int32_t* front, int32_t* fcount) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t b0 = (int64_t)blockIdx.x * blockDim.x; b0 < n; b0 += stride) {
    const int64_t v = b0 + threadIdx.x;
    bool app = false;
    if (v < n) {
      head[v] = -1;
      const int32_t sv = st[v];
      if (sv != -1) {
        if (lock[sv >> 2]) {
          st[v] = -1;
          pred[v] = -1;
          base[v] = (int32_t)v;
        } else {
          app = (sv & 3) == kOuter && ro[v + 1] > ro[v];
        }
      }
    }
    xbk::warp_append(app, (int32_t)v, front, fcount);  // one atomic per warp
  }
}

// Counters of one forest level (cleared at its start).
struct MmLevel {
  int32_t found, cand, err;
  int32_t attempts;  // set when an edge between two trees tried the locks
  unsigned long long scanned;
};

// Totals of one phase, accumulated by k_mm_level_end (cleared per phase).
struct MmPhase {
  unsigned long long scanned;
  int64_t found, levels, blossom_levels;
  int32_t attempted, err;
};

constexpr int kExpandWarps = 4;                  // warps per expand block
constexpr int kAppCap = 2 * xbp::kChunk;         // per-warp buffer of grown outer vertices

// One level: the frontier's adjacency entries in chunks of xbp::kChunk, one
// chunk per warp iteration (lane l of step it takes chunk entry 32 * it + l;
// the owner of an entry comes from the chunk's mask of entry starts).  Outer
// vertices grown by pair claims gather in the warp's buffer and go out with
// one atomic per flush.
template <typename OffT>
__global__ void __launch_bounds__(32 * kExpandWarps) k_mm_expand(
    const int32_t* __restrict__ front, const int64_t* __restrict__ eoff, const int64_t* __restrict__ ebase,
    const int32_t* __restrict__ chunk_first, const int64_t* __restrict__ edges_p,
    const int64_t* __restrict__ nchunks_p, const int32_t* __restrict__ fcount_p, const int32_t* __restrict__ ci,
    const int32_t* __restrict__ mate, int32_t* st, int32_t* pred, const int32_t* __restrict__ base, int32_t* lock,
    int32_t* next, int32_t* next_count, int2* found, int2* cand, int32_t* cand_next, int32_t* head,
    int64_t cand_cap, int64_t n, MmLevel* lv) {
  constexpr int kItems = xbp::kItems, kChunk = xbp::kChunk;
  __shared__ OffT s_base_all[kExpandWarps][kChunk + 1];   // spanned entry: column-index position minus eoff
  __shared__ int32_t s_v_all[kExpandWarps][kChunk + 1];   // spanned entry: its vertex
  __shared__ uint32_t s_mask_all[kExpandWarps][kItems];   // bit e: a spanned entry starts at chunk edge e
  __shared__ int32_t s_app_all[kExpandWarps][kAppCap];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  OffT* s_base = s_base_all[wib];
  int32_t* s_v = s_v_all[wib];
  uint32_t* s_mask = s_mask_all[wib];
  int32_t* s_app = s_app_all[wib];
  const uint32_t le_mask = (2u << lane) - 1u;
  const int64_t E = *edges_p, nchunks = *nchunks_p;
  const int32_t fcount = *fcount_p;
  const int64_t gw = (int64_t)blockIdx.x * kExpandWarps + wib, nw = (int64_t)gridDim.x * kExpandWarps;
  int32_t napp = 0;  // warp-uniform
  for (int64_t c = gw; c < nchunks; c += nw) {
    const int64_t E0 = c * kChunk;
    const int32_t len = (int32_t)min((int64_t)kChunk, E - E0);
    const int32_t vlo = chunk_first[c];
    const int32_t vhi = c + 1 < nchunks ? chunk_first[c + 1] : fcount - 1;
    const int32_t nv = vhi - vlo + 1;
    __syncwarp();
    if (lane < kItems) s_mask[lane] = 0u;
    __syncwarp();
    int32_t rel0 = 0;
    for (int32_t j = lane; j < nv; j += 32) {
      const int64_t rel = eoff[vlo + j] - E0;
      s_base[j] = (OffT)ebase[vlo + j];
      s_v[j] = front[vlo + j];
      if (j == 0) rel0 = (int32_t)max(rel, (int64_t)-1);
      if (rel >= 0 && rel < kChunk) atomicOr(&s_mask[rel >> 5], 1u << (rel & 31));
    }
    __syncwarp();
    int32_t run = (__shfl_sync(0xffffffffu, rel0, 0) < 0 ? 1 : 0) - 1;
    int32_t vv[kItems], w[kItems];
#pragma unroll
    for (int it = 0; it < kItems; it++) {
      const uint32_t m = s_mask[it];
      const int32_t e = 32 * it + lane;
      const int32_t j = run + __popc(m & le_mask);
      run += __popc(m);
      vv[it] = -1;
      w[it] = 0;
      if (e < len) {
        vv[it] = s_v[j];
        w[it] = ci[(int64_t)s_base[j] + E0 + e];
      }
    }
    int32_t sw[kItems], mv[kItems];
#pragma unroll
    for (int it = 0; it < kItems; it++) {
      sw[it] = vv[it] >= 0 ? *(volatile int32_t*)&st[w[it]] : -2;
      mv[it] = vv[it] >= 0 ? mate[vv[it]] : -1;
    }
#pragma unroll
    for (int it = 0; it < kItems; it++) {
      bool grow = false;
      int32_t grown = 0;
      const int32_t v = vv[it];
      // a locked tree holds an augmenting path of this phase (or is being
      // tried for one right now): its vertices take no further part
      const int32_t rv = v >= 0 ? st[v] >> 2 : 0;  // outer, stable during the level
      if (v >= 0 && w[it] != mv[it] && sw[it] != -2 && *(volatile int32_t*)&lock[rv] == 0) {
        if (sw[it] == -1) {
          const int32_t mw = mate[w[it]];
          if (mw >= 0) {
            const int32_t lk = min(w[it], mw), other = max(w[it], mw);
            const int32_t lab_lk = lk == w[it] ? kInner : kOuter;
            if (atomicCAS(&st[lk], -1, mm_state(rv, lab_lk)) == -1) {
              pred[w[it]] = v;
              st[other] = mm_state(rv, lab_lk == kInner ? kOuter : kInner);
              grow = true;
              grown = mw;
            }
          }
        } else if ((sw[it] & 3) == kOuter && *(volatile int32_t*)&lock[sw[it] >> 2] == 0) {
          const int32_t rw = sw[it] >> 2;
          if (rw != rv) {
            lv->attempts = 1;
            const int32_t a = min(rv, rw), b = max(rv, rw);
            if (atomicExch(&lock[a], 1) == 0) {
              if (atomicExch(&lock[b], 1) == 0) {
                const int32_t k = atomicAdd(&lv->found, 1);
                found[k] = make_int2(v, w[it]);
              } else {
                atomicExch(&lock[a], 0);
              }
            }
          } else {
            const int32_t bv = mm_find_ro(base, v, n), bw = mm_find_ro(base, w[it], n);
            if (bv < 0 || bw < 0) {
              atomicExch(&lv->err, 1);
            } else if (bv != bw) {
              const int32_t k = atomicAdd(&lv->cand, 1);
              if (k < cand_cap) {
                cand[k] = make_int2(v, w[it]);
                cand_next[k] = atomicExch(&head[rv], k);
              } else {
                atomicExch(&lv->err, 2);
              }
            }
          }
        }
      }
      const unsigned bal = __ballot_sync(0xffffffffu, grow);
      if (grow) s_app[napp + __popc(bal & (le_mask >> 1))] = grown;
      napp += __popc(bal);
    }
    if (napp > kAppCap - kChunk || c + nw >= nchunks) {  // room for one more chunk, or the warp's last chunk
      __syncwarp();
      int32_t basei = 0;
      if (lane == 0 && napp) basei = atomicAdd(next_count, napp);
      basei = __shfl_sync(0xffffffffu, basei, 0);
      for (int32_t i = lane; i < napp; i += 32) next[basei + i] = s_app[i];
      napp = 0;
    }
  }
}

// Flips the recorded augmenting paths (their trees are disjoint).
__device__ __forceinline__ bool mm_flip_walk(int32_t u, int32_t pu, int32_t* mate, const int32_t* pred, int64_t n) {
  for (int64_t i = 0; i <= n; i++) {
    const int32_t old = mate[pu];
    mate[u] = pu;
    mate[pu] = u;
    if (old < 0) return true;
    u = old;
    pu = pred[u];
    if (pu < 0) return false;
  }
  return false;
}

__global__ void k_mm_flip(const int2* __restrict__ found, const int32_t* __restrict__ nfound_p, int32_t* mate,
                          const int32_t* __restrict__ pred, int64_t n, MmLevel* lv) {
  const int32_t nfound = *nfound_p;
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nfound; i += gridDim.x * blockDim.x) {
    const int32_t v = found[i].x, w = found[i].y;
    const int32_t ow = mate[w];
    bool ok = mm_flip_walk(w, v, mate, pred, n);  // w joins v; v's side up to its root
    if (ok && ow >= 0) {
      const int32_t p = pred[ow];
      ok = p >= 0 && mm_flip_walk(ow, p, mate, pred, n);  // w's old mate up to w's root
    }
    if (!ok) atomicExch(&lv->err, 3);
  }
}

// Contracts the blossom candidates; the thread holding a tree's list head
// processes that tree's whole list.
__global__ void k_mm_blossom(const int2* __restrict__ cand, const int32_t* __restrict__ ncand_p,
                             const int32_t* __restrict__ cand_next, int32_t* head, int32_t* st,
                             const int32_t* __restrict__ mate, int32_t* pred, int32_t* base, int32_t* stamp,
                             int32_t* tick, const int32_t* __restrict__ lock, int32_t* next, int32_t* next_count,
                             int64_t n, MmLevel* lv) {
  const int32_t ncand = *ncand_p;
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ncand; i += gridDim.x * blockDim.x) {
    const int32_t r = st[cand[i].x] >> 2;
    if (head[r] != i) continue;
    if (lock[r]) {  // the tree's augmenting path was flipped this level: it is out of the phase
      head[r] = -1;
      continue;
    }
    int32_t* err = &lv->err;
    int64_t guard = 0;
    for (int32_t c = i; c >= 0; c = cand_next[c]) {
      if (++guard > ncand) {
        atomicExch(err, 4);
        break;
      }
      const int32_t v = cand[c].x, w = cand[c].y;
      if (mm_find(base, v, n, err) == mm_find(base, w, n, err)) continue;
      const int32_t t = atomicAdd(tick, 1) + 1;
      // top: the first base on w's path that v's path to the root also meets
      int32_t a = v, top = -1;
      for (int64_t s = 0; s <= n; s++) {
        a = mm_find(base, a, n, err);
        stamp[a] = t;
        if (mate[a] < 0) break;
        a = pred[mate[a]];
        if (a < 0) break;
      }
      int32_t b = w;
      for (int64_t s = 0; s <= n; s++) {
        b = mm_find(base, b, n, err);
        if (stamp[b] == t) {
          top = b;
          break;
        }
        if (mate[b] < 0) break;
        b = pred[mate[b]];
        if (b < 0) break;
      }
      if (top < 0) {
        atomicExch(err, 5);
        return;
      }
      // reroute pred across the cycle, counting the steps of each side
      int64_t steps[2] = {0, 0};
      for (int side = 0; side < 2; side++) {
        int32_t x = side ? w : v, across = side ? v : w;
        while (mm_find(base, x, n, err) != top) {
          const int32_t m = mate[x];
          if (m < 0 || steps[side] > n) {
            atomicExch(err, 6);
            return;
          }
          pred[x] = across;
          across = m;
          x = pred[m];
          steps[side]++;
        }
      }
      // merge the cycle's bases into the top; its inner vertices turn outer
      for (int side = 0; side < 2; side++) {
        int32_t x = side ? w : v;
        for (int64_t s = 0; s < steps[side]; s++) {
          const int32_t m = mate[x];
          const int32_t bx = mm_find(base, x, n, err), bm = mm_find(base, m, n, err);
          base[bx] = top;
          base[bm] = top;
          base[top] = top;
          if ((st[m] & 3) == kInner) {
            st[m] = mm_state(r, kOuter);
            next[atomicAdd(next_count, 1)] = m;
          }
          x = pred[m];
        }
      }
    }
    head[r] = -1;
  }
}

// Level control for the device-side loop: clear the level's counters and
// the output frontier's count; afterwards fold them into the phase totals
// and decide whether the WHILE loop takes another level.
__global__ void k_mm_level_begin(int32_t* next_count, MmLevel* lv) {
  *next_count = 0;
  lv->found = lv->cand = lv->err = lv->attempts = 0;
  lv->scanned = 0;
}

__global__ void k_mm_level_end(const int32_t* __restrict__ in_count, const int32_t* __restrict__ next_count,
                               const MmLevel* __restrict__ lv, MmPhase* ph, int64_t level_cap, int in_graph,
                               cudaGraphConditionalHandle loop) {
  if (*in_count > 0) {
    ph->levels++;
    ph->scanned += lv->scanned;
    ph->found += lv->found;
    ph->blossom_levels += lv->cand > 0;
    ph->attempted |= lv->attempts;
    ph->err |= lv->err;
  }
  if (ph->levels > level_cap) ph->err |= 8;
  if (in_graph) cudaGraphSetConditional(loop, (*next_count > 0 && ph->err == 0) ? 1u : 0u);
}

struct MmWork {
  int32_t *st, *pred, *base, *lock, *head, *stamp, *front[2], *cand_next, *tick, *fcnt, *chunk_first;
  int2 *found, *cand;
  int64_t *eoff, *ebase, *tsum, *scal;
  MmLevel *lv, *sticky;  // per-level counters; errors of the flips (cleared per call)
  MmPhase* ph;
};

// One forest level on stream s from front[cur] into front[cur ^ 1], every
// count read on the device (so the same launches serve the captured loop).
template <typename OffT>
void emit_level(const MmWork& wk, const xb_graph* g, int32_t* d_mate, int64_t cand_cap, int cur, int max_tiles,
                int expand_grid, int sms, cudaStream_t s, xbe::ClassTimer* timer = nullptr) {
  const OffT* ro = (const OffT*)g->d_ro;
  const int64_t n = g->n;
  int32_t* in_cnt = wk.fcnt + cur;
  int32_t* out_cnt = wk.fcnt + (cur ^ 1);
  // classes when timed: 2 = control and partition, 0 = expansion, 1 = flips and blossoms
  if (timer) timer->begin();
  k_mm_level_begin<<<1, 1, 0, s>>>(out_cnt, wk.lv);
  xbp::k_lb_tile_sums<OffT><<<max_tiles, xbp::kThreads, 0, s>>>(wk.front[cur], in_cnt, ro, wk.tsum);
  xbp::k_lb_tile_scan<<<1, 1024, 0, s>>>(wk.tsum, in_cnt, wk.scal, wk.scal + 1, &wk.lv->scanned);
  xbp::k_lb_offsets<OffT><<<max_tiles, xbp::kThreads, 0, s>>>(wk.front[cur], in_cnt, ro, wk.tsum, wk.eoff, wk.ebase,
                                                               wk.chunk_first);
  if (timer) {
    timer->end(2, 4);
    timer->begin();
  }
  k_mm_expand<OffT><<<expand_grid, 32 * kExpandWarps, 0, s>>>(
      wk.front[cur], wk.eoff, wk.ebase, wk.chunk_first, wk.scal, wk.scal + 1, in_cnt, g->d_ci, d_mate, wk.st, wk.pred,
      wk.base, wk.lock, wk.front[cur ^ 1], out_cnt, wk.found, wk.cand, wk.cand_next, wk.head, cand_cap, n, wk.lv);
  if (timer) {
    timer->end(0, 1);
    timer->begin();
  }
  // flips first: their trees stay locked, so the blossom pass skips them
  k_mm_flip<<<sms * 4, 128, 0, s>>>(wk.found, &wk.lv->found, d_mate, wk.pred, n, wk.sticky);
  k_mm_blossom<<<sms * 8, 128, 0, s>>>(wk.cand, &wk.lv->cand, wk.cand_next, wk.head, wk.st, d_mate, wk.pred, wk.base,
                                       wk.stamp, wk.tick, wk.lock, wk.front[cur ^ 1], out_cnt, n, wk.lv);
  if (timer) timer->end(1, 2);
}

// The level loop of one phase as a graph: a WHILE node whose body takes a
// level from front[0] into front[1] and one back; k_mm_level_end keeps the
// loop going while the next frontier is not empty.
template <typename OffT>
xb_status capture_phase_loop(const MmWork& wk, const xb_graph* g, int32_t* d_mate, int64_t cand_cap, int max_tiles,
                             int expand_grid, int sms, cudaStream_t s, cudaStream_t body, cudaGraphExec_t* exec) {
  XB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
  cudaGraphConditionalHandle h;
  xb_status st = xbe::make_handle(s, 1, cudaGraphCondAssignDefault, &h);
  cudaGraph_t wbody = nullptr;
  if (st == XB_OK) st = xbe::add_conditional(s, h, cudaGraphCondTypeWhile, 1, &wbody);
  if (st == XB_OK) {
    if (cudaStreamBeginCaptureToGraph(body, wbody, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
      st = fail(XB_ERR_CUDA, "matching: body capture failed to start");
    } else {
      for (int cur = 0; cur < 2; cur++) {
        emit_level<OffT>(wk, g, d_mate, cand_cap, cur, max_tiles, expand_grid, sms, body);
        k_mm_level_end<<<1, 1, 0, body>>>(wk.fcnt + cur, wk.fcnt + (cur ^ 1), wk.lv, wk.ph, g->n + 1, 1, h);
      }
      if (cudaGetLastError() != cudaSuccess) st = fail(XB_ERR_CUDA, "matching: a captured launch failed");
      st = xbe::end_body(body, st);
    }
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &graph);
  if (st == XB_OK && e != cudaSuccess) st = fail(XB_ERR_CUDA, std::string("matching capture: ") + cudaGetErrorString(e));
  if (st == XB_OK && cudaGraphInstantiate(exec, graph, 0) != cudaSuccess) {
    cudaGetLastError();
    st = fail(XB_ERR_CUDA, "matching: graph instantiation failed");
  }
  if (graph) cudaGraphDestroy(graph);
  return st;
}

template <typename OffT>
xb_status run_match(xb_ctx* c, xb_graph* g, int32_t* d_mate, const MmWork& wk, int64_t cand_cap, xb_stats* st) {
  cudaStream_t s = c->stream;
  const int64_t n = g->n;
  const OffT* ro = (const OffT*)g->d_ro;
  const int sms = c->num_sms;
  const int vgrid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8));
  const int max_tiles = (int)((n + xbp::kTile - 1) / xbp::kTile);
  MmPhase* h = (MmPhase*)c->h_ctr;  // pinned host scratch
  static_assert(sizeof(MmPhase) + 2 * sizeof(int32_t) <= sizeof(xbk::Ctrs), "pinned scratch too small");
  int32_t* h_cnt = (int32_t*)(h + 1);
  int expand_per_sm = 0;
  XB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&expand_per_sm, k_mm_expand<OffT>, 32 * kExpandWarps, 0));
  const int expand_grid = sms * std::max(expand_per_sm, 1);
  // per-class timing needs a host-driven loop (events around each launch);
  // otherwise each phase's levels run as one captured WHILE loop
  const bool timed = c->tuning.timing != 0;
  xbe::ClassTimer timer{c, st, timed};
  cudaStream_t body = nullptr;
  cudaGraphExec_t exec = nullptr;
  struct Cleanup {
    cudaStream_t& b;
    cudaGraphExec_t& e;
    ~Cleanup() {
      if (e) cudaGraphExecDestroy(e);
      if (b) cudaStreamDestroy(b);
    }
  } cleanup{body, exec};
  if (!timed) {
    XB_CUDA(cudaStreamCreateWithFlags(&body, cudaStreamNonBlocking));
    xb_status cs = capture_phase_loop<OffT>(wk, g, d_mate, cand_cap, max_tiles, expand_grid, sms, s, body, &exec);
    if (cs != XB_OK) return cs;
  }
  int64_t phases = 0, levels = 0, blossom_levels = 0, flips = 0, idle_phases = 0, launches = 0;
  unsigned long long scanned = 0;
  bool reuse = false;  // next phase keeps the trees that flipped nothing
  for (;;) {
    if (phases > n / 2 + 1) return fail(XB_ERR_STATE, "matching: phase bound exceeded");
    phases++;
    XB_CUDA(cudaMemsetAsync(wk.fcnt, 0, 2 * sizeof(int32_t), s));
    XB_CUDA(cudaMemsetAsync(wk.ph, 0, sizeof(MmPhase), s));
    timer.begin();
    if (!reuse) {
      k_mm_init<OffT><<<vgrid, 256, 0, s>>>(n, ro, d_mate, wk.st, wk.pred, wk.base, wk.lock, wk.head, wk.front[0],
                                            wk.fcnt);
    } else {
      k_mm_reinit<OffT><<<vgrid, 256, 0, s>>>(n, ro, wk.st, wk.pred, wk.base, wk.lock, wk.head, wk.front[0], wk.fcnt);
      XB_CUDA(cudaMemsetAsync(wk.lock, 0, sizeof(int32_t) * (size_t)n, s));
    }
    XB_LAUNCH_CHECK("matching init");
    timer.end(2, 1);
    if (!timed) {
      XB_CUDA(cudaGraphLaunch(exec, s));
    } else {
      // the same levels, one by one from the host
      XB_CUDA(cudaMemcpyAsync(h_cnt, wk.fcnt, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      XB_CUDA(cudaStreamSynchronize(s));
      int cur = 0;
      for (int64_t lvl = 0; h_cnt[0] > 0; lvl++) {
        if (lvl > n) return fail(XB_ERR_STATE, "matching: level bound exceeded");
        emit_level<OffT>(wk, g, d_mate, cand_cap, cur, max_tiles, expand_grid, sms, s, &timer);
        k_mm_level_end<<<1, 1, 0, s>>>(wk.fcnt + cur, wk.fcnt + (cur ^ 1), wk.lv, wk.ph, n + 1, 0, 0);
        XB_LAUNCH_CHECK("matching level");
        launches++;
        XB_CUDA(cudaMemcpyAsync(h_cnt, wk.fcnt + (cur ^ 1), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        XB_CUDA(cudaStreamSynchronize(s));
        cur ^= 1;
      }
    }
    XB_CUDA(cudaMemcpyAsync(h, wk.ph, sizeof(MmPhase), cudaMemcpyDeviceToHost, s));
    XB_CUDA(cudaMemcpyAsync(h_cnt, &wk.sticky->err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    XB_CUDA(cudaStreamSynchronize(s));
    if (h->err) return fail(XB_ERR_STATE, "matching: inconsistent forest (" + std::to_string(h->err) + ")");
    if (h_cnt[0]) return fail(XB_ERR_STATE, "matching: flip walk failed");
    levels += h->levels;
    if (!timed) {  // kernels the graph ran: 8 per level, levels in pairs (an odd count runs one empty level)
      const int64_t L = h->levels;
      launches += 8 * (L == 0 ? 2 : L + (L & 1));
    }
    blossom_levels += h->blossom_levels;
    scanned += h->scanned;
    flips += h->found;
    if (h->found > 0) {
      idle_phases = 0;
      reuse = true;
      continue;
    }
    // No path flipped.  A search in which no two trees ever met proves the
    // matching maximum; one whose lock attempts all gave way is repeated
    // from a fresh forest.
    if (!h->attempted) break;
    reuse = false;
    if (++idle_phases > 64) return fail(XB_ERR_STATE, "matching: searches keep failing to lock their paths");
  }
  if (st) {
    st->batches = (int32_t)std::min<int64_t>(phases, INT32_MAX);
    st->levels = (int32_t)std::min<int64_t>(levels, INT32_MAX);
    st->pull_levels = (int32_t)std::min<int64_t>(blossom_levels, INT32_MAX);
    st->edges_scanned = (int64_t)scanned;
    st->edges_traversed = (int64_t)scanned;
    st->vertices_scanned = flips;
    st->class_launches[0] += launches;  // the level kernels (timed runs count them per class instead)
    // algorithmic bytes of the expansion: a column index and the neighbour's state word per scanned entry
    st->class_bytes[0] = (int64_t)scanned * 8;
    st->algo_bytes = st->class_bytes[0];
  }
  return XB_OK;
}

template <typename T>
T* carve_ints(char*& p, int64_t count) {
  T* r = (T*)p;
  p += ((sizeof(T) * (size_t)std::max<int64_t>(count, 1) + 255) / 256) * 256;
  return r;
}

}  // namespace

extern "C" {

xb_status xb_max_match(xb_ctx* c, const xb_graph* gc, int32_t* mate, uint32_t flags, xb_stats* st) {
  xbi::clear_error();
  xb_graph* g = const_cast<xb_graph*>(gc);
  if (!c || !g || !mate) return fail(XB_ERR_ARG, "null argument");
  if (!g->ctx) return fail(XB_ERR_STATE, "the graph's context was destroyed");
  if (g->ctx->device != c->device) return fail(XB_ERR_ARG, "graph lives on another device");
  if (g->n >= (int64_t)1 << 29) return fail(XB_ERR_CAPACITY, "matching supports fewer than 2^29 vertices");
  if (st) std::memset(st, 0, sizeof(*st));
  XB_CUDA(cudaSetDevice(c->device));
  const int64_t n = g->n, m = g->m;
  const int64_t cand_cap = std::max<int64_t>(m, 1);
  // state, pred, base, lock, head, stamp, two frontiers, mate: int32 x n; found: n int2;
  // candidates: m int2 + m links; partition: eoff and ebase (n int64), tile sums, chunk owners;
  // counters.  Each region is rounded up to 256 bytes.
  const size_t bytes = 256 * 28 + 4 * (size_t)n * 9 + 8 * (size_t)n + 12 * (size_t)cand_cap + 16 * (size_t)n +
                       8 * (size_t)(n / xbp::kTile + 2) + 4 * (size_t)(m / xbp::kChunk + 2) + 256;
  {
    const xb_status ws = xbe::ensure_scratch(c, bytes, "matching");
    if (ws != XB_OK) return ws;
  }
  char* p = (char*)c->ws;
  MmWork wk;
  wk.st = carve_ints<int32_t>(p, n);
  wk.pred = carve_ints<int32_t>(p, n);
  wk.base = carve_ints<int32_t>(p, n);
  wk.lock = carve_ints<int32_t>(p, n);
  wk.head = carve_ints<int32_t>(p, n);
  wk.stamp = carve_ints<int32_t>(p, n);
  wk.front[0] = carve_ints<int32_t>(p, n);
  wk.front[1] = carve_ints<int32_t>(p, n);
  wk.found = carve_ints<int2>(p, n);
  wk.cand = carve_ints<int2>(p, cand_cap);
  wk.cand_next = carve_ints<int32_t>(p, cand_cap);
  int32_t* d_mate = carve_ints<int32_t>(p, n);
  wk.tick = carve_ints<int32_t>(p, 1);
  wk.fcnt = carve_ints<int32_t>(p, 2);
  wk.lv = carve_ints<MmLevel>(p, 1);
  wk.sticky = carve_ints<MmLevel>(p, 1);
  wk.ph = carve_ints<MmPhase>(p, 1);
  wk.eoff = carve_ints<int64_t>(p, n);
  wk.ebase = carve_ints<int64_t>(p, n);
  wk.tsum = carve_ints<int64_t>(p, n / xbp::kTile + 2);
  wk.scal = carve_ints<int64_t>(p, 4);
  wk.chunk_first = carve_ints<int32_t>(p, m / xbp::kChunk + 2);
  if ((size_t)(p - (char*)c->ws) > bytes) return fail(XB_ERR_STATE, "matching workspace layout");
  cudaStream_t s = c->stream;
  const bool dev = (flags & XB_OUT_DEVICE) != 0;
  XB_CUDA(cudaMemcpyAsync(d_mate, mate, sizeof(int32_t) * (size_t)n,
                          dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  XB_CUDA(cudaMemsetAsync(wk.tick, 0, sizeof(int32_t), s));
  XB_CUDA(cudaMemsetAsync(wk.stamp, 0, sizeof(int32_t) * (size_t)n, s));
  XB_CUDA(cudaMemsetAsync(wk.lv, 0, sizeof(MmLevel), s));
  XB_CUDA(cudaMemsetAsync(wk.sticky, 0, sizeof(MmLevel), s));
  const int vgrid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)c->num_sms * 8));
  if (g->off64)
    k_mm_check<int64_t><<<vgrid, 256, 0, s>>>(n, (const int64_t*)g->d_ro, g->d_ci, d_mate, &wk.lv->err);
  else
    k_mm_check<int32_t><<<vgrid, 256, 0, s>>>(n, (const int32_t*)g->d_ro, g->d_ci, d_mate, &wk.lv->err);
  XB_LAUNCH_CHECK("matching check");
  int32_t bad = 0;
  XB_CUDA(cudaMemcpyAsync(&bad, &wk.lv->err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  XB_CUDA(cudaStreamSynchronize(s));
  if (bad) return fail(XB_ERR_ARG, "the initial matching is not a matching of this graph");
  XB_CUDA(cudaEventRecord(c->ev0, s));
  xb_status r = g->off64 ? run_match<int64_t>(c, g, d_mate, wk, cand_cap, st)
                         : run_match<int32_t>(c, g, d_mate, wk, cand_cap, st);
  if (r != XB_OK) {
    cudaStreamSynchronize(s);
    return r;
  }
  XB_CUDA(cudaEventRecord(c->ev1, s));
  XB_CUDA(cudaMemcpyAsync(mate, d_mate, sizeof(int32_t) * (size_t)n,
                          dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  XB_CUDA(cudaStreamSynchronize(s));
  if (st) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    st->device_ms = ms;
    int64_t size = 0;
    if (!dev) {
      for (int64_t v = 0; v < n; v++) size += mate[v] >= 0;
      st->reached = size / 2;
    }
  }
  return XB_OK;
}

}  // extern "C"
