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
//  - a phase starts a fresh forest: every exposed vertex is an outer root;
//  - a level expands all outer frontier vertices (warp per vertex):
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
//    (thread per path) and the phase ends;
//  - otherwise the candidates are contracted, one thread per tree walking
//    its list: the cycle's top is the first common blossom base on the two
//    paths to the root, `pred` of the outer vertices on the cycle is
//    rerouted across it (so a later augmenting path can be read back
//    through the blossom), the bases are merged into the top (union-find),
//    and the inner vertices on the cycle become outer frontier vertices;
//  - a search whose frontier runs empty without augmenting paths proves the
//    matching maximum.
//
// State word per vertex: -1 outside the forest, else root * 4 + label
// (1 outer, 2 inner), written in one store so a reader sees a whole state.
// A reader that finds a pair half claimed skips it: if the vertex is outer
// it will scan the edge itself on the next level.  Every walk over tree or
// blossom pointers is bounded by n steps and reports XB_ERR_STATE on
// overrun instead of looping.
#include "xb_engine_common.cuh"

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

__global__ void k_mm_init(int64_t n, const int32_t* __restrict__ mate, int32_t* st, int32_t* pred, int32_t* base,
                          int32_t* lock, int32_t* head, int32_t* front, int32_t* fcount) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const bool exposed = mate[v] < 0;
    st[v] = exposed ? mm_state((int32_t)v, kOuter) : -1;
    pred[v] = -1;
    base[v] = (int32_t)v;
    lock[v] = 0;
    head[v] = -1;
    if (exposed) front[atomicAdd(fcount, 1)] = (int32_t)v;
  }
}

struct MmLevel {
  int32_t next_count, found, cand, err;
  unsigned long long scanned;
};

template <typename OffT>
__global__ void k_mm_expand(const int32_t* __restrict__ front, int32_t fcount, const OffT* __restrict__ ro,
                            const int32_t* __restrict__ ci, const int32_t* __restrict__ mate, int32_t* st,
                            int32_t* pred, const int32_t* __restrict__ base, int32_t* lock, int32_t* next,
                            int2* found, int2* cand, int32_t* cand_next, int32_t* head, int64_t cand_cap,
                            int64_t n, MmLevel* lv) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long scanned = 0;
  for (int64_t i = warp; i < fcount; i += nwarps) {
    const int32_t v = front[i];
    const int32_t mv = mate[v];
    const int32_t rv = st[v] >> 2;  // outer, stable during the level
    const int64_t beg = ro[v], end = ro[v + 1];
    scanned += (unsigned long long)(end - beg);
    int32_t bv = -2;  // base of v, looked up on first need
    for (int64_t e0 = beg; e0 < end; e0 += 32) {  // warp-uniform windows
      const int64_t e = e0 + lane;
      bool grow = false;
      int32_t grown = 0;
      if (e < end) {
        const int32_t w = ci[e];
        if (w != mv) {
          const int32_t sw = *(volatile int32_t*)&st[w];
          if (sw == -1) {
            const int32_t mw = mate[w];
            if (mw >= 0) {
              const int32_t lk = min(w, mw), other = max(w, mw);
              const int32_t lab_lk = lk == w ? kInner : kOuter;
              if (atomicCAS(&st[lk], -1, mm_state(rv, lab_lk)) == -1) {
                pred[w] = v;
                st[other] = mm_state(rv, lab_lk == kInner ? kOuter : kInner);
                grow = true;
                grown = mw;
              }
            }
          } else if ((sw & 3) == kOuter) {
            const int32_t rw = sw >> 2;
            if (rw != rv) {
              const int32_t a = min(rv, rw), b = max(rv, rw);
              if (atomicExch(&lock[a], 1) == 0) {
                if (atomicExch(&lock[b], 1) == 0) {
                  const int32_t k = atomicAdd(&lv->found, 1);
                  found[k] = make_int2(v, w);
                } else {
                  atomicExch(&lock[a], 0);
                }
              }
            } else {
              if (bv == -2) bv = mm_find_ro(base, v, n);
              const int32_t bw = mm_find_ro(base, w, n);
              if (bv < 0 || bw < 0) {
                atomicExch(&lv->err, 1);
              } else if (bv != bw) {
                const int32_t k = atomicAdd(&lv->cand, 1);
                if (k < cand_cap) {
                  cand[k] = make_int2(v, w);
                  cand_next[k] = atomicExch(&head[rv], k);
                } else {
                  atomicExch(&lv->err, 2);
                }
              }
            }
          }
        }
      }
      xbk::warp_append(grow, grown, next, &lv->next_count);
    }
  }
  scanned = xbk::warp_sum_u64(scanned);
  if (lane == 0 && scanned) atomicAdd(&lv->scanned, scanned);
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

__global__ void k_mm_flip(const int2* __restrict__ found, int32_t nfound, int32_t* mate,
                          const int32_t* __restrict__ pred, int64_t n, MmLevel* lv) {
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
__global__ void k_mm_blossom(const int2* __restrict__ cand, int32_t ncand, const int32_t* __restrict__ cand_next,
                             int32_t* head, int32_t* st, const int32_t* __restrict__ mate, int32_t* pred,
                             int32_t* base, int32_t* stamp, int32_t* tick, int32_t* next, int64_t n,
                             MmLevel* lv) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ncand; i += gridDim.x * blockDim.x) {
    const int32_t r = st[cand[i].x] >> 2;
    if (head[r] != i) continue;
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
            next[atomicAdd(&lv->next_count, 1)] = m;
          }
          x = pred[m];
        }
      }
    }
    head[r] = -1;
  }
}

struct MmWork {
  int32_t *st, *pred, *base, *lock, *head, *stamp, *front[2], *cand_next, *tick, *fcount;
  int2 *found, *cand;
  MmLevel* lv;
};

template <typename OffT>
xb_status run_match(xb_ctx* c, xb_graph* g, int32_t* d_mate, const MmWork& wk, int64_t cand_cap, xb_stats* st) {
  cudaStream_t s = c->stream;
  const int64_t n = g->n;
  const OffT* ro = (const OffT*)g->d_ro;
  const int sms = c->num_sms;
  const int vgrid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8));
  MmLevel* h = (MmLevel*)c->h_ctr;  // pinned host scratch
  static_assert(sizeof(MmLevel) <= sizeof(xbk::Ctrs), "pinned scratch too small");
  int64_t phases = 0, levels = 0, blossom_levels = 0, flips = 0;
  unsigned long long scanned = 0;
  // classes: 0 = forest expansion, 1 = flips and blossom contraction, 2 = phase init
  xbe::ClassTimer timer{c, st, c->tuning.timing != 0};
  for (;;) {
    if (phases > n / 2 + 1) return fail(XB_ERR_STATE, "matching: phase bound exceeded");
    phases++;
    XB_CUDA(cudaMemsetAsync(wk.fcount, 0, sizeof(int32_t), s));
    timer.begin();
    k_mm_init<<<vgrid, 256, 0, s>>>(n, d_mate, wk.st, wk.pred, wk.base, wk.lock, wk.head, wk.front[0], wk.fcount);
    XB_LAUNCH_CHECK("matching init");
    timer.end(2, 1);
    int32_t fcount = 0;
    XB_CUDA(cudaMemcpyAsync(&h->next_count, wk.fcount, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    XB_CUDA(cudaStreamSynchronize(s));
    fcount = h->next_count;
    if (fcount == 0) break;  // perfect matching
    int cur = 0;
    bool flipped = false;
    for (int64_t lvl = 0; fcount > 0; lvl++) {
      if (lvl > n) return fail(XB_ERR_STATE, "matching: level bound exceeded");
      levels++;
      XB_CUDA(cudaMemsetAsync(wk.lv, 0, sizeof(MmLevel), s));
      const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)fcount + 7) / 8, (int64_t)sms * 16));
      timer.begin();
      k_mm_expand<OffT><<<grid, 256, 0, s>>>(wk.front[cur], fcount, ro, g->d_ci, d_mate, wk.st, wk.pred, wk.base,
                                             wk.lock, wk.front[cur ^ 1], wk.found, wk.cand, wk.cand_next, wk.head,
                                             cand_cap, n, wk.lv);
      XB_LAUNCH_CHECK("matching expand");
      timer.end(0, 1);
      XB_CUDA(cudaMemcpyAsync(h, wk.lv, sizeof(MmLevel), cudaMemcpyDeviceToHost, s));
      XB_CUDA(cudaStreamSynchronize(s));
      if (h->err) return fail(XB_ERR_STATE, "matching: expand found an inconsistent forest (" + std::to_string(h->err) + ")");
      scanned += h->scanned;
      if (h->found > 0) {
        const int32_t nf = h->found;
        timer.begin();
        k_mm_flip<<<(nf + 127) / 128, 128, 0, s>>>(wk.found, nf, d_mate, wk.pred, n, wk.lv);
        XB_LAUNCH_CHECK("matching flip");
        timer.end(1, 1);
        XB_CUDA(cudaMemcpyAsync(&h->err, &wk.lv->err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        XB_CUDA(cudaStreamSynchronize(s));
        if (h->err) return fail(XB_ERR_STATE, "matching: flip walk failed");
        flips += nf;
        flipped = true;
        break;
      }
      if (h->cand > 0) {
        const int32_t nc = h->cand;
        blossom_levels++;
        timer.begin();
        k_mm_blossom<<<(nc + 127) / 128, 128, 0, s>>>(wk.cand, nc, wk.cand_next, wk.head, wk.st, d_mate, wk.pred,
                                                      wk.base, wk.stamp, wk.tick, wk.front[cur ^ 1], n, wk.lv);
        XB_LAUNCH_CHECK("matching blossoms");
        timer.end(1, 1);
        XB_CUDA(cudaMemcpyAsync(h, wk.lv, sizeof(MmLevel), cudaMemcpyDeviceToHost, s));
        XB_CUDA(cudaStreamSynchronize(s));
        if (h->err) return fail(XB_ERR_STATE, "matching: blossom walk failed (" + std::to_string(h->err) + ")");
      }
      fcount = h->next_count;
      cur ^= 1;
    }
    if (!flipped) break;  // the search ran out without an augmenting path: maximum
  }
  if (st) {
    st->batches = (int32_t)std::min<int64_t>(phases, INT32_MAX);
    st->levels = (int32_t)std::min<int64_t>(levels, INT32_MAX);
    st->pull_levels = (int32_t)std::min<int64_t>(blossom_levels, INT32_MAX);
    st->edges_scanned = (int64_t)scanned;
    st->edges_traversed = (int64_t)scanned;
    st->vertices_scanned = flips;
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
  // state, pred, base, lock, head, stamp, two frontiers, tick, count: int32 x n;
  // found: n int2; candidates: m int2 + m links; mate: n; the level counters
  const size_t bytes = 256 * 16 + 4 * (size_t)n * 9 + 8 * (size_t)n + 12 * (size_t)cand_cap + 4 * (size_t)n + 256;
  if (c->ws_bytes < bytes || !c->ws) {
    if (c->ws) cudaFree(c->ws);
    c->ws = nullptr;
    c->ws_bytes = 0;
    if (cudaMalloc(&c->ws, bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(XB_ERR_OOM, "matching work allocation failed");
    }
    c->ws_bytes = bytes;
  }
  c->ws_key[0] = -1;  // the traversal's zero invariants no longer hold in the workspace
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
  wk.fcount = carve_ints<int32_t>(p, 1);
  wk.lv = carve_ints<MmLevel>(p, 1);
  if ((size_t)(p - (char*)c->ws) > bytes) return fail(XB_ERR_STATE, "matching workspace layout");
  cudaStream_t s = c->stream;
  const bool dev = (flags & XB_OUT_DEVICE) != 0;
  XB_CUDA(cudaMemcpyAsync(d_mate, mate, sizeof(int32_t) * (size_t)n,
                          dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  XB_CUDA(cudaMemsetAsync(wk.tick, 0, sizeof(int32_t), s));
  XB_CUDA(cudaMemsetAsync(wk.stamp, 0, sizeof(int32_t) * (size_t)n, s));
  XB_CUDA(cudaMemsetAsync(wk.lv, 0, sizeof(MmLevel), s));
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
