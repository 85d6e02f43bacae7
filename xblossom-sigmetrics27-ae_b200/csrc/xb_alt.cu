// xb_alt.cu -- xb_traverse in alternating mode: the alternating forest of a
// matching, grown from every exposed vertex at once.
//
// The expansion of the reference's alternating mode (ExpandAlternatingForest,
// apps/xb/src/xblsm_gpu/xblossom_gpu_engine_10.cu:270-359; the (w, v) records
// of ExpandTwoNodes, apps/xb/src/include/path_table/path_table.h:256-271): a
// matched pair (w, mate w) next to an outer vertex v of level 2d joins v's
// tree, w inner at level 2d+1 with parent v, its mate outer at level 2d+2
// with parent w.  Where the reference's claims race, the result here is
// fixed: w's parent is its smallest outer neighbour of level 2d, and when both
// ends of a pair qualify, the end with the smaller such neighbour (then the
// smaller id) is the inner one.  Edges between outer vertices label nothing
// (augmenting paths and blossoms are the matching engine's business,
// xb_max_match).
//
// Per level: the outer frontier proposes itself to its unlabeled matched
// neighbours by atomicMin (the first proposal to a vertex lists it), a
// resolve pass labels each proposed pair once, a clear pass resets the
// proposals.  Warp per frontier vertex, 32-entry windows.
#include "xb_engine_common.cuh"

using xbi::fail;

namespace {

__global__ void k_alt_init(int64_t n, const int32_t* __restrict__ mate, int32_t* level, int32_t* parent,
                           int32_t* owner, int32_t* cand, int32_t* front, int32_t* fcount, int32_t* bad) {
  // warp-uniform rounds, so the frontier appends go out one atomic per warp
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t b0 = (int64_t)blockIdx.x * blockDim.x; b0 < n; b0 += stride) {
    const int64_t v = b0 + threadIdx.x;
    bool app = false;
    if (v < n) {
      const int32_t m = mate[v];
      cand[v] = INT32_MAX;
      if (m < -1 || m >= n || m == v || (m >= 0 && mate[m] != v)) atomicAdd(bad, 1);
      if (m < 0) {
        level[v] = 0;
        parent[v] = owner[v] = (int32_t)v;
        app = true;
      } else {
        level[v] = parent[v] = owner[v] = -1;
      }
    }
    xbk::warp_append(app, (int32_t)v, front, fcount);
  }
}

// mate[v] must be a neighbour of v (sorted adjacency).
template <typename OffT>
__global__ void k_alt_check_edges(int64_t n, const OffT* __restrict__ ro, const int32_t* __restrict__ ci,
                                  const int32_t* __restrict__ mate, int32_t* bad) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t m = mate[v];
    if (m < 0 || m >= n) continue;
    int64_t lo = ro[v], hi = ro[v + 1];
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (ci[mid] < m) lo = mid + 1;
      else hi = mid;
    }
    if (lo == (int64_t)ro[v + 1] || ci[lo] != m) atomicAdd(bad, 1);
  }
}

template <typename OffT>
__global__ void k_alt_propose(const int32_t* __restrict__ front, int32_t fcount, const OffT* __restrict__ ro,
                              const int32_t* __restrict__ ci, const int32_t* __restrict__ mate,
                              const int32_t* __restrict__ level, int32_t* cand, int32_t* touched,
                              int32_t* tcount, unsigned long long* scanned) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long sc = 0;
  for (int64_t i = warp; i < fcount; i += nwarps) {
    const int32_t v = front[i];
    const int64_t beg = ro[v], end = ro[v + 1];
    sc += (unsigned long long)(end - beg);
    for (int64_t e0 = beg; e0 < end; e0 += 32) {  // warp-uniform windows
      const int64_t e = e0 + lane;
      bool first = false;
      int32_t w = 0;
      if (e < end) {
        w = ci[e];
        if (level[w] == -1 && mate[w] >= 0) first = atomicMin(&cand[w], v) == INT32_MAX;
      }
      xbk::warp_append(first, w, touched, tcount);
    }
  }
  sc = xbk::warp_sum_u64(sc);
  if (lane == 0 && sc) atomicAdd(scanned, sc);
}

__global__ void k_alt_resolve(const int32_t* __restrict__ touched, const int32_t* __restrict__ tcount_p,
                              const int32_t* __restrict__ mate, const int32_t* __restrict__ cand, int32_t d,
                              int32_t* level, int32_t* parent, int32_t* owner, int32_t* next, int32_t* ncount) {
  const int32_t tcount = *tcount_p;
  // warp-uniform rounds: the next frontier takes one atomic per warp
  for (int32_t b0 = blockIdx.x * blockDim.x; b0 < tcount; b0 += gridDim.x * blockDim.x) {
    const int32_t i = b0 + (int32_t)threadIdx.x;
    bool app = false;
    int32_t x = 0;
    if (i < tcount) {
      const int32_t w = touched[i];
      x = mate[w];
      const int32_t cw = cand[w], cx = cand[x];
      if (cx == INT32_MAX || cw < cx || (cw == cx && w < x)) {  // else x is the inner one
        const int32_t r = owner[cw];
        level[w] = 2 * d + 1;
        parent[w] = cw;
        owner[w] = r;
        level[x] = 2 * d + 2;
        parent[x] = w;
        owner[x] = r;
        app = true;
      }
    }
    xbk::warp_append(app, x, next, ncount);
  }
}

__global__ void k_alt_clear(const int32_t* __restrict__ touched, const int32_t* __restrict__ tcount_p, int32_t* cand) {
  const int32_t tcount = *tcount_p;
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < tcount; i += gridDim.x * blockDim.x)
    cand[touched[i]] = INT32_MAX;
}

struct AltCounters {
  int32_t count[2], tcount, bad;
  unsigned long long scanned;
};

template <typename OffT>
xb_status run_alt(xb_ctx* c, xb_graph* g, int32_t* mate, int32_t* level, int32_t* parent, int32_t* owner,
                  int32_t* cand, int32_t* front0, int32_t* front1, int32_t* touched, AltCounters* dc, xb_stats* st) {
  cudaStream_t s = c->stream;
  const int64_t n = g->n;
  const OffT* ro = (const OffT*)g->d_ro;
  const int sms = c->num_sms;
  const int vgrid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8));
  AltCounters* h = (AltCounters*)c->h_ctr;  // pinned host scratch
  static_assert(sizeof(AltCounters) <= sizeof(xbk::Ctrs), "pinned scratch too small");
  XB_CUDA(cudaMemsetAsync(dc, 0, sizeof(AltCounters), s));
  k_alt_init<<<vgrid, 256, 0, s>>>(n, mate, level, parent, owner, cand, front0, &dc->count[0], &dc->bad);
  k_alt_check_edges<OffT><<<vgrid, 256, 0, s>>>(n, ro, g->d_ci, mate, &dc->bad);
  XB_LAUNCH_CHECK("alternating init");
  XB_CUDA(cudaMemcpyAsync(h, dc, sizeof(AltCounters), cudaMemcpyDeviceToHost, s));
  XB_CUDA(cudaStreamSynchronize(s));
  if (h->bad) return fail(XB_ERR_ARG, "the matching is not a matching of this graph");
  int32_t fcount = h->count[0];
  int64_t rounds = 0, launches = 2;
  int32_t* fr[2] = {front0, front1};
  int cur = 0;
  for (int32_t d = 0; fcount > 0; d++) {
    if (d > n) return fail(XB_ERR_STATE, "alternating forest: level bound exceeded");
    rounds++;
    XB_CUDA(cudaMemsetAsync(&dc->tcount, 0, sizeof(int32_t), s));
    XB_CUDA(cudaMemsetAsync(&dc->count[cur ^ 1], 0, sizeof(int32_t), s));
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)fcount + 7) / 8, (int64_t)sms * 16));
    k_alt_propose<OffT><<<grid, 256, 0, s>>>(fr[cur], fcount, ro, g->d_ci, mate, level, cand, touched, &dc->tcount,
                                             &dc->scanned);
    k_alt_resolve<<<sms * 8, 256, 0, s>>>(touched, &dc->tcount, mate, cand, d, level, parent, owner, fr[cur ^ 1],
                                          &dc->count[cur ^ 1]);
    k_alt_clear<<<sms * 8, 256, 0, s>>>(touched, &dc->tcount, cand);
    XB_LAUNCH_CHECK("alternating level");
    launches += 3;
    XB_CUDA(cudaMemcpyAsync(h, dc, sizeof(AltCounters), cudaMemcpyDeviceToHost, s));
    XB_CUDA(cudaStreamSynchronize(s));
    cur ^= 1;
    fcount = h->count[cur];
  }
  if (st) {
    st->levels = (int32_t)rounds;
    st->edges_scanned = (int64_t)h->scanned;
    st->edges_traversed = (int64_t)h->scanned;
    st->class_launches[0] = launches;
  }
  return XB_OK;
}

}  // namespace

namespace xbe {

// Alternating mode of xb_traverse.  All arrays are n int32; host pointers,
// or device pointers with XB_OUT_DEVICE.
xb_status traverse_alternating(xb_ctx* c, xb_graph* g, const int32_t* matching, int32_t* level, int32_t* parent,
                               int32_t* owner, uint32_t flags, xb_stats* st) {
  if (!matching || !level || !parent || !owner) return fail(XB_ERR_ARG, "alternating mode needs matching, level, parent and owner");
  const int64_t n = g->n;
  const bool dev = (flags & XB_OUT_DEVICE) != 0;
  // work: mate copy, 3 output arrays (host output), proposals, two frontiers, touched list, counters
  const size_t ints = (size_t)n * (dev ? 5 : 8);
  const size_t bytes = sizeof(int32_t) * ints + 16 * 256 + sizeof(AltCounters);
  {
    const xb_status ws = ensure_scratch(c, bytes, "alternating-mode");
    if (ws != XB_OK) return ws;
  }
  char* p = (char*)c->ws;
  auto take = [&](size_t count) {
    int32_t* r = (int32_t*)p;
    p += ((sizeof(int32_t) * std::max<size_t>(count, 1) + 255) / 256) * 256;
    return r;
  };
  int32_t* cand = take((size_t)n);
  int32_t* f0 = take((size_t)n);
  int32_t* f1 = take((size_t)n);
  int32_t* touched = take((size_t)n);
  int32_t *d_mate = const_cast<int32_t*>(matching), *d_level = level, *d_parent = parent, *d_owner = owner;
  cudaStream_t s = c->stream;
  if (!dev) {
    d_mate = take((size_t)n);
    d_level = take((size_t)n);
    d_parent = take((size_t)n);
    d_owner = take((size_t)n);
    XB_CUDA(cudaMemcpyAsync(d_mate, matching, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, s));
  }
  AltCounters* dc = (AltCounters*)take(sizeof(AltCounters) / sizeof(int32_t) + 1);
  if ((size_t)(p - (char*)c->ws) > bytes) return fail(XB_ERR_STATE, "alternating-mode workspace layout");
  XB_CUDA(cudaEventRecord(c->ev0, s));
  xb_status r = g->off64 ? run_alt<int64_t>(c, g, d_mate, d_level, d_parent, d_owner, cand, f0, f1, touched, dc, st)
                         : run_alt<int32_t>(c, g, d_mate, d_level, d_parent, d_owner, cand, f0, f1, touched, dc, st);
  if (r != XB_OK) {
    cudaStreamSynchronize(s);
    return r;
  }
  XB_CUDA(cudaEventRecord(c->ev1, s));
  if (!dev) {
    XB_CUDA(cudaMemcpyAsync(level, d_level, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, s));
    XB_CUDA(cudaMemcpyAsync(parent, d_parent, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, s));
    XB_CUDA(cudaMemcpyAsync(owner, d_owner, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, s));
  }
  XB_CUDA(cudaStreamSynchronize(s));
  if (st) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    st->device_ms = ms;
    if (!dev) {
      int64_t reached = 0;
      for (int64_t v = 0; v < n; v++) reached += level[v] >= 0;
      st->reached = reached;
    }
  }
  return XB_OK;
}

}  // namespace xbe
