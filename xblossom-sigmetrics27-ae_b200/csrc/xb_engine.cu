// xb_engine.cu -- device context, resident graphs and the plain per-call
// traversal path of libxbtrav.so (C ABI in include/xbtrav.h).
//
// The plain path mirrors the reference engine's control structure
// (FindAndFlipAugmentingPathInAlternatingForest's host loop,
// apps/xb/src/xblsm_gpu/xblossom_gpu_engine_10.cu:72-185): a host-side level
// loop that launches one level step, reads the frontier counters back and
// decides the next step.  Unlike the reference it reads one 200-byte counter
// block per level (instead of four D2H scalars plus a device sync per queue
// swap) and traverses B (32 or 64) sources per launch sequence.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "xb_internal.h"
#include "xb_kernels.cuh"

using xbi::fail;

#define XB_CUDA(call)                                                                        \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) return fail(XB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define XB_LAUNCH_CHECK(what)                                                                \
  do {                                                                                       \
    cudaError_t e_ = cudaGetLastError();                                                     \
    if (e_ != cudaSuccess) return fail(XB_ERR_CUDA, std::string("launch ") + what + ": " + cudaGetErrorString(e_)); \
  } while (0)

struct xb_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  xb_tuning tuning{};
  // workspace
  void* ws = nullptr;
  size_t ws_bytes = 0;
  int64_t ws_key[3] = {-1, -1, -1};  // (n, word bytes, words) of the current layout
  xbk::Ctrs* d_ctr = nullptr;
  xbk::Ctrs* h_ctr = nullptr;  // pinned
  int32_t* d_src = nullptr;
  int64_t src_cap = 0;
  int32_t* d_stage = nullptr;  // device staging for host-bound tables
  size_t stage_bytes = 0;
  int32_t epoch = 1;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evc0 = nullptr, evc1 = nullptr;
};

struct xb_graph {
  xb_ctx* ctx = nullptr;
  int64_t n = 0, m = 0, max_deg = 0;
  bool off64 = false;
  void* d_ro = nullptr;
  int32_t* d_ci = nullptr;
  std::vector<int64_t> h_ro;
  int32_t* d_heavy = nullptr;  // vertices with degree > heavy_thr, ascending
  int32_t* d_hpar = nullptr;   // per heavy vertex, 64 parent slots of the table pass
  int2* d_hitems = nullptr;    // (heavy index, chunk) items of the table pass
  int64_t n_hitems = 0;
  int2* d_hub_items = nullptr;  // (heavy index, chunk) items of the hub pull
  int64_t n_hub_items = 0;
  int32_t* d_hidx_of = nullptr;  // vertex -> index in the heavy list (-1 for light)
  int32_t n_heavy = 0;
  int32_t heavy_thr = -1;
};

namespace {

// Edges per work item of the heavy-vertex table scan.
constexpr int kTableChunk = 4096;
// Vertices above this degree (hubs) are pulled in chunks by many warps; the
// other heavy vertices by one warp each.
constexpr int kHubDegree = 4096;
constexpr int kHubChunk = 2048;
// Parent slots per heavy vertex: up to 64 sources x 4 words.
constexpr int kHparRow = 256;

struct WsLayout {
  size_t seen, F, N, p01, ph, pushed, p8, touched, fl_light, fl_heavy, nl_light, nl_heavy, stamp, total;
  int64_t plane_stride;  // in words
  int nplanes_alloc;
};

int bitlen_levels(int64_t n) {
  // levels are in [0, n-1]; number of bits to hold n-1, at least 3
  int b = 0;
  int64_t x = n > 1 ? n - 1 : 0;
  while (x) {
    b++;
    x >>= 1;
  }
  return std::max(3, b);
}

size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

WsLayout layout_for(int64_t n, int word_bytes, int nw) {
  WsLayout L{};
  const size_t sw = align_up((size_t)n * nw * word_bytes);
  const size_t li = align_up((size_t)std::max<int64_t>(n, 1) * 4);
  L.nplanes_alloc = bitlen_levels(n);
  L.plane_stride = (int64_t)(sw / word_bytes);
  size_t o = 0;
  L.seen = o; o += sw;
  L.F = o; o += sw;
  L.N = o; o += sw;
  L.p01 = o; o += 2 * sw;
  L.ph = o; o += sw * (L.nplanes_alloc - 2);
  L.pushed = o; o += sw;
  L.p8 = o; o += align_up((size_t)n * nw * word_bytes * 8);  // 8 position planes per (vertex, word)
  L.touched = o; o += li;
  L.fl_light = o; o += li;
  L.fl_heavy = o; o += li;
  L.nl_light = o; o += li;
  L.nl_heavy = o; o += li;
  L.stamp = o; o += li;
  L.total = o;
  return L;
}

// The F/N "all zero between calls" invariant and the epoch stamps hold per
// layout; a call with another (n, word size, words) places the regions at
// other offsets, so the used range is cleared whenever the layout changes.
xb_status ensure_workspace(xb_ctx* c, const WsLayout& L, int64_t n, int wbytes, int nw) {
  const int64_t key[3] = {n, wbytes, nw};
  if (c->ws_bytes >= L.total && c->ws) {
    if (std::memcmp(key, c->ws_key, sizeof(key)) != 0) {
      XB_CUDA(cudaMemsetAsync(c->ws, 0, L.total, c->stream));
      std::memcpy(c->ws_key, key, sizeof(key));
      c->epoch = 1;
    }
    return XB_OK;
  }
  std::memcpy(c->ws_key, key, sizeof(key));
  c->epoch = 1;
  if (c->ws) {
    cudaFree(c->ws);
    c->ws = nullptr;
    c->ws_bytes = 0;
  }
  cudaError_t e = cudaMalloc(&c->ws, L.total);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(XB_ERR_OOM, "workspace allocation of " + std::to_string(L.total) + " bytes failed");
  }
  c->ws_bytes = L.total;
  // F, N and the stamps must start zero; everything else is reset per pass
  XB_CUDA(cudaMemsetAsync(c->ws, 0, L.total, c->stream));
  return XB_OK;
}

xb_status ensure_sources(xb_ctx* c, int64_t k) {
  if (c->src_cap >= k) return XB_OK;
  if (c->d_src) cudaFree(c->d_src);
  c->d_src = nullptr;
  c->src_cap = 0;
  if (cudaMalloc(&c->d_src, sizeof(int32_t) * std::max<int64_t>(k, 1)) != cudaSuccess) {
    cudaGetLastError();
    return fail(XB_ERR_OOM, "source buffer allocation failed");
  }
  c->src_cap = k;
  return XB_OK;
}

xb_status ensure_stage(xb_ctx* c, size_t bytes) {
  if (c->stage_bytes >= bytes) return XB_OK;
  if (c->d_stage) cudaFree(c->d_stage);
  c->d_stage = nullptr;
  c->stage_bytes = 0;
  if (cudaMalloc(&c->d_stage, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(XB_ERR_OOM, "table staging allocation failed");
  }
  c->stage_bytes = bytes;
  return XB_OK;
}

xb_status ensure_heavy(xb_graph* g, int thr) {
  if (g->heavy_thr == thr) return XB_OK;
  std::vector<int32_t> hv;
  for (int64_t v = 0; v < g->n; v++)
    if (g->h_ro[v + 1] - g->h_ro[v] > thr) hv.push_back((int32_t)v);
  if (g->d_heavy) cudaFree(g->d_heavy);
  if (g->d_hpar) cudaFree(g->d_hpar);
  g->d_heavy = nullptr;
  g->d_hpar = nullptr;
  g->heavy_thr = -1;
  if (cudaMalloc(&g->d_heavy, sizeof(int32_t) * std::max<size_t>(hv.size(), 1)) != cudaSuccess ||
      cudaMalloc(&g->d_hpar, sizeof(int32_t) * kHparRow * std::max<size_t>(hv.size(), 1)) != cudaSuccess) {
    cudaGetLastError();
    return fail(XB_ERR_OOM, "heavy list allocation failed");
  }
  if (!hv.empty())
    XB_CUDA(cudaMemcpy(g->d_heavy, hv.data(), sizeof(int32_t) * hv.size(), cudaMemcpyHostToDevice));
  {
    std::vector<int32_t> hidx_of((size_t)g->n, -1);
    for (size_t i = 0; i < hv.size(); i++) hidx_of[hv[i]] = (int32_t)i;
    if (g->d_hidx_of) cudaFree(g->d_hidx_of);
    g->d_hidx_of = nullptr;
    if (cudaMalloc(&g->d_hidx_of, sizeof(int32_t) * (size_t)g->n) != cudaSuccess) {
      cudaGetLastError();
      return fail(XB_ERR_OOM, "heavy index map allocation failed");
    }
    XB_CUDA(cudaMemcpy(g->d_hidx_of, hidx_of.data(), sizeof(int32_t) * (size_t)g->n, cudaMemcpyHostToDevice));
  }
  // (heavy index, chunk) work items of the table pass, heaviest vertices first
  // (ids ascend roughly with falling degree in R-MAT-like graphs, so this is
  // the list order)
  std::vector<int2> items;
  for (size_t i = 0; i < hv.size(); i++) {
    const int64_t d = g->h_ro[hv[i] + 1] - g->h_ro[hv[i]];
    for (int64_t c = 0; c * kTableChunk < d; c++) items.push_back(make_int2((int)i, (int)c));
  }
  if (g->d_hitems) cudaFree(g->d_hitems);
  g->d_hitems = nullptr;
  if (cudaMalloc(&g->d_hitems, sizeof(int2) * std::max<size_t>(items.size(), 1)) != cudaSuccess) {
    cudaGetLastError();
    return fail(XB_ERR_OOM, "heavy item list allocation failed");
  }
  if (!items.empty())
    XB_CUDA(cudaMemcpy(g->d_hitems, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice));
  g->n_hitems = (int64_t)items.size();
  // (heavy index, chunk) items of the hub pull
  std::vector<int2> hub_items;
  for (size_t i = 0; i < hv.size(); i++) {
    const int64_t d = g->h_ro[hv[i] + 1] - g->h_ro[hv[i]];
    if (d <= kHubDegree) continue;
    for (int64_t c = 0; c * kHubChunk < d; c++) hub_items.push_back(make_int2((int)i, (int)c));
  }
  if (g->d_hub_items) cudaFree(g->d_hub_items);
  g->d_hub_items = nullptr;
  if (cudaMalloc(&g->d_hub_items, sizeof(int2) * std::max<size_t>(hub_items.size(), 1)) != cudaSuccess) {
    cudaGetLastError();
    return fail(XB_ERR_OOM, "hub item list allocation failed");
  }
  if (!hub_items.empty())
    XB_CUDA(cudaMemcpy(g->d_hub_items, hub_items.data(), sizeof(int2) * hub_items.size(), cudaMemcpyHostToDevice));
  g->n_hub_items = (int64_t)hub_items.size();
  g->n_heavy = (int32_t)hv.size();
  g->heavy_thr = thr;
  return XB_OK;
}

struct ClassTimer {
  xb_ctx* c;
  xb_stats* st;
  bool on;
  void begin() {
    if (on) cudaEventRecord(c->evc0, c->stream);
  }
  void end(int cls, int64_t launches) {
    if (st) st->class_launches[cls] += launches;
    if (!on) return;
    cudaEventRecord(c->evc1, c->stream);
    cudaEventSynchronize(c->evc1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->evc0, c->evc1);
    if (st) st->class_ms[cls] += ms;
  }
};

// Algorithmic bytes of a pass's level steps: the row-offset pair of every
// scanned vertex, colIndices + the gathered frontier words of every scanned
// edge, and a three-word sweep (seen read, seen and next-frontier write) of
// every swept vertex.
template <typename W, int NW, typename OffT>
int64_t level_bytes(const xbk::BatchCtr& b) {
  const int64_t R = (int64_t)sizeof(OffT) * 2;
  const int64_t wbytes = (int64_t)sizeof(W) * NW;
  return R * (int64_t)b.vertices_scanned + (4 + wbytes) * (int64_t)b.edges_scanned +
         3 * wbytes * (int64_t)b.vertices_swept;
}

// Algorithmic bytes of a pass's table pass: per vertex its row offsets, seen,
// level planes and parent-position planes (per word), the colIndices entry of
// every recorded parent, colIndices + gathered plane pair of every searched
// edge, and the two written tables.
template <typename W, int NW, typename OffT>
int64_t table_bytes(const xbk::BatchCtr& b, int64_t n, int kb) {
  const int64_t R = (int64_t)sizeof(OffT) * 2;
  return (int64_t)NW * n * (R + (int64_t)sizeof(W) * (1 + b.nplanes + 8)) + 4 * (int64_t)b.reached +
         (4 + 2 * (int64_t)sizeof(W)) * (int64_t)b.parent_edges + 8 * (int64_t)kb * n;
}

// Pointers and constants of one traversal pass (a workspace + counters).
template <typename W, int NW, typename OffT>
struct PassRes {
  int64_t n = 0;
  const OffT* ro = nullptr;
  const int32_t* ci = nullptr;
  W* seen = nullptr;
  W* buf[2] = {nullptr, nullptr};  // frontier words; buf[cur] = F, buf[cur ^ 1] = N
  xbk::Planes<W, NW> pl{};
  W* pushed = nullptr;
  W* ppos = nullptr;
  int32_t* touched = nullptr;
  xbk::Lists lists[2] = {};  // lists[cur] = current frontier, lists[cur ^ 1] = next
  int32_t* stamp = nullptr;
  xbk::Ctrs* ctr = nullptr;
  int32_t* hpar = nullptr;
  int heavy = 256;
  size_t state_bytes = 0, plane_bytes = 0, ppos_bytes = 0;
  int nplanes_alloc = 3;
};

template <typename W, int NW, typename OffT>
PassRes<W, NW, OffT> pass_res(const xb_graph* g, void* ws, const WsLayout& L, xbk::Ctrs* ctr, int32_t* hpar,
                              int heavy) {
  PassRes<W, NW, OffT> p;
  char* base = (char*)ws;
  p.n = g->n;
  p.ro = (const OffT*)g->d_ro;
  p.ci = g->d_ci;
  p.seen = (W*)(base + L.seen);
  p.buf[0] = (W*)(base + L.F);
  p.buf[1] = (W*)(base + L.N);
  p.pl = xbk::Planes<W, NW>{(W*)(base + L.p01), (W*)(base + L.ph), L.plane_stride};
  p.pushed = (W*)(base + L.pushed);
  p.ppos = (W*)(base + L.p8);
  p.touched = (int32_t*)(base + L.touched);
  p.lists[0] = xbk::Lists{(int32_t*)(base + L.fl_light), (int32_t*)(base + L.fl_heavy)};
  p.lists[1] = xbk::Lists{(int32_t*)(base + L.nl_light), (int32_t*)(base + L.nl_heavy)};
  p.stamp = (int32_t*)(base + L.stamp);
  p.ctr = ctr;
  p.hpar = hpar;
  p.heavy = heavy;
  p.state_bytes = (size_t)g->n * NW * sizeof(W);
  p.plane_bytes = (size_t)L.plane_stride * sizeof(W);
  p.ppos_bytes = p.state_bytes * 8;
  p.nplanes_alloc = L.nplanes_alloc;
  return p;
}

template <typename W, int NW>
xbk::Masks<W, NW> active_mask(int kb) {
  constexpr int B = xbk::WB<W>::bits;
  xbk::Masks<W, NW> a{};
  for (int i = 0; i < NW; i++) {
    const int lo = i * B, hi = std::min(kb, (i + 1) * B);
    W m = 0;
    for (int b = lo; b < hi; b++) m |= (W)1 << (b - lo);
    a.w[i] = m;
  }
  return a;
}

// Launch shapes of the level-step kernels.
struct StepShape {
  int push_light_grid;   // 0: skip
  dim3 push_heavy_grid;  // .y == 0: skip
  int finalize_grid;
  int pull_grid;
  int heavy_grid;
  int hub_grid;
  int commit_grid;
  int clear_grid;
};

template <typename W, int NW>
constexpr int pull_warps() {
  // the pull tile keeps 8 position words per lane and word in shared memory
  return (xbk::WB<W>::bits * NW * 32 * 8 > 40 * 1024) ? 4 : 8;
}

// Pass start: clear the per-pass state, reset counters, seed the sources.
template <typename W, int NW, typename OffT>
xb_status emit_pass_init(const PassRes<W, NW, OffT>& p, const xb_graph* g, const int32_t* src, int kb,
                         cudaStream_t s, int sms) {
  XB_CUDA(cudaMemsetAsync(p.seen, 0, p.state_bytes, s));
  XB_CUDA(cudaMemsetAsync(p.pl.p01, 0, 2 * p.plane_bytes, s));
  XB_CUDA(cudaMemsetAsync(p.pl.ph, 0, p.plane_bytes, s));
  XB_CUDA(cudaMemsetAsync(p.pushed, 0, p.state_bytes, s));
  XB_CUDA(cudaMemsetAsync(p.ppos, 0, p.ppos_bytes, s));
  if (g->n_heavy > 0) {  // parent slots of the heavy vertices (hub pulls fold in with atomicMin)
    const int64_t hcount = (int64_t)g->n_heavy * kHparRow;
    xbk::k_fill<int32_t><<<(int)std::min<int64_t>((hcount + 255) / 256, (int64_t)sms * 8), 256, 0, s>>>(p.hpar, hcount,
                                                                                                   INT32_MAX);
  }
  xbk::k_pass_init<<<1, 1, 0, s>>>(p.ctr, (long long)g->m);
  xbk::k_init_batch<W, NW, OffT><<<1, 256, 0, s>>>(src, kb, p.ro, p.buf[0], p.seen, p.pl, active_mask<W, NW>(kb),
                                                   p.heavy, p.lists[0], p.ctr);
  XB_LAUNCH_CHECK("pass init");
  return XB_OK;
}

template <typename W, int NW, typename OffT>
xb_status emit_push(const PassRes<W, NW, OffT>& p, const xb_graph* g, int cur, const StepShape& sh, int kb,
                    cudaStream_t s, int64_t* launches) {
  constexpr int PUSH_CHUNK = 2048;
  W* F = p.buf[cur];
  W* N = p.buf[cur ^ 1];
  const xbk::Lists fl = p.lists[cur], nl = p.lists[cur ^ 1];
  if (sh.push_light_grid > 0) {
    xbk::k_push_light<W, NW, OffT><<<sh.push_light_grid, 256, 0, s>>>(fl.light, &p.ctr->lv[cur].n_light, p.ro, p.ci, F,
                                                                      p.seen, N, p.stamp, p.touched, p.ctr, cur);
    (*launches)++;
  }
  if (sh.push_heavy_grid.y > 0) {
    xbk::k_push_heavy<W, NW, OffT><<<sh.push_heavy_grid, 256, 0, s>>>(fl.heavy, &p.ctr->lv[cur].n_heavy, p.ro, p.ci, F,
                                                                      p.seen, N, p.stamp, p.touched, p.ctr, cur,
                                                                      PUSH_CHUNK);
    xbk::k_clear_list<W, NW><<<sh.clear_grid, 256, 0, s>>>(fl.heavy, &p.ctr->lv[cur].n_heavy, F);
    *launches += 2;
  }
  xbk::k_push_finalize<W, NW, OffT><<<sh.finalize_grid, 256, 0, s>>>(p.touched, p.ro, N, p.seen, p.pl,
                                                                     active_mask<W, NW>(kb), p.heavy, nl, p.ctr, cur,
                                                                     p.pushed);
  (*launches)++;
  XB_LAUNCH_CHECK("push step");
  return XB_OK;
}

template <typename W, int NW, typename OffT>
xb_status emit_pull(const PassRes<W, NW, OffT>& p, const xb_graph* g, int cur, const StepShape& sh, int kb,
                    cudaStream_t s, int64_t* launches) {
  constexpr int PW = pull_warps<W, NW>();
  W* F = p.buf[cur];
  W* N = p.buf[cur ^ 1];
  const xbk::Lists fl = p.lists[cur], nl = p.lists[cur ^ 1];
  const xbk::Masks<W, NW> active = active_mask<W, NW>(kb);
  xbk::k_pull_tiles<W, NW, OffT, PW, 4><<<sh.pull_grid, PW * 32, 0, s>>>(p.n, p.ro, p.ci, F, p.seen, N, p.pl, active,
                                                                         p.heavy, nl, p.ctr, cur, p.ppos);
  (*launches)++;
  if (g->n_heavy > 0) {
    xbk::k_pull_heavy<W, NW, OffT, 4><<<sh.heavy_grid, 256, 0, s>>>(g->d_heavy, g->n_heavy, p.ro, p.ci, F, p.seen, N,
                                                                    p.pl, active, p.heavy, kHubDegree, nl, p.ctr, cur,
                                                                    p.hpar);
    (*launches)++;
    if (g->n_hub_items > 0) {
      xbk::k_pull_hubs<W, NW, OffT, 4><<<sh.hub_grid, 256, 0, s>>>(g->d_heavy, g->d_hub_items, g->n_hub_items, p.ro,
                                                                   p.ci, F, p.seen, N, active, p.ctr, cur, kHubChunk,
                                                                   p.hpar);
      xbk::k_pull_hub_commit<W, NW, OffT><<<sh.commit_grid, 256, 0, s>>>(g->d_heavy, g->n_heavy, p.ro, p.seen, N, p.pl,
                                                                        active, p.heavy, kHubDegree, nl, p.ctr, cur);
      *launches += 2;
    }
  }
  xbk::k_clear_frontier<W, NW><<<sh.clear_grid, 256, 0, s>>>(F, p.n, fl, p.ctr, cur);
  (*launches)++;
  XB_LAUNCH_CHECK("pull step");
  return XB_OK;
}

// Table pass of one pass (all its words).  Row s of a word's tables starts at
// lv_base + (wi*B + s) * row_stride.
template <typename W, int NW, typename OffT>
xb_status emit_tables(const PassRes<W, NW, OffT>& p, const xb_graph* g, const int32_t* src, int kb, int32_t* lv_base,
                      int32_t* pr_base, bool search_heavy, cudaStream_t s, int sms, int64_t* launches) {
  constexpr int B = xbk::WB<W>::bits;
  constexpr int TAB_WARPS = (B == 64) ? 4 : 8;
  const int64_t ntiles = (p.n + 31) / 32;
  const int tab_grid = (int)std::max<int64_t>(1, std::min<int64_t>((ntiles + TAB_WARPS - 1) / TAB_WARPS, (int64_t)sms * 16));
  for (int wi = 0; wi < NW; wi++) {
    const int kbw = std::min(B, kb - wi * B);
    if (kbw <= 0) break;
    int32_t* lv_out = lv_base + (int64_t)wi * B * p.n;
    int32_t* pr_out = pr_base + (int64_t)wi * B * p.n;
    const int32_t* wsrc = src + wi * B;
    if (g->n_heavy > 0 && search_heavy) {
      // heavy vertices reached by a push step at level >= 2: search their parents
      const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(g->n_hitems, (int64_t)sms * 8));
      xbk::k_tables_heavy_scan<W, NW, OffT><<<grid, 256, 0, s>>>(g->d_heavy, g->d_hitems, g->n_hitems, p.ro, p.ci,
                                                                 p.seen, p.pl, wi, kTableChunk, p.hpar, p.ctr,
                                                                 p.pushed);
      (*launches)++;
    }
    xbk::k_tables<W, NW, OffT, TAB_WARPS, 4><<<tab_grid, TAB_WARPS * 32, 0, s>>>(
        p.n, p.ro, p.ci, p.seen, p.pl, wi, kbw, p.heavy, lv_out, pr_out, p.ctr, p.ppos, p.pushed, wsrc, g->d_hidx_of,
        p.hpar);
    (*launches)++;
  }
  XB_LAUNCH_CHECK("tables");
  return XB_OK;
}

template <typename W, int NW, typename OffT>
StepShape max_shape(const xb_graph* g, int sms) {
  constexpr int PW = pull_warps<W, NW>();
  StepShape sh{};
  const int64_t n = g->n;
  const int64_t ntiles = (n + 31) / 32;
  sh.push_light_grid = sms * 16;
  sh.push_heavy_grid = dim3((unsigned)std::max<int64_t>(1, std::min<int64_t>((g->max_deg + 2047) / 2048, 64)),
                            (unsigned)std::max<int64_t>(1, std::min<int64_t>(g->n_heavy, 65535)));
  if (g->n_heavy == 0) sh.push_heavy_grid.y = 0;
  sh.finalize_grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8));
  sh.pull_grid = (int)std::max<int64_t>(1, std::min<int64_t>((ntiles + PW - 1) / PW, (int64_t)sms * 8));
  sh.heavy_grid = (int)std::max<int64_t>(1, std::min<int64_t>((g->n_heavy + 7) / 8, (int64_t)sms * 16));
  sh.hub_grid = (int)std::max<int64_t>(1, std::min<int64_t>((g->n_hub_items + 7) / 8, (int64_t)sms * 16));
  sh.commit_grid = (int)std::max<int64_t>(1, std::min<int64_t>((g->n_heavy + 255) / 256, (int64_t)sms * 4));
  sh.clear_grid = sms * 8;
  return sh;
}

template <typename W, int NW, typename OffT>
xb_status run_plain(xb_ctx* c, xb_graph* g, const int32_t* d_sources, int32_t k, int32_t* level_out,
                    int32_t* parent_out, bool out_dev, xb_stats* st) {
  constexpr int B = xbk::WB<W>::bits;
  constexpr int SPP = B * NW;  // sources per pass
  const int64_t n = g->n;
  const int heavy = std::max(32, c->tuning.heavy_degree);
  xb_status s = ensure_heavy(g, heavy);
  if (s != XB_OK) return s;
  const WsLayout L = layout_for(n, (int)sizeof(W), NW);
  s = ensure_workspace(c, L, n, (int)sizeof(W), NW);
  if (s != XB_OK) return s;
  if (!out_dev) {
    s = ensure_stage(c, sizeof(int32_t) * 2 * (size_t)SPP * (size_t)n);
    if (s != XB_OK) return s;
  }
  PassRes<W, NW, OffT> p = pass_res<W, NW, OffT>(g, c->ws, L, c->d_ctr, g->d_hpar, heavy);
  const int sms = c->num_sms;
  const float alpha = c->tuning.pull_alpha > 0 ? c->tuning.pull_alpha : 64.0f;
  ClassTimer timer{c, st, c->tuning.timing != 0};
  const StepShape mx = max_shape<W, NW, OffT>(g, sms);
  int max_levels = 0;

  for (int64_t k0 = 0; k0 < k; k0 += SPP) {
    const int kb = (int)std::min<int64_t>(SPP, k - k0);
    timer.begin();
    s = emit_pass_init<W, NW, OffT>(p, g, d_sources + k0, kb, c->stream, sms);
    if (s != XB_OK) return s;
    timer.end(2, 3);
    int cur = 0;
    for (;;) {
      // the device decides the step; the host reads the decision back
      xbk::k_step_begin<<<1, 1, 0, c->stream>>>(p.ctr, cur, alpha, p.nplanes_alloc, 0, 0);
      XB_LAUNCH_CHECK("step begin");
      XB_CUDA(cudaMemcpyAsync(c->h_ctr, p.ctr, sizeof(xbk::Ctrs), cudaMemcpyDeviceToHost, c->stream));
      XB_CUDA(cudaStreamSynchronize(c->stream));
      const xbk::BatchCtr bc = c->h_ctr->b;
      if (bc.dir == 2) break;
      const xbk::LevelCtr lc = c->h_ctr->lv[cur];
      timer.begin();
      int64_t launches = 1;
      if (bc.zero_plane >= 3) {
        xbk::k_zero_plane<W><<<sms * 8, 256, 0, c->stream>>>(p.pl.ph, p.pl.stride, n * NW, p.ctr);
        launches++;
      }
      StepShape sh = mx;
      if (bc.dir == 0) {
        sh.push_light_grid = lc.n_light > 0 ? (int)std::min<int64_t>(((int64_t)lc.n_light + 7) / 8, (int64_t)sms * 16) : 0;
        sh.push_heavy_grid.y = lc.n_heavy > 0 ? (unsigned)std::min<int64_t>(lc.n_heavy, 65535) : 0;
        sh.clear_grid = (int)std::max<int64_t>(1, std::min<int64_t>((lc.n_heavy * NW + 255) / 256, (int64_t)sms * 8));
        s = emit_push<W, NW, OffT>(p, g, cur, sh, kb, c->stream, &launches);
        if (st) st->push_levels++;
      } else {
        s = emit_pull<W, NW, OffT>(p, g, cur, sh, kb, c->stream, &launches);
        if (st) st->pull_levels++;
      }
      if (s != XB_OK) return s;
      timer.end(0, launches);
      cur ^= 1;
    }
    max_levels = std::max(max_levels, c->h_ctr->b.level);
    timer.begin();
    int64_t launches = 0;
    int32_t* lv_base = out_dev ? level_out + k0 * n : c->d_stage;
    int32_t* pr_base = out_dev ? parent_out + k0 * n : c->d_stage + (size_t)SPP * n;
    s = emit_tables<W, NW, OffT>(p, g, d_sources + k0, kb, lv_base, pr_base, c->h_ctr->b.pushed_deep != 0, c->stream,
                                 sms, &launches);
    if (s != XB_OK) return s;
    timer.end(1, launches);
    if (!out_dev) {
      XB_CUDA(cudaMemcpyAsync(level_out + k0 * n, lv_base, sizeof(int32_t) * (size_t)kb * n, cudaMemcpyDeviceToHost,
                              c->stream));
      XB_CUDA(cudaMemcpyAsync(parent_out + k0 * n, pr_base, sizeof(int32_t) * (size_t)kb * n, cudaMemcpyDeviceToHost,
                              c->stream));
    }
    XB_CUDA(cudaMemcpyAsync(c->h_ctr, p.ctr, sizeof(xbk::Ctrs), cudaMemcpyDeviceToHost, c->stream));
    XB_CUDA(cudaStreamSynchronize(c->stream));
    if (st) {
      const xbk::BatchCtr& b = c->h_ctr->b;
      st->edges_traversed += (int64_t)b.edges_traversed;
      st->reached += (int64_t)b.reached;
      st->edges_scanned += (int64_t)b.edges_scanned;
      st->vertices_scanned += (int64_t)b.vertices_scanned;
      st->vertices_swept += (int64_t)b.vertices_swept;
      st->parent_edges_scanned += (int64_t)b.parent_edges;
      st->batches += 1;
      const int64_t lvl_bytes = level_bytes<W, NW, OffT>(b);
      const int64_t tab_bytes = table_bytes<W, NW, OffT>(b, n, kb);
      st->class_bytes[0] += lvl_bytes;
      st->class_bytes[1] += tab_bytes;
      st->algo_bytes += lvl_bytes + tab_bytes;
    }
  }
  if (st) st->levels = std::max(st->levels, max_levels);
  return XB_OK;
}

template <typename W, typename OffT>
xb_status dispatch_nw(xb_ctx* c, xb_graph* g, const int32_t* d_src, int32_t k, int32_t* lv, int32_t* pr, bool od,
                      xb_stats* st) {
  switch (c->tuning.words) {
    case 1: return run_plain<W, 1, OffT>(c, g, d_src, k, lv, pr, od, st);
    case 2: return run_plain<W, 2, OffT>(c, g, d_src, k, lv, pr, od, st);
    case 4: return run_plain<W, 4, OffT>(c, g, d_src, k, lv, pr, od, st);
    default: return fail(XB_ERR_ARG, "tuning.words must be 1, 2 or 4");
  }
}

}  // namespace

extern "C" {

xb_status xb_ctx_create(int32_t device, xb_ctx** out) {
  xbi::clear_error();
  if (!out) return fail(XB_ERR_ARG, "null out");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(XB_ERR_NODEV, std::string("no CUDA device: ") + cudaGetErrorString(e));
  }
  if (device < 0 || device >= ndev) return fail(XB_ERR_ARG, "device index out of range");
  XB_CUDA(cudaSetDevice(device));
  std::unique_ptr<xb_ctx> c(new xb_ctx());
  c->device = device;
  XB_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
  XB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  XB_CUDA(cudaMalloc(&c->d_ctr, sizeof(xbk::Ctrs)));
  XB_CUDA(cudaMemset(c->d_ctr, 0, sizeof(xbk::Ctrs)));  // epoch 0: below every step's stamp
  XB_CUDA(cudaMallocHost(&c->h_ctr, sizeof(xbk::Ctrs)));
  XB_CUDA(cudaEventCreate(&c->ev0));
  XB_CUDA(cudaEventCreate(&c->ev1));
  XB_CUDA(cudaEventCreate(&c->evc0));
  XB_CUDA(cudaEventCreate(&c->evc1));
  c->tuning.word_bits = 64;
  c->tuning.words = 1;
  // pull unless the frontier's edges are under 1/64 of the unfinished edges:
  // pull steps record parents as they go, push steps leave them to a search
  c->tuning.pull_alpha = 64.0f;
  c->tuning.heavy_degree = 256;
  c->tuning.timing = 0;
  *out = c.release();
  return XB_OK;
}

xb_status xb_ctx_destroy(xb_ctx* c) {
  xbi::clear_error();
  if (!c) return XB_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->ws) cudaFree(c->ws);
  if (c->d_src) cudaFree(c->d_src);
  if (c->d_stage) cudaFree(c->d_stage);
  if (c->d_ctr) cudaFree(c->d_ctr);
  if (c->h_ctr) cudaFreeHost(c->h_ctr);
  for (cudaEvent_t ev : {c->ev0, c->ev1, c->evc0, c->evc1})
    if (ev) cudaEventDestroy(ev);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return XB_OK;
}

xb_status xb_ctx_set_tuning(xb_ctx* c, const xb_tuning* t) {
  xbi::clear_error();
  if (!c || !t) return fail(XB_ERR_ARG, "null argument");
  if (t->word_bits != 32 && t->word_bits != 64) return fail(XB_ERR_ARG, "word_bits must be 32 or 64");
  if (t->words != 1 && t->words != 2 && t->words != 4) return fail(XB_ERR_ARG, "words must be 1, 2 or 4");
  if (!(t->pull_alpha > 0)) return fail(XB_ERR_ARG, "pull_alpha must be positive");
  if (t->heavy_degree < 32 || t->heavy_degree > (1 << 20))
    return fail(XB_ERR_ARG, "heavy_degree must be in [32, 2^20]");
  c->tuning = *t;
  return XB_OK;
}

xb_status xb_ctx_get_tuning(const xb_ctx* c, xb_tuning* t) {
  xbi::clear_error();
  if (!c || !t) return fail(XB_ERR_ARG, "null argument");
  *t = c->tuning;
  return XB_OK;
}

xb_status xb_ctx_workspace_bytes(const xb_ctx* c, int64_t* bytes) {
  xbi::clear_error();
  if (!c || !bytes) return fail(XB_ERR_ARG, "null argument");
  *bytes = (int64_t)(c->ws_bytes + c->stage_bytes + sizeof(int32_t) * c->src_cap);
  return XB_OK;
}

xb_status xb_ctx_get_stream(const xb_ctx* c, void** stream) {
  xbi::clear_error();
  if (!c || !stream) return fail(XB_ERR_ARG, "null argument");
  *stream = (void*)c->stream;
  return XB_OK;
}

xb_status xb_graph_upload(xb_ctx* c, int64_t n, const void* row_offsets, int32_t offsets_are_64bit, int64_t m,
                          const int32_t* col_indices, xb_graph** out) {
  xbi::clear_error();
  if (!c || !out || !row_offsets) return fail(XB_ERR_ARG, "null argument");
  if (n < 1 || n >= INT32_MAX) return fail(XB_ERR_ARG, "n must be in [1, 2^31-1)");
  std::vector<int64_t> ro((size_t)n + 1);
  if (offsets_are_64bit) {
    std::memcpy(ro.data(), row_offsets, sizeof(int64_t) * (n + 1));
  } else {
    const int32_t* r32 = (const int32_t*)row_offsets;
    for (int64_t i = 0; i <= n; i++) ro[i] = r32[i];
  }
  if (ro[n] != m) return fail(XB_ERR_ARG, "row_offsets[n] != m");
  xb_status s = xbi::validate_csr(n, ro.data(), col_indices);
  if (s != XB_OK) return s;
  XB_CUDA(cudaSetDevice(c->device));
  std::unique_ptr<xb_graph> g(new xb_graph());
  g->ctx = c;
  g->n = n;
  g->m = m;
  g->off64 = m >= (int64_t)INT32_MAX;
  for (int64_t v = 0; v < n; v++) g->max_deg = std::max(g->max_deg, ro[v + 1] - ro[v]);
  const size_t ro_bytes = (g->off64 ? 8 : 4) * (size_t)(n + 1);
  if (cudaMalloc(&g->d_ro, ro_bytes) != cudaSuccess ||
      cudaMalloc(&g->d_ci, sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1)) != cudaSuccess) {
    cudaGetLastError();
    if (g->d_ro) cudaFree(g->d_ro);
    if (g->d_ci) cudaFree(g->d_ci);
    return fail(XB_ERR_OOM, "graph allocation failed");
  }
  if (g->off64) {
    XB_CUDA(cudaMemcpy(g->d_ro, ro.data(), ro_bytes, cudaMemcpyHostToDevice));
  } else {
    std::vector<int32_t> r32((size_t)n + 1);
    for (int64_t i = 0; i <= n; i++) r32[i] = (int32_t)ro[i];
    XB_CUDA(cudaMemcpy(g->d_ro, r32.data(), ro_bytes, cudaMemcpyHostToDevice));
  }
  if (m > 0) XB_CUDA(cudaMemcpy(g->d_ci, col_indices, sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice));
  g->h_ro = std::move(ro);
  *out = g.release();
  return XB_OK;
}

xb_status xb_graph_from_host_csr(xb_ctx* c, const xb_host_csr* h, xb_graph** out) {
  xbi::clear_error();
  if (!h) return fail(XB_ERR_ARG, "null host csr");
  return xb_graph_upload(c, h->n, h->ro.data(), 1, h->ro[h->n], h->ci.data(), out);
}

xb_status xb_graph_load_csr_text(xb_ctx* c, const char* row_path, const char* col_path, xb_graph** out) {
  xb_host_csr* h = nullptr;
  xb_status s = xb_csr_load_text(row_path, col_path, &h);
  if (s != XB_OK) return s;
  s = xb_graph_from_host_csr(c, h, out);
  xb_csr_free(h);
  return s;
}

xb_status xb_graph_free(xb_graph* g) {
  xbi::clear_error();
  if (!g) return XB_OK;
  cudaSetDevice(g->ctx->device);
  if (g->d_ro) cudaFree(g->d_ro);
  if (g->d_ci) cudaFree(g->d_ci);
  if (g->d_heavy) cudaFree(g->d_heavy);
  if (g->d_hpar) cudaFree(g->d_hpar);
  if (g->d_hitems) cudaFree(g->d_hitems);
  if (g->d_hub_items) cudaFree(g->d_hub_items);
  if (g->d_hidx_of) cudaFree(g->d_hidx_of);
  delete g;
  return XB_OK;
}

xb_status xb_graph_info(const xb_graph* g, int64_t* n, int64_t* m, int64_t* max_degree) {
  xbi::clear_error();
  if (!g) return fail(XB_ERR_ARG, "null graph");
  if (n) *n = g->n;
  if (m) *m = g->m;
  if (max_degree) *max_degree = g->max_deg;
  return XB_OK;
}

xb_status xb_select_sources(const xb_graph* g, uint64_t seed, int32_t k, int32_t* out) {
  xbi::clear_error();
  if (!g) return fail(XB_ERR_ARG, "null graph");
  return xbi::select_sources(g->n, g->h_ro.data(), seed, k, out);
}

xb_status xb_traverse(xb_ctx* c, const xb_graph* gc, const int32_t* sources, int32_t k, int32_t mode,
                      const int32_t* matching, int32_t* level, int32_t* parent, int32_t* owner, uint32_t flags,
                      xb_stats* st) {
  xbi::clear_error();
  xb_graph* g = const_cast<xb_graph*>(gc);
  if (!c || !g) return fail(XB_ERR_ARG, "null context or graph");
  if (g->ctx->device != c->device) return fail(XB_ERR_ARG, "graph lives on another device");
  if (mode != XB_MODE_PLAIN) return fail(XB_ERR_ARG, "only XB_MODE_PLAIN is supported by xb_traverse");
  if (matching || owner) return fail(XB_ERR_ARG, "matching/owner must be NULL in plain mode");
  if (k < 0) return fail(XB_ERR_ARG, "negative source count");
  if (k > 0 && (!sources || !level || !parent)) return fail(XB_ERR_ARG, "null sources or output tables");
  if (st) std::memset(st, 0, sizeof(*st));
  if (k == 0) return XB_OK;
  XB_CUDA(cudaSetDevice(c->device));
  const bool src_dev = (flags & XB_SOURCES_DEVICE) != 0;
  const bool out_dev = (flags & XB_OUT_DEVICE) != 0;
  // validate sources (host copy)
  std::vector<int32_t> hs((size_t)k);
  if (src_dev) {
    XB_CUDA(cudaMemcpy(hs.data(), sources, sizeof(int32_t) * k, cudaMemcpyDeviceToHost));
  } else {
    std::memcpy(hs.data(), sources, sizeof(int32_t) * k);
  }
  for (int32_t i = 0; i < k; i++)
    if (hs[i] < 0 || hs[i] >= g->n) return fail(XB_ERR_ARG, "source " + std::to_string(i) + " out of range");
  xb_status s = ensure_sources(c, k);
  if (s != XB_OK) return s;
  XB_CUDA(cudaMemcpyAsync(c->d_src, hs.data(), sizeof(int32_t) * k, cudaMemcpyHostToDevice, c->stream));
  XB_CUDA(cudaEventRecord(c->ev0, c->stream));
  if (c->tuning.word_bits == 64) {
    s = g->off64 ? dispatch_nw<unsigned long long, int64_t>(c, g, c->d_src, k, level, parent, out_dev, st)
                 : dispatch_nw<unsigned long long, int32_t>(c, g, c->d_src, k, level, parent, out_dev, st);
  } else {
    s = g->off64 ? dispatch_nw<unsigned int, int64_t>(c, g, c->d_src, k, level, parent, out_dev, st)
                 : dispatch_nw<unsigned int, int32_t>(c, g, c->d_src, k, level, parent, out_dev, st);
  }
  if (s != XB_OK) {
    cudaStreamSynchronize(c->stream);
    c->ws_key[0] = -1;  // the zero invariants may be broken: clear on the next call
    return s;
  }
  XB_CUDA(cudaEventRecord(c->ev1, c->stream));
  XB_CUDA(cudaEventSynchronize(c->ev1));
  if (st) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    st->device_ms = ms;
  }
  return XB_OK;
}

}  // extern "C"
