// xb_engine_common.cuh -- definitions shared by the plain path (xb_engine.cu)
// and the batched path (xb_batched.cu) of libxbtrav.so: the context and
// graph objects, the workspace layout of one traversal pass and the functions
// that enqueue a pass's kernels on a stream.  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "xb_internal.h"
#include "xb_kernels.cuh"

namespace xbe {
struct BatchState;
}

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
  int32_t** d_rows = nullptr;  // row-pointer tables of the table pass (2*B per word)
  int64_t rows_cap = 0;
  int32_t* d_fifo = nullptr;  // work areas of the FIFO-parent pass
  size_t fifo_cap = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evc0 = nullptr, evc1 = nullptr;
  xbe::BatchState* batch = nullptr;  // resources of xb_traverse_batched (created on first use)
  std::vector<xb_graph*> graphs;     // live graphs uploaded through this context
};

// Device CSR arrays, shared by the graphs that view them (one upload, or all
// instances of a batch upload); freed with the last view.
struct xb_csr_store {
  int device = 0;
  void* ro = nullptr;
  int32_t* ci = nullptr;
  ~xb_csr_store() {
    if (ro || ci) {
      cudaSetDevice(device);
      if (ro) cudaFree(ro);
      if (ci) cudaFree(ci);
    }
  }
};

struct xb_graph {
  xb_ctx* ctx = nullptr;  // null once the context is destroyed (the graph can only be freed then)
  int64_t n = 0, m = 0, max_deg = 0;
  bool off64 = false;
  std::shared_ptr<xb_csr_store> store;
  void* d_ro = nullptr;     // this graph's row offsets inside store->ro
  int32_t* d_ci = nullptr;  // this graph's colIndices inside store->ci (16-byte aligned)
  std::vector<int64_t> h_ro;
  int32_t* d_heavy = nullptr;  // vertices with degree > heavy_thr, ascending
  int32_t* d_hpar = nullptr;   // per heavy vertex, 64 parent slots of the table pass
  int2* d_hitems = nullptr;    // (heavy index, chunk) items of the table pass
  int64_t n_hitems = 0;
  int2* d_hub_items = nullptr;  // (heavy index, chunk) items of the hub pull
  int64_t n_hub_items = 0;
  int32_t* d_hidx_of = nullptr;  // vertex -> index in the heavy list (-1 for light)
  int32_t* d_lorder = nullptr;   // light vertices (degree 1..heavy_thr) by falling degree
  int64_t n_lorder = 0;
  int32_t* d_lchunk = nullptr;   // chunk starts in d_lorder (n_lchunks + 1 entries)
  int32_t n_lchunks = 0;
  int32_t n_heavy = 0;
  int32_t heavy_thr = -1;
  uint64_t version = 0;  // bumped whenever the heavy-vertex arrays are rebuilt
  int32_t* d_w = nullptr;  // edge weights (xb_graph_set_weights), one per colIndices entry
  std::vector<int64_t> h_reach2;  // per vertex, its neighbours' degree sum (computed on first use)
};

namespace xbe {

using xbi::fail;

// Edges per work item of the heavy-vertex table scan.
constexpr int kTableChunk = 4096;
// Vertices above this degree (hubs) are pulled in chunks by many warps; the
// other heavy vertices by one warp each.
constexpr int kHubDegree = 4096;
constexpr int kHubChunk = 2048;
// Parent slots per heavy vertex: up to 64 sources x 4 words.
constexpr int kHparRow = 256;
// Source rows whose FIFO parents are computed at once (one block each).
constexpr int kFifoGroup = 64;
// Zero entries allocated past the end of a resident colIndices array.
constexpr int64_t kCiPad = 16;

struct WsLayout {
  size_t seen, F, N, p01, ph, pushed, p8, touched, fl_light, fl_heavy, nl_light, nl_heavy, stamp, fbits, nbits, cdone,
      total;
  int64_t plane_stride;  // in words
  int nplanes_alloc;
};

inline int bitlen_levels(int64_t n) {
  // levels are in [0, n-1]; number of bits to hold n-1, at least 3
  int b = 0;
  int64_t x = n > 1 ? n - 1 : 0;
  while (x) {
    b++;
    x >>= 1;
  }
  return std::max(3, b);
}

inline size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

inline WsLayout layout_for(int64_t n, int word_bytes, int nw) {
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
  const size_t bw = align_up((size_t)((std::max<int64_t>(n, 1) + 31) / 32) * 4);  // one bit per vertex
  L.fbits = o; o += bw;
  L.nbits = o; o += bw;
  L.cdone = o; o += align_up((size_t)std::max<int64_t>(n, 1));  // one byte per light chunk (at most n)
  L.total = o;
  return L;
}

// Builds (or keeps) the graph's heavy-vertex arrays for cutoff thr.
xb_status ensure_heavy(xb_graph* g, int thr);
// Fills g->h_reach2 (once per graph) on the graph's context's device.
xb_status ensure_reach2(xb_graph* g);

// Releases the batched path's resources of a context.
void batch_state_free(BatchState* b);
// Drops the batched path's cached graphs that reference g.
void batch_forget_graph(xb_ctx* c, const xb_graph* g);

// Creates a conditional handle in the graph stream s is capturing into.
inline xb_status make_handle(cudaStream_t s, unsigned dflt, unsigned flags, cudaGraphConditionalHandle* h) {
  cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  XB_CUDA(cudaStreamGetCaptureInfo(s, &cst, nullptr, &g, nullptr, nullptr));
  if (cst != cudaStreamCaptureStatusActive) return fail(XB_ERR_STATE, "stream is not capturing");
  XB_CUDA(cudaGraphConditionalHandleCreate(h, g, dflt, flags));
  return XB_OK;
}

// Adds a conditional node on handle h after the work captured so far on s and
// makes it the stream's only dependency; returns its body graphs.
inline xb_status add_conditional(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                          unsigned size, cudaGraph_t* bodies) {
  cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  XB_CUDA(cudaStreamGetCaptureInfo(s, &cst, nullptr, &g, &deps, &nd));
  if (cst != cudaStreamCaptureStatusActive) return fail(XB_ERR_STATE, "stream is not capturing");
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = type;
  np.conditional.size = size;
  cudaGraphNode_t node = nullptr;
  XB_CUDA(cudaGraphAddNode(&node, g, deps, nd, &np));
  for (unsigned i = 0; i < size; i++) bodies[i] = np.conditional.phGraph_out[i];
  XB_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
  return XB_OK;
}

// Ends a capture into a body graph whatever happened inside it; keeps the
// first error.
inline xb_status end_body(cudaStream_t s, xb_status st) {
  cudaGraph_t out = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &out);
  if (st != XB_OK) return st;
  if (e != cudaSuccess) return fail(XB_ERR_CUDA, std::string("body capture: ") + cudaGetErrorString(e));
  return XB_OK;
}

xb_status ensure_scratch(xb_ctx* c, size_t bytes, const char* what);

// Level at which a pass's loop stops with the error flag: the structural
// bound 2^planes (levels of a correct traversal stay below it), or the
// context's tuning.level_cap when that is lower.
inline int level_bound(const xb_ctx* c, int nplanes_alloc) {
  int64_t b = nplanes_alloc >= 31 ? (int64_t)INT32_MAX : ((int64_t)1 << nplanes_alloc);
  if (c->tuning.level_cap > 0) b = std::min<int64_t>(b, c->tuning.level_cap);
  return (int)b;
}

// Frontier size below which a step after a pull pushes (tuning.push_beta;
// 0 = the alpha rule alone).
inline long long push_below(const xb_ctx* c, const xb_graph* g) {
  return c->tuning.push_beta > 0 ? (long long)((double)g->n / (double)c->tuning.push_beta) : 0;
}

// Stable order of sources by out-degree, highest first, equal degrees by
// their neighbours' degree sum, highest first (the pass grouping of
// tuning.source_order 0: a pass's sources then reach the graph's core at the
// same level).  key(i) gives the i-th source's vertex.
template <typename Key>
xb_status order_by_degree(xb_graph* g, std::vector<int64_t>& order, Key key) {
  const xb_status s = ensure_reach2(g);
  if (s != XB_OK) return s;
  const int64_t* ro = g->h_ro.data();
  const int64_t* r2 = g->h_reach2.data();
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
    const int64_t va = key(a), vb = key(b);
    const int64_t da = ro[va + 1] - ro[va], db = ro[vb + 1] - ro[vb];
    return da != db ? da > db : r2[va] > r2[vb];
  });
  return XB_OK;
}

// Refuses a working-memory allocation above the context's tuning.workspace_cap.
inline xb_status check_workspace_cap(const xb_ctx* c, size_t bytes, const char* what) {
  if (c->tuning.workspace_cap > 0 && (int64_t)bytes > c->tuning.workspace_cap)
    return fail(XB_ERR_OOM, std::string(what) + " of " + std::to_string(bytes) +
                                " bytes exceeds the workspace cap of " + std::to_string(c->tuning.workspace_cap));
  return XB_OK;
}
xb_status traverse_alternating(xb_ctx* c, xb_graph* g, const int32_t* matching, int32_t* level, int32_t* parent,
                               int32_t* owner, uint32_t flags, xb_stats* st);

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

template <typename W, int NW, typename OffT>
int64_t level_bytes(const xbk::BatchCtr& b) {
  return xbk::level_bytes_of(b, (int)sizeof(OffT) * 2, (int)sizeof(W), NW);
}

template <typename W, int NW, typename OffT>
int64_t table_bytes(const xbk::BatchCtr& b, int64_t n, int kb) {
  return xbk::table_bytes_of(b, n, kb, (int)sizeof(OffT) * 2, (int)sizeof(W), NW);
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
  int tile = 0;  // xb_tuning.tile: launch tile of the pull and table kernels
  size_t state_bytes = 0, plane_bytes = 0, ppos_bytes = 0;
  int64_t bit_words = 0;  // 32-bit words of a frontier bitmap
  uint8_t* cdone = nullptr;  // light chunks with no wanted vertex for the rest of the pass
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
  p.lists[0] = xbk::Lists{(int32_t*)(base + L.fl_light), (int32_t*)(base + L.fl_heavy), (uint32_t*)(base + L.fbits)};
  p.lists[1] = xbk::Lists{(int32_t*)(base + L.nl_light), (int32_t*)(base + L.nl_heavy), (uint32_t*)(base + L.nbits)};
  p.bit_words = (g->n + 31) / 32;
  p.cdone = (uint8_t*)(base + L.cdone);
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
                         cudaStream_t s, int sms, bool clear_frontiers = false) {
  if (clear_frontiers) {  // a workspace shared by passes of other layouts: F, N and the stamps start zero
    XB_CUDA(cudaMemsetAsync(p.buf[0], 0, p.state_bytes, s));
    XB_CUDA(cudaMemsetAsync(p.buf[1], 0, p.state_bytes, s));
    XB_CUDA(cudaMemsetAsync(p.stamp, 0, sizeof(int32_t) * (size_t)p.n, s));
  }
  XB_CUDA(cudaMemsetAsync(p.seen, 0, p.state_bytes, s));
  XB_CUDA(cudaMemsetAsync(p.lists[0].bits, 0, sizeof(uint32_t) * (size_t)p.bit_words, s));
  XB_CUDA(cudaMemsetAsync(p.lists[1].bits, 0, sizeof(uint32_t) * (size_t)p.bit_words, s));
  XB_CUDA(cudaMemsetAsync(p.pl.p01, 0, 2 * p.plane_bytes, s));
  XB_CUDA(cudaMemsetAsync(p.pl.ph, 0, p.plane_bytes, s));
  XB_CUDA(cudaMemsetAsync(p.pushed, 0, p.state_bytes, s));
  if (g->n_lchunks > 0) XB_CUDA(cudaMemsetAsync(p.cdone, 0, (size_t)g->n_lchunks, s));
  if (g->n_heavy > 0) {  // parent slots of the heavy vertices (hub pulls fold in with atomicMin)
    const int64_t hcount = (int64_t)g->n_heavy * kHparRow;
    xbk::k_fill<int32_t><<<(int)std::min<int64_t>((hcount + 255) / 256, (int64_t)sms * 8), 256, 0, s>>>(p.hpar, hcount,
                                                                                                   INT32_MAX);
  }
  xbk::k_pass_init<<<1, 1, 0, s>>>(p.ctr, (long long)g->m);
  xbk::k_init_batch<W, NW, OffT><<<1, 256, 0, s>>>(src, kb, p.ro, p.buf[0], p.seen, p.pl, active_mask<W, NW>(kb),
                                                   p.heavy, p.lists[0], p.ctr, p.ppos);
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
                                                                     p.pushed, fl.bits, p.bit_words, p.ppos);
  (*launches)++;
  XB_LAUNCH_CHECK("push step");
  return XB_OK;
}

// Blocks of `threads` threads of `kernel` resident per SM (occupancy query).
template <typename K>
int resident_blocks(K kernel, int threads) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, 0) != cudaSuccess) {
    cudaGetLastError();
    b = 1;
  }
  return std::max(1, b);
}

// Light vertices pulled one per lane (k_pull_lanes) for every layout up to
// four words per vertex; warps per block shrink with the words so the
// per-warp queues and position-plane columns stay within static shared
// memory (8 warps up to two words, 4 for four).
template <int NW>
constexpr bool pull_by_lanes() {
  return NW <= 4;
}
template <int NW>
constexpr int lane_warps() {
  return NW <= 2 ? 8 : 4;
}

// Rounds of 32 edges a heavy-pull warp keeps in flight: one at four words
// per vertex, where the gathered words of a round fill the registers and
// three blocks per SM (80 registers) beat more rounds at two blocks.  Tile 1
// (xb_tuning.tile) keeps two rounds in flight at every layout.
template <int NW>
constexpr int heavy_rounds() {
  return NW == 4 ? 1 : 4;
}
constexpr int kHeavyRoundsTile1 = 2;
// Warps per block of the table pass: 4 at tile 0, 8 at tile 1.
constexpr int kTabWarps0 = 4, kTabWarps1 = 8;

template <typename W, int NW, typename OffT>
xb_status emit_pull(const PassRes<W, NW, OffT>& p, const xb_graph* g, int cur, const StepShape& sh, int kb,
                    cudaStream_t s, int64_t* launches) {
  constexpr int PW = pull_warps<W, NW>();
  W* F = p.buf[cur];
  W* N = p.buf[cur ^ 1];
  const xbk::Lists fl = p.lists[cur], nl = p.lists[cur ^ 1];
  const xbk::Masks<W, NW> active = active_mask<W, NW>(kb);
  if constexpr (pull_by_lanes<NW>()) {
    if (g->n_lorder > 0) {
      xbk::k_pull_lanes<W, NW, OffT, lane_warps<NW>()><<<sh.pull_grid, lane_warps<NW>() * 32, 0, s>>>(
          g->n_lchunks, g->d_lchunk, g->d_lorder, p.ro, p.ci, F, p.seen, N, p.pl, active, p.heavy, nl, p.ctr, cur,
          p.ppos, p.n, fl.bits, p.cdone);
      (*launches)++;
    }
  } else {
    xbk::k_pull_tiles<W, NW, OffT, PW, 4><<<sh.pull_grid, PW * 32, 0, s>>>(p.n, p.ro, p.ci, F, p.seen, N, p.pl,
                                                                           active, p.heavy, nl, p.ctr, cur, p.ppos);
    (*launches)++;
  }
  if (g->n_heavy > 0) {
    // heavy vertices with wanted bits first (into the push steps' touched list,
    // unused by a pull step), then one warp per listed vertex
    xbk::k_heavy_want<W, NW, OffT><<<sh.commit_grid, 256, 0, s>>>(g->d_heavy, g->n_heavy, p.ro, p.seen, active,
                                                                  kHubDegree, p.ctr, cur, p.touched);
    if (p.tile == 1)
      xbk::k_pull_heavy<W, NW, OffT, kHeavyRoundsTile1><<<sh.heavy_grid, 256, 0, s>>>(
          g->d_heavy, p.touched, p.ro, p.ci, F, p.seen, N, p.pl, active, p.heavy, kHubDegree, nl, p.ctr, cur, p.hpar,
          p.n, fl.bits);
    else
      xbk::k_pull_heavy<W, NW, OffT, heavy_rounds<NW>()><<<sh.heavy_grid, 256, 0, s>>>(
          g->d_heavy, p.touched, p.ro, p.ci, F, p.seen, N, p.pl, active, p.heavy, kHubDegree, nl, p.ctr, cur, p.hpar,
          p.n, fl.bits);
    *launches += 2;
    if (g->n_hub_items > 0) {
      xbk::k_pull_hubs<W, NW, OffT, 4><<<sh.hub_grid, 256, 0, s>>>(g->d_heavy, g->d_hub_items, g->n_hub_items, p.ro,
                                                                   p.ci, F, p.seen, N, active, p.ctr, cur, kHubChunk,
                                                                   p.hpar, p.n, fl.bits);
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

// Table pass of one pass (all its words).  rows (device) holds 2*B row
// pointers per word: rows[wi*2B + s] is the level row and rows[wi*2B + B + s]
// the parent row of the word's source s.
template <typename W, int NW, typename OffT>
xb_status emit_tables(const PassRes<W, NW, OffT>& p, const xb_graph* g, const int32_t* src, int kb,
                      int32_t* const* rows, bool search_heavy, cudaStream_t s, int sms, int64_t* launches,
                      xbk::RowDigest* dig = nullptr) {
  constexpr int B = xbk::WB<W>::bits;
  const int TAB_WARPS = p.tile == 1 ? kTabWarps1 : kTabWarps0;
  const int64_t ntiles = (p.n + 31) / 32;
  const int tab_grid = (int)std::max<int64_t>(
      1, std::min<int64_t>((ntiles + TAB_WARPS - 1) / TAB_WARPS, (int64_t)sms * 16 * kTabWarps0 / TAB_WARPS));
  for (int wi = 0; wi < NW; wi++) {
    if (kb - wi * B <= 0) break;
    if (g->n_heavy > 0 && search_heavy) {
      // heavy vertices reached by a push step at level >= 2: search their parents
      const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((g->n_hitems + 31) / 32, (int64_t)sms * 8));
      xbk::k_tables_heavy_scan<W, NW, OffT><<<grid, 256, 0, s>>>(g->d_heavy, g->d_hitems, g->n_hitems, p.ro, p.ci,
                                                                 p.seen, p.pl, wi, kTableChunk, p.hpar, p.ctr,
                                                                 p.pushed);
      (*launches)++;
    }
  }
  // all words of the pass in one launch (a tile's words share sectors)
  // dig: every row is digest-only; the table pass sums the digests instead
  // of writing rows
  if (dig && p.tile == 1)
    xbk::k_tables<W, NW, OffT, kTabWarps1, 2, true><<<tab_grid, kTabWarps1 * 32, 0, s>>>(
        p.n, p.ro, p.ci, p.seen, p.pl, kb, p.heavy, rows, p.ctr, p.ppos, p.pushed, src, g->d_hidx_of, p.hpar, dig);
  else if (dig)
    xbk::k_tables<W, NW, OffT, kTabWarps0, 4, true><<<tab_grid, kTabWarps0 * 32, 0, s>>>(
        p.n, p.ro, p.ci, p.seen, p.pl, kb, p.heavy, rows, p.ctr, p.ppos, p.pushed, src, g->d_hidx_of, p.hpar, dig);
  else if (p.tile == 1)
    xbk::k_tables<W, NW, OffT, kTabWarps1, 2><<<tab_grid, kTabWarps1 * 32, 0, s>>>(
        p.n, p.ro, p.ci, p.seen, p.pl, kb, p.heavy, rows, p.ctr, p.ppos, p.pushed, src, g->d_hidx_of, p.hpar);
  else
    xbk::k_tables<W, NW, OffT, kTabWarps0, 4><<<tab_grid, kTabWarps0 * 32, 0, s>>>(
        p.n, p.ro, p.ci, p.seen, p.pl, kb, p.heavy, rows, p.ctr, p.ppos, p.pushed, src, g->d_hidx_of, p.hpar);
  (*launches)++;
  XB_LAUNCH_CHECK("tables");
  return XB_OK;
}

// Fills a pass's row-pointer table (host side, 2*B per word) for kb sources
// whose level / parent rows start at lv0 / pr0 and follow each other every n
// int32.
template <typename W, int NW>
void fill_rows(int32_t** rows, int kb, int32_t* lv0, int32_t* pr0, int64_t n) {
  constexpr int B = xbk::WB<W>::bits;
  for (int wi = 0; wi < NW; wi++)
    for (int s = 0; s < B; s++) {
      const int j = wi * B + s;
      rows[wi * 2 * B + s] = j < kb ? lv0 + (int64_t)j * n : nullptr;
      rows[wi * 2 * B + B + s] = j < kb ? pr0 + (int64_t)j * n : nullptr;
    }
}

template <typename W, int NW, typename OffT>
StepShape max_shape(const xb_graph* g, int sms, int tile) {
  constexpr int PW = pull_warps<W, NW>();
  StepShape sh{};
  const int64_t n = g->n;
  const int64_t ntiles = (n + 31) / 32;
  sh.push_light_grid = sms * 16;
  sh.push_heavy_grid = dim3((unsigned)std::max<int64_t>(1, std::min<int64_t>((g->max_deg + 2047) / 2048, 64)),
                            (unsigned)std::max<int64_t>(1, std::min<int64_t>(g->n_heavy, 65535)));
  if (g->n_heavy == 0) sh.push_heavy_grid.y = 0;
  sh.finalize_grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8));
  if constexpr (pull_by_lanes<NW>()) {
    // persistent: warps take chunks of the light list from a counter
    constexpr int LW = lane_warps<NW>();
    static const int lane_res = resident_blocks(xbk::k_pull_lanes<W, NW, OffT, LW>, LW * 32);
    sh.pull_grid = (int)std::max<int64_t>(
        1, std::min<int64_t>(((int64_t)g->n_lchunks + LW - 1) / LW, (int64_t)sms * lane_res));
  } else {
    sh.pull_grid = (int)std::max<int64_t>(1, std::min<int64_t>((ntiles + PW - 1) / PW, (int64_t)sms * 8));
  }
  static const int heavy_res0 = resident_blocks(xbk::k_pull_heavy<W, NW, OffT, heavy_rounds<NW>()>, 256);
  static const int heavy_res1 = resident_blocks(xbk::k_pull_heavy<W, NW, OffT, kHeavyRoundsTile1>, 256);
  const int heavy_res = tile == 1 ? heavy_res1 : heavy_res0;
  sh.heavy_grid = (int)std::max<int64_t>(1, std::min<int64_t>((g->n_heavy + 7) / 8, (int64_t)sms * heavy_res));
  sh.hub_grid = (int)std::max<int64_t>(1, std::min<int64_t>((g->n_hub_items + 7) / 8, (int64_t)sms * 16));
  sh.commit_grid = (int)std::max<int64_t>(1, std::min<int64_t>((g->n_heavy + 255) / 256, (int64_t)sms * 4));
  sh.clear_grid = sms * 8;
  return sh;
}

// Launch shapes for steps the device decides (a captured graph): the count-
// driven kernels stride over whatever the frontier holds, so their grids are
// fixed, bounded by the graph's size and by a few waves of the GPU.
template <typename W, int NW, typename OffT>
StepShape graph_shape(const xb_graph* g, int sms, int tile) {
  StepShape sh = max_shape<W, NW, OffT>(g, sms, tile);
  const int64_t n = g->n;
  sh.push_light_grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 7) / 8, (int64_t)sms * 16));
  if (g->n_heavy > 0)
    sh.push_heavy_grid = dim3((unsigned)std::max<int64_t>(1, std::min<int64_t>((g->max_deg + 2047) / 2048, 16)),
                              (unsigned)std::min<int64_t>(g->n_heavy, sms));
  sh.clear_grid = (int)std::max<int64_t>(1, std::min<int64_t>((n * NW + 255) / 256, (int64_t)sms * 8));
  return sh;
}

}  // namespace xbe
