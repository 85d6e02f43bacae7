// xb_batched.cu -- xb_traverse_batched: every query of a batch traversed by
// one launch of a cached CUDA graph.
//
// Plan.  The sources of all queries on the same graph are concatenated and cut
// into passes of B*NW sources (B = 32 or 64 per word), so small queries share
// words; each source row of a pass carries its own output row pointers (the
// table pass writes through a row table), which is what lets one word serve
// several queries.  Passes are spread over C chains by longest-processing-time
// first; a chain owns a workspace, counters and heavy-parent slots and runs its
// passes back to back, while the chains run concurrently.
//
// Graph.  Per pass: the pass init (memsets, counters, sources) at top level,
// then a WHILE node whose body holds two level steps (even and odd frontier
// buffers); each step is k_step_begin (a one-thread kernel that decides push /
// pull / done from the frontier counters and sets the SWITCH handle), the
// level-plane clear, and a SWITCH node with a push body and a pull body whose
// kernels take fixed grids and stride over whatever the frontier holds.
// k_loop_end sets the WHILE handle.  After the loop come the table pass and
// the pass's fold into the per-chain totals; for host outputs the table pass
// writes one of two staging slots of the chain and a D2H copy of that slot
// runs beside the chain's next pass.
//
// The reference drives every level from the host (four D2H scalars and a
// device sync per frontier swap, xblossom_gpu_engine_10.cu:72-185 and
// enode_queue.h:40-64); nothing here returns to the host until the batch ends.
#include <map>
#include <memory>

#include "xb_engine_common.cuh"

using xbi::fail;

namespace xbe {

constexpr int kMaxChains = 16;
constexpr size_t kMaxCached = 8;
// One-pass graphs a serving slot keeps (one per source count seen, at most 64 x 4 words).
constexpr size_t kSlotMaxCached = 80;

struct Chain {
  void* ws = nullptr;
  size_t ws_bytes = 0;
  xbk::Ctrs* ctr = nullptr;
  int32_t* hpar = nullptr;
  size_t hpar_count = 0;
  int32_t* stage = nullptr;  // two slots of 2*SPP rows of n_max int32 (level rows, then parent rows)
  size_t stage_bytes = 0;
  cudaStream_t cs = nullptr, cps = nullptr;  // capture streams: compute, copies
  cudaEvent_t ev_tab = nullptr, ev_free[2] = {nullptr, nullptr}, ev_join = nullptr, ev_join_cp = nullptr;
};

struct CachedGraph {
  std::vector<uint64_t> key;
  cudaGraphExec_t exec = nullptr;
  std::vector<const xb_graph*> graphs;
  uint64_t last_use = 0;
};

// A serving slot: one pass in flight at a time on its own stream, with its
// own workspace (so slots run concurrently), staging, scratch rows for
// digest-only sources, and cached one-pass graphs.
constexpr int kMaxSlots = 16;
constexpr int kSlotMaxRows = 256;  // 64 sources x 4 words

struct SlotState {
  bool init = false, busy = false;
  int priority = 0;  // 1: the slot's stream has the device's greatest priority (xb_slot_set_priority)
  int kb = 0;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  xbk::Ctrs* ctr = nullptr;
  int32_t* hpar = nullptr;
  size_t hpar_bytes = 0;
  int32_t* scratch = nullptr;  // level rows then parent rows of a pass, n_scratch apart
  size_t scratch_bytes = 0;
  int64_t n_scratch = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  int32_t *d_src = nullptr, *h_src = nullptr;
  int32_t **d_rows = nullptr, **h_rows = nullptr;
  int32_t *d_flags = nullptr, *h_flags = nullptr;
  xbk::PassSum *d_sum = nullptr, *h_sum = nullptr;
  xbk::RowDigest *d_dig = nullptr, *h_dig = nullptr;
  std::vector<CachedGraph> cache;
  uint64_t gen = 1, tick = 0;
};

struct BatchState {
  int device = 0;
  SlotState slots[kMaxSlots];
  Chain chains[kMaxChains];
  xbk::PassSum* d_sums = nullptr;  // one per chain
  xbk::PassSum* h_sums = nullptr;  // pinned
  int32_t* d_src = nullptr;
  int32_t* h_src = nullptr;  // pinned
  int64_t src_cap = 0;
  int32_t** d_rows = nullptr;
  int32_t** h_rows = nullptr;  // pinned
  int64_t rows_cap = 0;
  cudaStream_t origin = nullptr, body[2] = {nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr;
  uint64_t gen = 1;  // bumped whenever a buffer a cached graph points at is reallocated
  uint64_t tick = 0;
  std::vector<CachedGraph> cache;
  int level_bound = 0;  // of the pass being captured (xbe::level_bound)
  long long push_below = 0;  // of the pass being captured (xbe::push_below)
};

namespace {

void drop_cache(BatchState* b) {
  for (auto& e : b->cache)
    if (e.exec) cudaGraphExecDestroy(e.exec);
  b->cache.clear();
}

xb_status make_state(xb_ctx* c) {
  if (c->batch) return XB_OK;
  std::unique_ptr<BatchState> b(new BatchState());
  b->device = c->device;
  XB_CUDA(cudaMalloc(&b->d_sums, sizeof(xbk::PassSum) * kMaxChains));
  XB_CUDA(cudaMallocHost(&b->h_sums, sizeof(xbk::PassSum) * kMaxChains));
  XB_CUDA(cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking));
  for (auto& s : b->body) XB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  XB_CUDA(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
  for (auto& ch : b->chains) {
    XB_CUDA(cudaStreamCreateWithFlags(&ch.cs, cudaStreamNonBlocking));
    XB_CUDA(cudaStreamCreateWithFlags(&ch.cps, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&ch.ev_tab, &ch.ev_free[0], &ch.ev_free[1], &ch.ev_join, &ch.ev_join_cp})
      XB_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  }
  c->batch = b.release();
  return XB_OK;
}

// Grows a device buffer to at least `bytes` (contents not kept).
template <typename T>
xb_status grow(T** p, size_t* cap_bytes, size_t bytes, uint64_t* gen, const char* what) {
  if (*cap_bytes >= bytes && *p) return XB_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap_bytes = 0;
  (*gen)++;
  if (cudaMalloc((void**)p, std::max<size_t>(bytes, 256)) != cudaSuccess) {
    cudaGetLastError();
    return fail(XB_ERR_OOM, std::string(what) + " allocation of " + std::to_string(bytes) + " bytes failed");
  }
  *cap_bytes = bytes;
  return XB_OK;
}

// Where one source row of a pass goes.
struct RowDst {
  int32_t item;  // query index
  int32_t idx;   // source index within the query
};

struct PassPlan {
  const xb_graph* g = nullptr;
  int kb = 0;
  int64_t src_off = 0;  // into the batch's source buffer
  std::vector<RowDst> rows;
  bool host = false;  // some row goes to host memory (through a staging slot)
  int chain = 0, slot = 0;
  double cost = 0;
};

// One level step inside the WHILE body (captured on b0): decide, clear the
// new level plane, then SWITCH into the push or the pull body (captured on b1).
template <typename W, int NW, typename OffT>
xb_status capture_step(BatchState* bs, const PassRes<W, NW, OffT>& p, const xb_graph* g, int cur, int kb,
                       float alpha, const StepShape& sh, int sms) {
  cudaStream_t b0 = bs->body[0], b1 = bs->body[1];
  cudaGraphConditionalHandle hsw;
  xb_status st = make_handle(b0, 2, cudaGraphCondAssignDefault, &hsw);
  if (st != XB_OK) return st;
  xbk::k_step_begin<<<1, 1, 0, b0>>>(p.ctr, cur, alpha, p.nplanes_alloc, bs->level_bound, 1, hsw, bs->push_below);
  xbk::k_zero_plane<W><<<(int)std::max<int64_t>(1, std::min<int64_t>((p.n * NW + 255) / 256, (int64_t)sms * 8)), 256,
                         0, b0>>>(p.pl.ph, p.pl.stride, p.n * NW, p.ctr);
  XB_LAUNCH_CHECK("step control");
  cudaGraph_t br[2];
  st = add_conditional(b0, hsw, cudaGraphCondTypeSwitch, 2, br);
  if (st != XB_OK) return st;
  int64_t launches = 0;
  XB_CUDA(cudaStreamBeginCaptureToGraph(b1, br[0], nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  st = end_body(b1, emit_push<W, NW, OffT>(p, g, cur, sh, kb, b1, &launches));
  if (st != XB_OK) return st;
  XB_CUDA(cudaStreamBeginCaptureToGraph(b1, br[1], nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  return end_body(b1, emit_pull<W, NW, OffT>(p, g, cur, sh, kb, b1, &launches));
}

// The level loop of one pass, as a WHILE node on stream s: each iteration
// takes the step on the even buffers, then on the odd ones.
template <typename W, int NW, typename OffT>
xb_status capture_level_loop(BatchState* bs, const PassRes<W, NW, OffT>& p, const xb_graph* g, int kb, float alpha,
                             const StepShape& sh, cudaStream_t s, int sms) {
  cudaGraphConditionalHandle hwhile;
  xb_status st = make_handle(s, 1, cudaGraphCondAssignDefault, &hwhile);
  if (st != XB_OK) return st;
  cudaGraph_t wbody;
  st = add_conditional(s, hwhile, cudaGraphCondTypeWhile, 1, &wbody);
  if (st != XB_OK) return st;
  cudaStream_t b0 = bs->body[0];
  XB_CUDA(cudaStreamBeginCaptureToGraph(b0, wbody, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  for (int cur = 0; cur < 2 && st == XB_OK; cur++) st = capture_step<W, NW, OffT>(bs, p, g, cur, kb, alpha, sh, sms);
  if (st == XB_OK) {
    xbk::k_loop_end<<<1, 1, 0, b0>>>(p.ctr, 0, hwhile);
    if (cudaGetLastError() != cudaSuccess) st = fail(XB_ERR_CUDA, "launch k_loop_end failed");
  }
  return end_body(b0, st);
}

// A pass's resources for capture: workspace, counters, heavy-parent slots.
template <typename W, int NW, typename OffT>
PassRes<W, NW, OffT> capture_res(xb_ctx* c, const xb_graph* g, void* ws, xbk::Ctrs* ctr, int32_t* hpar) {
  const int heavy = std::max(32, c->tuning.heavy_degree);
  PassRes<W, NW, OffT> p = pass_res<W, NW, OffT>(g, ws, layout_for(g->n, (int)sizeof(W), NW), ctr, hpar, heavy);
  p.tile = c->tuning.tile;
  return p;
}

// First half of a captured pass on stream s: init and the device level loop.
template <typename W, int NW, typename OffT>
xb_status capture_pass_levels(xb_ctx* c, BatchState* bs, const PassRes<W, NW, OffT>& p, const xb_graph* g,
                              const int32_t* src, int kb, cudaStream_t s) {
  const int sms = c->num_sms;
  const float alpha = c->tuning.pull_alpha > 0 ? c->tuning.pull_alpha : 256.0f;
  const StepShape sh = graph_shape<W, NW, OffT>(g, sms, p.tile);
  bs->level_bound = level_bound(c, p.nplanes_alloc);
  bs->push_below = push_below(c, g);
  xb_status st = emit_pass_init<W, NW, OffT>(p, g, src, kb, s, sms, true);
  if (st != XB_OK) return st;
  return capture_level_loop<W, NW, OffT>(bs, p, g, kb, alpha, sh, s, sms);
}

// Second half: the table pass through the row table and the fold into *sum.
template <typename W, int NW, typename OffT>
xb_status capture_pass_tables(xb_ctx* c, const PassRes<W, NW, OffT>& p, const xb_graph* g, const int32_t* src,
                              int kb, int32_t* const* rows, xbk::PassSum* sum, cudaStream_t s,
                              xbk::RowDigest* dig = nullptr) {
  constexpr int B = xbk::WB<W>::bits;
  int64_t launches = 0;
  xb_status st = emit_tables<W, NW, OffT>(p, g, src, kb, rows, true, s, c->num_sms, &launches, dig);
  if (st != XB_OK) return st;
  const int hv = g->n_heavy > 0 ? 1 : 0;
  const int words = (kb + B - 1) / B;
  const int fixed_k = hv + 2 + words * hv + 1 + 1;  // fill, init x2, heavy scans, tables, accumulate
  const int push_k = 2 + 2 * hv;
  const int pull_k = 2 + 2 * hv + (g->n_hub_items > 0 ? 2 : 0);
  xbk::k_pass_accum<<<1, 1, 0, s>>>(p.ctr, sum, (long long)g->n, kb, (int)sizeof(OffT) * 2, (int)sizeof(W), NW,
                                    fixed_k, push_k, pull_k);
  XB_LAUNCH_CHECK("pass accumulate");
  return XB_OK;
}

// One pass on its chain's compute stream (and copy stream for host rows).
template <typename W, int NW, typename OffT>
xb_status capture_pass(xb_ctx* c, BatchState* bs, const PassPlan& pp, int64_t rows_off, int64_t n_stage,
                       const std::vector<xb_batch_item>& items, bool slot_used[kMaxChains][2]) {
  constexpr int B = xbk::WB<W>::bits;
  constexpr int SPP = B * NW;
  Chain& ch = bs->chains[pp.chain];
  const xb_graph* g = pp.g;
  const PassRes<W, NW, OffT> p = capture_res<W, NW, OffT>(c, g, ch.ws, ch.ctr, ch.hpar);
  const int32_t* src = bs->d_src + pp.src_off;
  xb_status st = capture_pass_levels<W, NW, OffT>(c, bs, p, g, src, pp.kb, ch.cs);
  if (st != XB_OK) return st;
  if (pp.host && slot_used[pp.chain][pp.slot]) XB_CUDA(cudaStreamWaitEvent(ch.cs, ch.ev_free[pp.slot], 0));
  st = capture_pass_tables<W, NW, OffT>(c, p, g, src, pp.kb, bs->d_rows + rows_off, bs->d_sums + pp.chain, ch.cs);
  if (st != XB_OK) return st;
  if (pp.host) {
    XB_CUDA(cudaEventRecord(ch.ev_tab, ch.cs));
    XB_CUDA(cudaStreamWaitEvent(ch.cps, ch.ev_tab, 0));
    // runs of consecutive rows of the same host query become one copy each
    const int32_t* lv_slot = ch.stage + (size_t)pp.slot * 2 * SPP * n_stage;
    const int32_t* pr_slot = lv_slot + (size_t)SPP * n_stage;
    const int64_t n = g->n;
    for (int j = 0; j < pp.kb;) {
      const xb_batch_item& it = items[pp.rows[j].item];
      if (it.flags & XB_OUT_DEVICE) {
        j++;
        continue;
      }
      int r = j + 1;
      while (r < pp.kb && pp.rows[r].item == pp.rows[j].item && pp.rows[r].idx == pp.rows[r - 1].idx + 1) r++;
      const size_t bytes = sizeof(int32_t) * (size_t)(r - j) * (size_t)n;
      // staging rows are n_stage apart; copy row by row when that differs from n
      if (n_stage == n) {
        XB_CUDA(cudaMemcpyAsync(it.level + (int64_t)pp.rows[j].idx * n, lv_slot + (size_t)j * n_stage, bytes,
                                cudaMemcpyDeviceToHost, ch.cps));
        XB_CUDA(cudaMemcpyAsync(it.parent + (int64_t)pp.rows[j].idx * n, pr_slot + (size_t)j * n_stage, bytes,
                                cudaMemcpyDeviceToHost, ch.cps));
      } else {
        XB_CUDA(cudaMemcpy2DAsync(it.level + (int64_t)pp.rows[j].idx * n, sizeof(int32_t) * n,
                                  lv_slot + (size_t)j * n_stage, sizeof(int32_t) * n_stage, sizeof(int32_t) * n,
                                  (size_t)(r - j), cudaMemcpyDeviceToHost, ch.cps));
        XB_CUDA(cudaMemcpy2DAsync(it.parent + (int64_t)pp.rows[j].idx * n, sizeof(int32_t) * n,
                                  pr_slot + (size_t)j * n_stage, sizeof(int32_t) * n_stage, sizeof(int32_t) * n,
                                  (size_t)(r - j), cudaMemcpyDeviceToHost, ch.cps));
      }
      j = r;
    }
    XB_CUDA(cudaEventRecord(ch.ev_free[pp.slot], ch.cps));
    slot_used[pp.chain][pp.slot] = true;
  }
  return XB_OK;
}

template <typename W, int NW>
xb_status capture_pass_any(xb_ctx* c, BatchState* bs, const PassPlan& pp, int64_t rows_off, int64_t n_stage,
                           const std::vector<xb_batch_item>& items, bool slot_used[kMaxChains][2]) {
  return pp.g->off64 ? capture_pass<W, NW, int64_t>(c, bs, pp, rows_off, n_stage, items, slot_used)
                     : capture_pass<W, NW, int32_t>(c, bs, pp, rows_off, n_stage, items, slot_used);
}

// Captures the whole plan into an executable graph.
template <typename W, int NW>
xb_status capture_plan(xb_ctx* c, BatchState* bs, const std::vector<PassPlan>& plan, int nch,
                       const std::vector<int64_t>& n_stage, const std::vector<xb_batch_item>& items,
                       cudaGraphExec_t* exec) {
  constexpr int SPP = xbk::WB<W>::bits * NW;
  cudaStream_t os = bs->origin;
  XB_CUDA(cudaStreamBeginCapture(os, cudaStreamCaptureModeRelaxed));
  xb_status st = XB_OK;
  bool host_chain[kMaxChains] = {};
  for (const auto& pp : plan) host_chain[pp.chain] |= pp.host;
  auto body = [&]() -> xb_status {
    XB_CUDA(cudaMemsetAsync(bs->d_sums, 0, sizeof(xbk::PassSum) * kMaxChains, os));
    XB_CUDA(cudaEventRecord(bs->ev_fork, os));
    for (int i = 0; i < nch; i++) {
      XB_CUDA(cudaStreamWaitEvent(bs->chains[i].cs, bs->ev_fork, 0));
      if (host_chain[i]) XB_CUDA(cudaStreamWaitEvent(bs->chains[i].cps, bs->ev_fork, 0));
    }
    bool slot_used[kMaxChains][2] = {};
    for (size_t j = 0; j < plan.size(); j++) {
      const xb_status s2 = capture_pass_any<W, NW>(c, bs, plan[j], (int64_t)j * 2 * SPP, n_stage[plan[j].chain],
                                                   items, slot_used);
      if (s2 != XB_OK) return s2;
    }
    for (int i = 0; i < nch; i++) {
      XB_CUDA(cudaEventRecord(bs->chains[i].ev_join, bs->chains[i].cs));
      XB_CUDA(cudaStreamWaitEvent(os, bs->chains[i].ev_join, 0));
      if (host_chain[i]) {
        XB_CUDA(cudaEventRecord(bs->chains[i].ev_join_cp, bs->chains[i].cps));
        XB_CUDA(cudaStreamWaitEvent(os, bs->chains[i].ev_join_cp, 0));
      }
    }
    return XB_OK;
  };
  st = body();
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(os, &graph);
  if (st == XB_OK && e != cudaSuccess) st = fail(XB_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(e));
  if (st == XB_OK) {
    const cudaError_t ei = cudaGraphInstantiate(exec, graph, 0);
    if (ei != cudaSuccess) st = fail(XB_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
  }
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();
  return st;
}

template <typename W, int NW>
xb_status run_batched(xb_ctx* c, const std::vector<xb_batch_item>& items, const std::vector<std::vector<int32_t>>& hsrc,
                      xb_stats* stats) {
  constexpr int B = xbk::WB<W>::bits;
  constexpr int SPP = B * NW;
  xb_status st = make_state(c);
  if (st != XB_OK) return st;
  BatchState* bs = c->batch;
  const int heavy = std::max(32, c->tuning.heavy_degree);

  // ---- plan: group by graph (first appearance), pack sources into passes
  std::vector<const xb_graph*> graphs;
  std::map<const xb_graph*, std::vector<RowDst>> by_graph;
  for (size_t i = 0; i < items.size(); i++) {
    const xb_graph* g = items[i].graph;
    if (items[i].k == 0) continue;
    if (!by_graph.count(g)) graphs.push_back(g);
    auto& v = by_graph[g];
    for (int32_t s = 0; s < items[i].k; s++) v.push_back(RowDst{(int32_t)i, s});
  }
  std::vector<PassPlan> plan;
  int64_t nsrc = 0;
  for (const xb_graph* g : graphs) {
    st = ensure_heavy(const_cast<xb_graph*>(g), heavy);
    if (st != XB_OK) return st;
    auto& v = by_graph[g];
    if (c->tuning.source_order == 0 && v.size() > (size_t)SPP) {  // passes grouped by source degree
      std::vector<int64_t> order(v.size());
      for (size_t j = 0; j < v.size(); j++) order[j] = (int64_t)j;
      st = order_by_degree(const_cast<xb_graph*>(g), order,
                           [&](int64_t j) { return (int64_t)hsrc[v[j].item][v[j].idx]; });
      if (st != XB_OK) return st;
      std::vector<RowDst> sorted(v.size());
      for (size_t j = 0; j < v.size(); j++) sorted[j] = v[order[j]];
      v.swap(sorted);
    }
    for (size_t j0 = 0; j0 < v.size(); j0 += SPP) {
      PassPlan pp;
      pp.g = g;
      pp.kb = (int)std::min<size_t>(SPP, v.size() - j0);
      pp.src_off = nsrc;
      pp.rows.assign(v.begin() + (ptrdiff_t)j0, v.begin() + (ptrdiff_t)(j0 + pp.kb));
      for (const auto& r : pp.rows) pp.host |= !(items[r.item].flags & XB_OUT_DEVICE);
      pp.cost = (double)g->m + 4.0 * (double)g->n;
      nsrc += pp.kb;
      plan.push_back(std::move(pp));
    }
  }
  if (plan.empty()) return XB_OK;
  const int nch = (int)std::min<int64_t>(std::max(1, c->tuning.chains), (int64_t)plan.size());
  {  // longest processing time first; within a chain, passes keep plan order
    std::vector<size_t> order(plan.size());
    for (size_t j = 0; j < order.size(); j++) order[j] = j;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return plan[a].cost > plan[b].cost; });
    std::vector<double> load((size_t)nch, 0.0);
    for (size_t j : order) {
      const int ci = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      plan[j].chain = ci;
      load[(size_t)ci] += plan[j].cost;
    }
    std::vector<PassPlan> sorted;
    sorted.reserve(plan.size());
    for (int ci = 0; ci < nch; ci++)
      for (auto& pp : plan)
        if (pp.chain == ci) sorted.push_back(pp);
    plan.swap(sorted);
    int next_slot[kMaxChains] = {};
    for (auto& pp : plan)
      if (pp.host) {
        pp.slot = next_slot[pp.chain];
        next_slot[pp.chain] ^= 1;
      }
  }

  // ---- per-chain resources
  std::vector<int64_t> n_stage((size_t)nch, 0);
  for (int ci = 0; ci < nch; ci++) {
    size_t ws = 0, hp = 1;
    int64_t nmax_host = 0;
    for (const auto& pp : plan) {
      if (pp.chain != ci) continue;
      ws = std::max(ws, layout_for(pp.g->n, (int)sizeof(W), NW).total);
      hp = std::max(hp, (size_t)std::max(pp.g->n_heavy, 1) * kHparRow);
      if (pp.host) nmax_host = std::max(nmax_host, pp.g->n);
    }
    Chain& ch = bs->chains[ci];
    size_t cap = ch.ws_bytes;
    st = (cap < ws || !ch.ws) ? check_workspace_cap(c, ws, "chain workspace") : XB_OK;
    if (st == XB_OK) st = grow(&ch.ws, &cap, ws, &bs->gen, "chain workspace");
    ch.ws_bytes = cap;
    if (st != XB_OK) return st;
    if (!ch.ctr) {
      XB_CUDA(cudaMalloc(&ch.ctr, sizeof(xbk::Ctrs)));
      XB_CUDA(cudaMemset(ch.ctr, 0, sizeof(xbk::Ctrs)));
      bs->gen++;
    }
    size_t hcap = ch.hpar_count * sizeof(int32_t);
    st = grow(&ch.hpar, &hcap, hp * sizeof(int32_t), &bs->gen, "heavy parent slots");
    ch.hpar_count = hcap / sizeof(int32_t);
    if (st != XB_OK) return st;
    if (nmax_host > 0) {
      size_t scap = ch.stage_bytes;
      st = grow(&ch.stage, &scap, sizeof(int32_t) * 2 * 2 * (size_t)SPP * (size_t)nmax_host, &bs->gen,
                "chain staging");
      ch.stage_bytes = scap;
      if (st != XB_OK) return st;
      n_stage[(size_t)ci] = (int64_t)(ch.stage_bytes / (sizeof(int32_t) * 4 * (size_t)SPP));
    }
  }
  // sources and row tables (pinned host mirrors, uploaded every call)
  const int64_t nrows = (int64_t)plan.size() * 2 * SPP;
  if (bs->src_cap < nsrc) {
    if (bs->d_src) cudaFree(bs->d_src);
    if (bs->h_src) cudaFreeHost(bs->h_src);
    bs->d_src = nullptr;
    bs->h_src = nullptr;
    bs->src_cap = 0;
    bs->gen++;
    if (cudaMalloc(&bs->d_src, sizeof(int32_t) * (size_t)nsrc) != cudaSuccess ||
        cudaMallocHost(&bs->h_src, sizeof(int32_t) * (size_t)nsrc) != cudaSuccess) {
      cudaGetLastError();
      return fail(XB_ERR_OOM, "batch source buffer allocation failed");
    }
    bs->src_cap = nsrc;
  }
  if (bs->rows_cap < nrows) {
    if (bs->d_rows) cudaFree(bs->d_rows);
    if (bs->h_rows) cudaFreeHost(bs->h_rows);
    bs->d_rows = nullptr;
    bs->h_rows = nullptr;
    bs->rows_cap = 0;
    bs->gen++;
    if (cudaMalloc(&bs->d_rows, sizeof(int32_t*) * (size_t)nrows) != cudaSuccess ||
        cudaMallocHost(&bs->h_rows, sizeof(int32_t*) * (size_t)nrows) != cudaSuccess) {
      cudaGetLastError();
      return fail(XB_ERR_OOM, "batch row table allocation failed");
    }
    bs->rows_cap = nrows;
  }
  // the previous launch has finished (every call ends synchronised), so the
  // pinned mirrors may be rewritten
  for (size_t j = 0; j < plan.size(); j++) {
    const PassPlan& pp = plan[j];
    int32_t** rows = bs->h_rows + (int64_t)j * 2 * SPP;
    const int64_t ns = n_stage[(size_t)pp.chain];
    int32_t* lv_slot = pp.host ? bs->chains[pp.chain].stage + (size_t)pp.slot * 2 * SPP * ns : nullptr;
    int32_t* pr_slot = pp.host ? lv_slot + (size_t)SPP * ns : nullptr;
    for (int s = 0; s < SPP; s++) {
      const int wi = s / B, b = s % B;
      int32_t* lv = nullptr;
      int32_t* pr = nullptr;
      if (s < pp.kb) {
        const RowDst r = pp.rows[s];
        const xb_batch_item& it = items[r.item];
        bs->h_src[pp.src_off + s] = hsrc[r.item][r.idx];
        if (it.flags & XB_OUT_DEVICE) {
          lv = it.level + (int64_t)r.idx * pp.g->n;
          pr = it.parent + (int64_t)r.idx * pp.g->n;
        } else {
          lv = lv_slot + (size_t)s * ns;
          pr = pr_slot + (size_t)s * ns;
        }
      }
      rows[wi * 2 * B + b] = lv;
      rows[wi * 2 * B + B + b] = pr;
    }
  }

  // ---- cached executable graph for this plan shape
  std::vector<uint64_t> key = {bs->gen,
                               (uint64_t)sizeof(W),
                               (uint64_t)NW,
                               (uint64_t)heavy,
                               0,
                               (uint64_t)nch,
                               (uint64_t)items.size(),
                               (uint64_t)c->tuning.level_cap,
                               (uint64_t)c->tuning.tile,
                               0};
  {
    uint32_t abits = 0, bbits = 0;
    std::memcpy(&abits, &c->tuning.pull_alpha, sizeof(abits));
    std::memcpy(&bbits, &c->tuning.push_beta, sizeof(bbits));
    key[4] = abits;
    key[9] = bbits;
  }
  bool any_host = false;
  for (const auto& it : items) {
    key.push_back((uint64_t)(uintptr_t)it.graph);
    key.push_back(it.graph->version);
    key.push_back((uint64_t)it.k);
    key.push_back((uint64_t)(it.flags & XB_OUT_DEVICE));
    if (!(it.flags & XB_OUT_DEVICE) && it.k > 0) {
      key.push_back((uint64_t)(uintptr_t)it.level);
      key.push_back((uint64_t)(uintptr_t)it.parent);
      any_host = true;
    }
  }
  // the captured host copies follow the rows' pass grouping, which depends
  // on the sources when they are grouped by degree
  if (any_host && c->tuning.source_order == 0)
    for (const auto& pp : plan)
      for (const auto& r : pp.rows) key.push_back(((uint64_t)(uint32_t)r.item << 32) | (uint32_t)r.idx);
  CachedGraph* hit = nullptr;
  for (auto& e : bs->cache)
    if (e.key == key) hit = &e;
  if (!hit) {
    // entries made before a reallocation point at freed buffers
    for (size_t i = 0; i < bs->cache.size();) {
      if (bs->cache[i].key[0] != bs->gen) {
        cudaGraphExecDestroy(bs->cache[i].exec);
        bs->cache.erase(bs->cache.begin() + (ptrdiff_t)i);
      } else {
        i++;
      }
    }
    if (bs->cache.size() >= kMaxCached) {
      auto lru = std::min_element(bs->cache.begin(), bs->cache.end(),
                                  [](const CachedGraph& a, const CachedGraph& b) { return a.last_use < b.last_use; });
      cudaGraphExecDestroy(lru->exec);
      bs->cache.erase(lru);
    }
    // the capture streams must not hold work of an earlier call
    XB_CUDA(cudaStreamSynchronize(c->stream));
    CachedGraph e;
    e.key = key;
    e.graphs = graphs;
    st = capture_plan<W, NW>(c, bs, plan, nch, n_stage, items, &e.exec);
    if (st != XB_OK) return st;
    bs->cache.push_back(std::move(e));
    hit = &bs->cache.back();
  }
  hit->last_use = ++bs->tick;

  // ---- launch
  XB_CUDA(cudaMemcpyAsync(bs->d_src, bs->h_src, sizeof(int32_t) * (size_t)nsrc, cudaMemcpyHostToDevice, c->stream));
  XB_CUDA(cudaMemcpyAsync(bs->d_rows, bs->h_rows, sizeof(int32_t*) * (size_t)nrows, cudaMemcpyHostToDevice,
                          c->stream));
  XB_CUDA(cudaEventRecord(c->ev0, c->stream));
  XB_CUDA(cudaGraphLaunch(hit->exec, c->stream));
  XB_CUDA(cudaEventRecord(c->ev1, c->stream));
  XB_CUDA(cudaMemcpyAsync(bs->h_sums, bs->d_sums, sizeof(xbk::PassSum) * kMaxChains, cudaMemcpyDeviceToHost,
                          c->stream));
  XB_CUDA(cudaStreamSynchronize(c->stream));
  for (int ci = 0; ci < nch; ci++)
    if (bs->h_sums[ci].errors)
      return fail(XB_ERR_STATE, "a pass's level loop ran past the level bound (corrupted traversal state)");
  if (stats) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    stats->device_ms = ms;
    for (int ci = 0; ci < nch; ci++) {
      const xbk::PassSum& s = bs->h_sums[ci];
      stats->edges_traversed += (int64_t)s.edges_traversed;
      stats->reached += (int64_t)s.reached;
      stats->edges_scanned += (int64_t)s.edges_scanned;
      stats->vertices_scanned += (int64_t)s.vertices_scanned;
      stats->vertices_swept += (int64_t)s.vertices_swept;
      stats->parent_edges_scanned += (int64_t)s.parent_edges;
      stats->class_bytes[0] += (int64_t)s.level_bytes;
      stats->class_bytes[1] += (int64_t)s.table_bytes;
      stats->algo_bytes += (int64_t)(s.level_bytes + s.table_bytes);
      stats->levels = std::max(stats->levels, s.max_level);
      stats->push_levels += s.push_levels;
      stats->pull_levels += s.pull_levels;
      stats->batches += s.passes;
    }
    for (int ci = 0; ci < nch; ci++) stats->class_launches[2] += (int64_t)bs->h_sums[ci].launches;
  }
  return XB_OK;
}

}  // namespace

namespace {

void slot_free(SlotState& sl) {
  if (sl.stream) cudaStreamSynchronize(sl.stream);
  for (auto& e : sl.cache)
    if (e.exec) cudaGraphExecDestroy(e.exec);
  sl.cache.clear();
  for (void* p : {(void*)sl.ws, (void*)sl.ctr, (void*)sl.hpar, (void*)sl.scratch, (void*)sl.d_src, (void*)sl.d_rows,
                  (void*)sl.d_flags, (void*)sl.d_sum, (void*)sl.d_dig})
    if (p) cudaFree(p);
  for (void* p : {(void*)sl.h_src, (void*)sl.h_rows, (void*)sl.h_flags, (void*)sl.h_sum, (void*)sl.h_dig})
    if (p) cudaFreeHost(p);
  if (sl.done) cudaEventDestroy(sl.done);
  if (sl.stream) cudaStreamDestroy(sl.stream);
  const int prio = sl.priority;  // a setting, kept across releases
  sl = SlotState();
  sl.priority = prio;
}

// The slot's stream: default priority, or the device's greatest.  A captured
// pass graph launched into it runs its kernels at the stream's priority.
xb_status slot_stream(SlotState& sl) {
  int least = 0, greatest = 0;
  XB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  XB_CUDA(cudaStreamCreateWithPriority(&sl.stream, cudaStreamNonBlocking, sl.priority ? greatest : 0));
  return XB_OK;
}

xb_status slot_init(SlotState& sl) {
  if (sl.init) return XB_OK;
  xb_status st = slot_stream(sl);
  if (st != XB_OK) return st;
  XB_CUDA(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
  XB_CUDA(cudaMalloc(&sl.d_src, sizeof(int32_t) * kSlotMaxRows));
  XB_CUDA(cudaMallocHost(&sl.h_src, sizeof(int32_t) * kSlotMaxRows));
  XB_CUDA(cudaMalloc(&sl.d_rows, sizeof(int32_t*) * 2 * kSlotMaxRows));
  XB_CUDA(cudaMallocHost(&sl.h_rows, sizeof(int32_t*) * 2 * kSlotMaxRows));
  XB_CUDA(cudaMalloc(&sl.d_flags, sizeof(int32_t) * kSlotMaxRows));
  XB_CUDA(cudaMallocHost(&sl.h_flags, sizeof(int32_t) * kSlotMaxRows));
  XB_CUDA(cudaMalloc(&sl.d_sum, sizeof(xbk::PassSum)));
  XB_CUDA(cudaMallocHost(&sl.h_sum, sizeof(xbk::PassSum)));
  XB_CUDA(cudaMalloc(&sl.d_dig, sizeof(xbk::RowDigest) * kSlotMaxRows));
  XB_CUDA(cudaMallocHost(&sl.h_dig, sizeof(xbk::RowDigest) * kSlotMaxRows));
  XB_CUDA(cudaMalloc(&sl.ctr, sizeof(xbk::Ctrs)));
  XB_CUDA(cudaMemset(sl.ctr, 0, sizeof(xbk::Ctrs)));
  sl.init = true;
  return XB_OK;
}

// Captures the one-pass graph of a slot: clear the totals, the pass, the
// digests of the flagged rows, and the copies of totals and digests to the
// slot's pinned mirrors.  all_digest: every row of the pass is digest-only,
// and the table pass sums the digests itself instead of writing rows for
// k_row_digest to read.
template <typename W, int NW, typename OffT>
xb_status capture_slot_pass(xb_ctx* c, BatchState* bs, SlotState& sl, const xb_graph* g, int kb, bool all_digest,
                            cudaGraphExec_t* exec) {
  constexpr int B = xbk::WB<W>::bits;
  cudaStream_t s = sl.stream;
  XB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
  auto body = [&]() -> xb_status {
    XB_CUDA(cudaMemsetAsync(sl.d_sum, 0, sizeof(xbk::PassSum), s));
    XB_CUDA(cudaMemsetAsync(sl.d_dig, 0, sizeof(xbk::RowDigest) * kSlotMaxRows, s));
    const PassRes<W, NW, OffT> p = capture_res<W, NW, OffT>(c, g, sl.ws, sl.ctr, sl.hpar);
    xb_status st = capture_pass_levels<W, NW, OffT>(c, bs, p, g, sl.d_src, kb, s);
    if (st != XB_OK) return st;
    st = capture_pass_tables<W, NW, OffT>(c, p, g, sl.d_src, kb, sl.d_rows, sl.d_sum, s,
                                          all_digest ? sl.d_dig : nullptr);
    if (st != XB_OK) return st;
    if (!all_digest) {
      const int gx = (int)std::max<int64_t>(1, std::min<int64_t>((g->n + 2047) / 2048, 64));
      xbk::k_row_digest<<<dim3((unsigned)gx, (unsigned)kb), 256, 0, s>>>(sl.d_rows, sl.d_flags, kb, B, g->n,
                                                                          sl.d_dig);
      XB_LAUNCH_CHECK("row digest");
    }
    XB_CUDA(cudaMemcpyAsync(sl.h_sum, sl.d_sum, sizeof(xbk::PassSum), cudaMemcpyDeviceToHost, s));
    XB_CUDA(cudaMemcpyAsync(sl.h_dig, sl.d_dig, sizeof(xbk::RowDigest) * kb, cudaMemcpyDeviceToHost, s));
    return XB_OK;
  };
  xb_status st = body();
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &graph);
  if (st == XB_OK && e != cudaSuccess) st = fail(XB_ERR_CUDA, std::string("slot capture: ") + cudaGetErrorString(e));
  if (st == XB_OK) {
    const cudaError_t ei = cudaGraphInstantiate(exec, graph, 0);
    if (ei != cudaSuccess) st = fail(XB_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
  }
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();
  return st;
}

template <typename W, int NW>
xb_status slot_launch(xb_ctx* c, int slot, xb_graph* g, const int32_t* sources, int kb,
                      int32_t* const* level_rows, int32_t* const* parent_rows) {
  constexpr int B = xbk::WB<W>::bits;
  constexpr int SPP = B * NW;
  if (kb < 1 || kb > SPP) return fail(XB_ERR_ARG, "a slot pass takes 1.." + std::to_string(SPP) + " sources");
  xb_status st = make_state(c);
  if (st != XB_OK) return st;
  BatchState* bs = c->batch;
  SlotState& sl = bs->slots[slot];
  if (sl.busy) return fail(XB_ERR_STATE, "slot " + std::to_string(slot) + " has a pass in flight");
  st = slot_init(sl);
  if (st != XB_OK) return st;
  const int heavy = std::max(32, c->tuning.heavy_degree);
  st = ensure_heavy(g, heavy);
  if (st != XB_OK) return st;
  // resources for this graph
  size_t cap = sl.ws_bytes;
  const size_t slot_ws = layout_for(g->n, (int)sizeof(W), NW).total;
  st = (cap < slot_ws || !sl.ws) ? check_workspace_cap(c, slot_ws, "slot workspace") : XB_OK;
  if (st == XB_OK) st = grow(&sl.ws, &cap, layout_for(g->n, (int)sizeof(W), NW).total, &sl.gen, "slot workspace");
  sl.ws_bytes = cap;
  if (st != XB_OK) return st;
  cap = sl.hpar_bytes;
  st = grow(&sl.hpar, &cap, sizeof(int32_t) * (size_t)std::max(g->n_heavy, 1) * kHparRow, &sl.gen, "slot heavy slots");
  sl.hpar_bytes = cap;
  if (st != XB_OK) return st;
  bool any_digest = false, all_digest = true;
  for (int j = 0; j < kb; j++) {
    if (!level_rows[j] != !parent_rows[j]) return fail(XB_ERR_ARG, "row " + std::to_string(j) + ": one of level/parent is NULL");
    any_digest |= level_rows[j] == nullptr;
    all_digest &= level_rows[j] == nullptr;
  }
  // scratch rows for the digest-only sources of a mixed pass; a pass of
  // digest-only sources sums its digests in the table pass and needs none
  if (any_digest && !all_digest) {  // SPP level rows then SPP parent rows, n_scratch entries apart
    cap = sl.scratch_bytes;
    st = grow(&sl.scratch, &cap, sizeof(int32_t) * 2 * SPP * (size_t)g->n, &sl.gen, "slot scratch rows");
    sl.scratch_bytes = cap;
    if (st != XB_OK) return st;
    sl.n_scratch = (int64_t)(sl.scratch_bytes / (sizeof(int32_t) * 2 * SPP));
  }
  // staging (the slot is idle: its previous pass has been collected)
  for (int j = 0; j < SPP; j++) {
    const int wi = j / B, b = j % B;
    int32_t* lv = nullptr;
    int32_t* pr = nullptr;
    int flag = 0;
    if (j < kb) {
      sl.h_src[j] = sources[j];
      lv = level_rows[j];
      pr = parent_rows[j];
      if (!lv) {
        if (!all_digest) {
          lv = sl.scratch + (size_t)j * sl.n_scratch;
          pr = sl.scratch + (size_t)(SPP + j) * sl.n_scratch;
        }
        flag = 1;
      }
    }
    sl.h_rows[wi * 2 * B + b] = lv;
    sl.h_rows[wi * 2 * B + B + b] = pr;
    sl.h_flags[j] = flag;
  }
  // cached one-pass graph
  uint32_t abits = 0, bbits = 0;
  std::memcpy(&abits, &c->tuning.pull_alpha, sizeof(abits));
  std::memcpy(&bbits, &c->tuning.push_beta, sizeof(bbits));
  const std::vector<uint64_t> key = {sl.gen, (uint64_t)(uintptr_t)g, g->version, (uint64_t)kb, sizeof(W), NW,
                                     (uint64_t)heavy, abits, (uint64_t)c->tuning.level_cap,
                                     (uint64_t)c->tuning.tile, (uint64_t)all_digest, bbits};
  CachedGraph* hit = nullptr;
  for (auto& e : sl.cache)
    if (e.key == key) hit = &e;
  if (!hit) {
    for (size_t i = 0; i < sl.cache.size();) {  // entries made before a reallocation
      if (sl.cache[i].key[0] != sl.gen) {
        cudaGraphExecDestroy(sl.cache[i].exec);
        sl.cache.erase(sl.cache.begin() + (ptrdiff_t)i);
      } else {
        i++;
      }
    }
    if (sl.cache.size() >= kSlotMaxCached) {
      auto lru = std::min_element(sl.cache.begin(), sl.cache.end(),
                                  [](const CachedGraph& a, const CachedGraph& b) { return a.last_use < b.last_use; });
      cudaGraphExecDestroy(lru->exec);
      sl.cache.erase(lru);
    }
    CachedGraph e;
    e.key = key;
    e.graphs = {g};
    st = g->off64 ? capture_slot_pass<W, NW, int64_t>(c, bs, sl, g, kb, all_digest, &e.exec)
                  : capture_slot_pass<W, NW, int32_t>(c, bs, sl, g, kb, all_digest, &e.exec);
    if (st != XB_OK) return st;
    sl.cache.push_back(std::move(e));
    hit = &sl.cache.back();
  }
  hit->last_use = ++sl.tick;
  XB_CUDA(cudaMemcpyAsync(sl.d_src, sl.h_src, sizeof(int32_t) * kb, cudaMemcpyHostToDevice, sl.stream));
  XB_CUDA(cudaMemcpyAsync(sl.d_rows, sl.h_rows, sizeof(int32_t*) * 2 * SPP, cudaMemcpyHostToDevice, sl.stream));
  XB_CUDA(cudaMemcpyAsync(sl.d_flags, sl.h_flags, sizeof(int32_t) * SPP, cudaMemcpyHostToDevice, sl.stream));
  XB_CUDA(cudaGraphLaunch(hit->exec, sl.stream));
  XB_CUDA(cudaEventRecord(sl.done, sl.stream));
  sl.busy = true;
  sl.kb = kb;
  return XB_OK;
}

// Collects a finished slot pass.
xb_status slot_collect(SlotState& sl, xb_stats* stats, xb_row_digest* digests) {
  sl.busy = false;
  const xbk::PassSum& s = *sl.h_sum;
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->edges_traversed = (int64_t)s.edges_traversed;
    stats->reached = (int64_t)s.reached;
    stats->edges_scanned = (int64_t)s.edges_scanned;
    stats->vertices_scanned = (int64_t)s.vertices_scanned;
    stats->vertices_swept = (int64_t)s.vertices_swept;
    stats->parent_edges_scanned = (int64_t)s.parent_edges;
    stats->class_bytes[0] = (int64_t)s.level_bytes;
    stats->class_bytes[1] = (int64_t)s.table_bytes;
    stats->algo_bytes = (int64_t)(s.level_bytes + s.table_bytes);
    stats->levels = s.max_level;
    stats->push_levels = s.push_levels;
    stats->pull_levels = s.pull_levels;
    stats->batches = s.passes;
    stats->class_launches[2] = (int64_t)s.launches;
  }
  if (digests)
    for (int j = 0; j < sl.kb; j++) {
      const xbk::RowDigest& d = sl.h_dig[j];
      digests[j].reached = (int64_t)d.reached;
      digests[j].level_sum = (int64_t)d.level_sum;
      digests[j].row_hash = (int64_t)d.row_hash;
      digests[j].depth = sl.h_flags[j] ? (int32_t)d.depth : -1;
      digests[j].pad = 0;
    }
  if (s.errors) return fail(XB_ERR_STATE, "the pass's level loop ran past the level bound (corrupted state)");
  return XB_OK;
}

}  // namespace

void batch_state_free(BatchState* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  for (auto& sl : b->slots) slot_free(sl);
  drop_cache(b);
  for (auto& ch : b->chains) {
    if (ch.ws) cudaFree(ch.ws);
    if (ch.ctr) cudaFree(ch.ctr);
    if (ch.hpar) cudaFree(ch.hpar);
    if (ch.stage) cudaFree(ch.stage);
    for (cudaEvent_t e : {ch.ev_tab, ch.ev_free[0], ch.ev_free[1], ch.ev_join, ch.ev_join_cp})
      if (e) cudaEventDestroy(e);
    if (ch.cs) cudaStreamDestroy(ch.cs);
    if (ch.cps) cudaStreamDestroy(ch.cps);
  }
  if (b->d_sums) cudaFree(b->d_sums);
  if (b->h_sums) cudaFreeHost(b->h_sums);
  if (b->d_src) cudaFree(b->d_src);
  if (b->h_src) cudaFreeHost(b->h_src);
  if (b->d_rows) cudaFree(b->d_rows);
  if (b->h_rows) cudaFreeHost(b->h_rows);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  for (auto s : b->body)
    if (s) cudaStreamDestroy(s);
  if (b->origin) cudaStreamDestroy(b->origin);
  delete b;
}

void batch_forget_graph(xb_ctx* c, const xb_graph* g) {
  if (!c || !c->batch) return;
  for (auto& sl : c->batch->slots)
    for (size_t i = 0; i < sl.cache.size();) {
      if (sl.cache[i].graphs.size() == 1 && sl.cache[i].graphs[0] == g) {
        if (sl.busy && sl.stream) cudaStreamSynchronize(sl.stream);
        cudaGraphExecDestroy(sl.cache[i].exec);
        sl.cache.erase(sl.cache.begin() + (ptrdiff_t)i);
      } else {
        i++;
      }
    }
  auto& cache = c->batch->cache;
  for (size_t i = 0; i < cache.size();) {
    bool uses = false;
    for (const xb_graph* x : cache[i].graphs) uses |= x == g;
    if (uses) {
      if (cache[i].exec) cudaGraphExecDestroy(cache[i].exec);
      cache.erase(cache.begin() + (ptrdiff_t)i);
    } else {
      i++;
    }
  }
}

}  // namespace xbe

extern "C" xb_status xb_traverse_batched(xb_ctx* c, const xb_batch_item* items, int32_t nitems, xb_stats* stats) {
  xbi::clear_error();
  if (!c) return fail(XB_ERR_ARG, "null context");
  if (nitems < 0 || (nitems > 0 && !items)) return fail(XB_ERR_ARG, "bad item list");
  if (stats) std::memset(stats, 0, sizeof(*stats));
  XB_CUDA(cudaSetDevice(c->device));
  std::vector<xb_batch_item> its(items, items + nitems);
  std::vector<std::vector<int32_t>> hsrc((size_t)nitems);
  for (int32_t i = 0; i < nitems; i++) {
    const xb_batch_item& it = its[(size_t)i];
    const std::string at = "item " + std::to_string(i) + ": ";
    if (!it.graph) return fail(XB_ERR_ARG, at + "null graph");
    if (!it.graph->ctx) return fail(XB_ERR_STATE, at + "the graph's context was destroyed");
    if (it.graph->ctx->device != c->device) return fail(XB_ERR_ARG, at + "graph lives on another device");
    if (it.k < 0) return fail(XB_ERR_ARG, at + "negative source count");
    if (it.flags & XB_PARENT_FIFO) return fail(XB_ERR_ARG, at + "FIFO parents are computed by xb_traverse only");
    if (it.k == 0) continue;
    if (!it.sources || !it.level || !it.parent) return fail(XB_ERR_ARG, at + "null sources or output tables");
    if (!(it.flags & XB_OUT_DEVICE)) {
      for (const int32_t* ptr : {it.level, it.parent}) {
        cudaPointerAttributes a{};
        if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess || a.type != cudaMemoryTypeHost) {
          cudaGetLastError();
          return fail(XB_ERR_ARG, at + "host tables must be page-locked (cudaHostAlloc / cudaHostRegister)");
        }
      }
    }
    auto& h = hsrc[(size_t)i];
    h.resize((size_t)it.k);
    if (it.flags & XB_SOURCES_DEVICE) {
      XB_CUDA(cudaMemcpy(h.data(), it.sources, sizeof(int32_t) * (size_t)it.k, cudaMemcpyDeviceToHost));
    } else {
      std::memcpy(h.data(), it.sources, sizeof(int32_t) * (size_t)it.k);
    }
    for (int32_t s = 0; s < it.k; s++)
      if (h[(size_t)s] < 0 || h[(size_t)s] >= it.graph->n)
        return fail(XB_ERR_ARG, at + "source " + std::to_string(s) + " out of range");
  }
  xb_status s = XB_OK;
  const int nw = c->tuning.words;
  if (c->tuning.word_bits == 64) {
    s = nw == 1 ? xbe::run_batched<unsigned long long, 1>(c, its, hsrc, stats)
        : nw == 2 ? xbe::run_batched<unsigned long long, 2>(c, its, hsrc, stats)
                  : xbe::run_batched<unsigned long long, 4>(c, its, hsrc, stats);
  } else {
    s = nw == 1 ? xbe::run_batched<unsigned int, 1>(c, its, hsrc, stats)
        : nw == 2 ? xbe::run_batched<unsigned int, 2>(c, its, hsrc, stats)
                  : xbe::run_batched<unsigned int, 4>(c, its, hsrc, stats);
  }
  if (s != XB_OK) {
    cudaStreamSynchronize(c->stream);
    cudaGetLastError();
  }
  return s;
}

extern "C" xb_status xb_slot_launch(xb_ctx* c, int32_t slot, const xb_graph* gc, const int32_t* sources, int32_t kb,
                                    int32_t* const* level_rows, int32_t* const* parent_rows) {
  xbi::clear_error();
  xb_graph* g = const_cast<xb_graph*>(gc);
  if (!c || !g || !sources || !level_rows || !parent_rows) return fail(XB_ERR_ARG, "null argument");
  if (slot < 0 || slot >= xbe::kMaxSlots) return fail(XB_ERR_ARG, "slot out of range");
  if (!g->ctx) return fail(XB_ERR_STATE, "the graph's context was destroyed");
  if (g->ctx->device != c->device) return fail(XB_ERR_ARG, "graph lives on another device");
  for (int32_t j = 0; j < kb; j++)
    if (sources[j] < 0 || sources[j] >= g->n) return fail(XB_ERR_ARG, "source " + std::to_string(j) + " out of range");
  XB_CUDA(cudaSetDevice(c->device));
  const int nw = c->tuning.words;
  xb_status s;
  if (c->tuning.word_bits == 64) {
    s = nw == 1 ? xbe::slot_launch<unsigned long long, 1>(c, slot, g, sources, kb, level_rows, parent_rows)
        : nw == 2 ? xbe::slot_launch<unsigned long long, 2>(c, slot, g, sources, kb, level_rows, parent_rows)
                  : xbe::slot_launch<unsigned long long, 4>(c, slot, g, sources, kb, level_rows, parent_rows);
  } else {
    s = nw == 1 ? xbe::slot_launch<unsigned int, 1>(c, slot, g, sources, kb, level_rows, parent_rows)
        : nw == 2 ? xbe::slot_launch<unsigned int, 2>(c, slot, g, sources, kb, level_rows, parent_rows)
                  : xbe::slot_launch<unsigned int, 4>(c, slot, g, sources, kb, level_rows, parent_rows);
  }
  return s;
}

extern "C" xb_status xb_slot_poll(xb_ctx* c, int32_t slot, int32_t* done, xb_stats* stats, xb_row_digest* digests) {
  xbi::clear_error();
  if (!c || !done) return fail(XB_ERR_ARG, "null argument");
  if (slot < 0 || slot >= xbe::kMaxSlots) return fail(XB_ERR_ARG, "slot out of range");
  if (!c->batch || !c->batch->slots[slot].busy) return fail(XB_ERR_STATE, "no pass in flight on this slot");
  xbe::SlotState& sl = c->batch->slots[slot];
  const cudaError_t q = cudaEventQuery(sl.done);
  if (q == cudaErrorNotReady) {
    *done = 0;
    return XB_OK;
  }
  if (q != cudaSuccess) {
    sl.busy = false;
    return fail(XB_ERR_CUDA, std::string("slot pass: ") + cudaGetErrorString(q));
  }
  *done = 1;
  return xbe::slot_collect(sl, stats, digests);
}

extern "C" xb_status xb_slot_wait(xb_ctx* c, int32_t slot, xb_stats* stats, xb_row_digest* digests) {
  xbi::clear_error();
  if (!c) return fail(XB_ERR_ARG, "null context");
  if (slot < 0 || slot >= xbe::kMaxSlots) return fail(XB_ERR_ARG, "slot out of range");
  if (!c->batch || !c->batch->slots[slot].busy) return fail(XB_ERR_STATE, "no pass in flight on this slot");
  xbe::SlotState& sl = c->batch->slots[slot];
  const cudaError_t e = cudaEventSynchronize(sl.done);
  if (e != cudaSuccess) {
    sl.busy = false;
    return fail(XB_ERR_CUDA, std::string("slot pass: ") + cudaGetErrorString(e));
  }
  return xbe::slot_collect(sl, stats, digests);
}

extern "C" xb_status xb_slot_set_priority(xb_ctx* c, int32_t slot, int32_t priority) {
  xbi::clear_error();
  if (!c) return fail(XB_ERR_ARG, "null context");
  if (slot < 0 || slot >= xbe::kMaxSlots) return fail(XB_ERR_ARG, "slot out of range");
  if (priority != 0 && priority != 1) return fail(XB_ERR_ARG, "priority must be 0 or 1");
  XB_CUDA(cudaSetDevice(c->device));
  xb_status st = xbe::make_state(c);
  if (st != XB_OK) return st;
  xbe::SlotState& sl = c->batch->slots[slot];
  if (sl.busy) return fail(XB_ERR_STATE, "slot " + std::to_string(slot) + " has a pass in flight");
  if (sl.priority == priority) return XB_OK;
  sl.priority = priority;
  if (sl.stream) {  // an initialised slot gets a new stream; its captured passes stay valid
    XB_CUDA(cudaStreamSynchronize(sl.stream));
    XB_CUDA(cudaStreamDestroy(sl.stream));
    sl.stream = nullptr;
    return xbe::slot_stream(sl);
  }
  return XB_OK;
}

extern "C" xb_status xb_slots_release(xb_ctx* c) {
  xbi::clear_error();
  if (!c) return fail(XB_ERR_ARG, "null context");
  if (!c->batch) return XB_OK;
  for (auto& sl : c->batch->slots)
    if (sl.busy) return fail(XB_ERR_STATE, "a slot has a pass in flight");
  cudaSetDevice(c->device);
  for (auto& sl : c->batch->slots) xbe::slot_free(sl);
  return XB_OK;
}

extern "C" xb_status xb_host_alloc(int64_t bytes, void** out) {
  xbi::clear_error();
  if (!out || bytes < 0) return fail(XB_ERR_ARG, "bad argument");
  *out = nullptr;
  if (cudaMallocHost(out, (size_t)std::max<int64_t>(bytes, 1)) != cudaSuccess) {
    cudaGetLastError();
    *out = nullptr;
    return fail(XB_ERR_OOM, "page-locked allocation of " + std::to_string(bytes) + " bytes failed");
  }
  return XB_OK;
}

extern "C" xb_status xb_host_free(void* p) {
  xbi::clear_error();
  if (p && cudaFreeHost(p) != cudaSuccess) {
    cudaGetLastError();
    return fail(XB_ERR_ARG, "not a page-locked allocation of this library");
  }
  return XB_OK;
}
