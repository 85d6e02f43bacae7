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
#include <cstdlib>
#include <memory>
#include <new>

#include "xb_engine_common.cuh"

using xbi::fail;

namespace xbe {

// Row offsets are stored as int32 unless the graph has 2^31 - 1 or more
// entries; XB_OFFSETS64=1 in the environment keeps int64 offsets for every
// graph uploaded while it is set (the int64 kernels' parity tests).
bool wide_offsets(int64_t m) {
  if (m >= (int64_t)INT32_MAX) return true;
  const char* e = std::getenv("XB_OFFSETS64");
  return e && e[0] == '1';
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
    }
    return XB_OK;
  }
  xb_status cs = check_workspace_cap(c, L.total, "traversal workspace");
  if (cs != XB_OK) return cs;
  std::memcpy(c->ws_key, key, sizeof(key));
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

// The context workspace as plain scratch of at least `bytes` for the paths
// other than the plain traversal (SSSP, matching, alternating mode); they
// leave the traversal's zero invariants broken, so its next call clears the
// workspace again.
xb_status ensure_scratch(xb_ctx* c, size_t bytes, const char* what) {
  if (c->ws_bytes < bytes || !c->ws) {
    const xb_status cs = check_workspace_cap(c, bytes, what);
    if (cs != XB_OK) return cs;
    if (c->ws) cudaFree(c->ws);
    c->ws = nullptr;
    c->ws_bytes = 0;
    if (cudaMalloc(&c->ws, bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(XB_ERR_OOM, std::string(what) + " work allocation of " + std::to_string(bytes) + " bytes failed");
    }
    c->ws_bytes = bytes;
  }
  c->ws_key[0] = -1;
  return XB_OK;
}

xb_status ensure_stage(xb_ctx* c, size_t bytes) {
  if (c->stage_bytes >= bytes) return XB_OK;
  const xb_status cs = check_workspace_cap(c, bytes, "table staging");
  if (cs != XB_OK) return cs;
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

xb_status ensure_rows(xb_ctx* c, int64_t count) {
  if (c->rows_cap >= count) return XB_OK;
  if (c->d_rows) cudaFree(c->d_rows);
  c->d_rows = nullptr;
  c->rows_cap = 0;
  if (cudaMalloc(&c->d_rows, sizeof(int32_t*) * (size_t)std::max<int64_t>(count, 1)) != cudaSuccess) {
    cudaGetLastError();
    return fail(XB_ERR_OOM, "row table allocation failed");
  }
  c->rows_cap = count;
  return XB_OK;
}

// Work areas of the FIFO-parent pass (two queues and counts per source row).
xb_status ensure_fifo(xb_ctx* c, size_t ints) {
  if (c->fifo_cap >= ints) return XB_OK;
  if (c->d_fifo) cudaFree(c->d_fifo);
  c->d_fifo = nullptr;
  c->fifo_cap = 0;
  if (cudaMalloc(&c->d_fifo, sizeof(int32_t) * std::max<size_t>(ints, 1)) != cudaSuccess) {
    cudaGetLastError();
    return fail(XB_ERR_OOM, "FIFO-parent work allocation failed");
  }
  c->fifo_cap = ints;
  return XB_OK;
}

xb_status ensure_reach2(xb_graph* g) {
  if ((int64_t)g->h_reach2.size() == g->n) return XB_OK;
  if (!g->ctx) return fail(XB_ERR_STATE, "the graph's context was destroyed");
  xb_ctx* c = g->ctx;
  XB_CUDA(cudaSetDevice(c->device));
  long long* d = nullptr;
  if (cudaMalloc(&d, sizeof(long long) * (size_t)g->n) != cudaSuccess) {
    cudaGetLastError();
    return fail(XB_ERR_OOM, "neighbour degree sum allocation failed");
  }
  std::vector<int64_t> h((size_t)g->n);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((g->n + 7) / 8, (int64_t)c->num_sms * 8));
  if (g->off64)
    xbk::k_reach2<int64_t><<<grid, 256, 0, c->stream>>>(g->n, (const int64_t*)g->d_ro, g->d_ci, d);
  else
    xbk::k_reach2<int32_t><<<grid, 256, 0, c->stream>>>(g->n, (const int32_t*)g->d_ro, g->d_ci, d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d, sizeof(long long) * (size_t)g->n, cudaMemcpyDeviceToHost,
                                            c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d);
  if (e != cudaSuccess) return fail(XB_ERR_CUDA, std::string("neighbour degree sums: ") + cudaGetErrorString(e));
  g->h_reach2.swap(h);
  return XB_OK;
}

xb_status ensure_heavy(xb_graph* g, int thr) {
  if (g->heavy_thr == thr) return XB_OK;
  // heavy vertices by falling degree (ties by ascending id): every heavy
  // index (hpar rows, work items, hidx_of) follows this order, and the pull
  // kernels hand the vertices out longest first
  std::vector<int32_t> hv;
  for (int64_t v = 0; v < g->n; v++)
    if (g->h_ro[v + 1] - g->h_ro[v] > thr) hv.push_back((int32_t)v);
  std::stable_sort(hv.begin(), hv.end(), [&](int32_t a, int32_t b) {
    return g->h_ro[a + 1] - g->h_ro[a] > g->h_ro[b + 1] - g->h_ro[b];
  });
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
  {  // light vertices by falling degree (counting sort; ties by ascending id)
    std::vector<int64_t> cnt((size_t)thr + 2, 0);
    for (int64_t v = 0; v < g->n; v++) {
      const int64_t d = g->h_ro[v + 1] - g->h_ro[v];
      if (d >= 1 && d <= thr) cnt[(size_t)(thr - d)]++;
    }
    int64_t acc = 0;
    for (auto& x : cnt) {
      const int64_t c = x;
      x = acc;
      acc += c;
    }
    std::vector<int32_t> lorder((size_t)acc);
    for (int64_t v = 0; v < g->n; v++) {
      const int64_t d = g->h_ro[v + 1] - g->h_ro[v];
      if (d >= 1 && d <= thr) lorder[(size_t)cnt[(size_t)(thr - d)]++] = (int32_t)v;
    }
    if (g->d_lorder) cudaFree(g->d_lorder);
    g->d_lorder = nullptr;
    if (cudaMalloc(&g->d_lorder, sizeof(int32_t) * std::max<size_t>(lorder.size(), 1)) != cudaSuccess) {
      cudaGetLastError();
      return fail(XB_ERR_OOM, "light vertex list allocation failed");
    }
    if (!lorder.empty())
      XB_CUDA(cudaMemcpy(g->d_lorder, lorder.data(), sizeof(int32_t) * lorder.size(), cudaMemcpyHostToDevice));
    g->n_lorder = (int64_t)lorder.size();
    // chunks of the list: at most kLaneChunk vertices, and a new chunk once
    // kLaneChunkEdges edges are reached
    std::vector<int32_t> lchunk{0};
    int64_t edges = 0;
    for (size_t i = 0; i < lorder.size(); i++) {
      const int64_t d = g->h_ro[lorder[i] + 1] - g->h_ro[lorder[i]];
      if (i > (size_t)lchunk.back() &&
          ((int64_t)i - lchunk.back() >= xbk::kLaneChunk || edges + d > xbk::kLaneChunkEdges)) {
        lchunk.push_back((int32_t)i);
        edges = 0;
      }
      edges += d;
    }
    lchunk.push_back((int32_t)lorder.size());
    if (g->d_lchunk) cudaFree(g->d_lchunk);
    g->d_lchunk = nullptr;
    if (cudaMalloc(&g->d_lchunk, sizeof(int32_t) * lchunk.size()) != cudaSuccess) {
      cudaGetLastError();
      return fail(XB_ERR_OOM, "light chunk table allocation failed");
    }
    XB_CUDA(cudaMemcpy(g->d_lchunk, lchunk.data(), sizeof(int32_t) * lchunk.size(), cudaMemcpyHostToDevice));
    g->n_lchunks = lorder.empty() ? 0 : (int32_t)lchunk.size() - 1;
  }
  // (heavy index, chunk) work items of the table pass, heaviest vertices first
  // (the list order)
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
  g->version++;
  return XB_OK;
}

template <typename W, int NW, typename OffT>
xb_status run_plain(xb_ctx* c, xb_graph* g, const int32_t* d_sources, const int64_t* perm, int32_t k,
                    int32_t* level_out, int32_t* parent_out, bool out_dev, bool fifo, xb_stats* st) {
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
  // row-pointer tables of every pass of the call, uploaded once
  const int64_t npass = (k + SPP - 1) / SPP;
  s = ensure_rows(c, npass * 2 * SPP);
  if (s != XB_OK) return s;
  {
    std::vector<int32_t*> rows((size_t)(npass * 2 * SPP));
    for (int64_t j = 0; j < npass; j++) {
      const int kb = (int)std::min<int64_t>(SPP, k - j * SPP);
      int32_t** pr = rows.data() + j * 2 * SPP;
      if (!out_dev) {
        fill_rows<W, NW>(pr, kb, c->d_stage, c->d_stage + (size_t)SPP * n, n);
        continue;
      }
      fill_rows<W, NW>(pr, kb, level_out, parent_out, 0);  // nullptr past kb
      for (int i = 0; i < kb; i++) {  // each source's row where the caller put it
        const int64_t r = perm[j * SPP + i];
        pr[(i / B) * 2 * B + i % B] = level_out + r * n;
        pr[(i / B) * 2 * B + B + i % B] = parent_out + r * n;
      }
    }
    XB_CUDA(cudaMemcpyAsync(c->d_rows, rows.data(), sizeof(int32_t*) * rows.size(), cudaMemcpyHostToDevice,
                            c->stream));
    XB_CUDA(cudaStreamSynchronize(c->stream));
  }
  PassRes<W, NW, OffT> p = pass_res<W, NW, OffT>(g, c->ws, L, c->d_ctr, g->d_hpar, heavy);
  p.tile = c->tuning.tile;
  const int sms = c->num_sms;
  const float alpha = c->tuning.pull_alpha > 0 ? c->tuning.pull_alpha : 256.0f;
  ClassTimer timer{c, st, c->tuning.timing != 0};
  const StepShape mx = max_shape<W, NW, OffT>(g, sms, p.tile);
  const int bound = level_bound(c, p.nplanes_alloc);
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
      xbk::k_step_begin<<<1, 1, 0, c->stream>>>(p.ctr, cur, alpha, p.nplanes_alloc, bound, 0, 0,
                                                push_below(c, g));
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
    if (c->h_ctr->b.err) {
      // the pass stopped with a live frontier: F / N are not all zero, so the
      // next call clears the workspace before it relies on that
      c->ws_key[0] = -1;
      return fail(XB_ERR_STATE, "the level loop ran past the level bound (corrupted traversal state)");
    }
    max_levels = std::max(max_levels, c->h_ctr->b.level);
    timer.begin();
    int64_t launches = 0;
    int32_t* lv_base = c->d_stage;
    int32_t* pr_base = c->d_stage + (size_t)SPP * n;
    s = emit_tables<W, NW, OffT>(p, g, d_sources + k0, kb, c->d_rows + (k0 / SPP) * 2 * SPP,
                                 c->h_ctr->b.pushed_deep != 0, c->stream, sms, &launches);
    if (s != XB_OK) return s;
    if (fifo) {  // parents by the FIFO rule, rewritten from the finished level rows
      const int group = std::min(kb, kFifoGroup);
      s = ensure_fifo(c, (size_t)group * 3 * (size_t)n);
      if (s != XB_OK) return s;
      for (int j0 = 0; j0 < kb; j0 += group) {
        xbk::k_fifo_parents<OffT><<<std::min(group, kb - j0), 1024, 0, c->stream>>>(
            n, p.ro, p.ci, c->d_rows + (k0 / SPP) * 2 * SPP, B, j0, kb, d_sources + k0, c->d_fifo, 3 * n);
        launches++;
      }
      XB_LAUNCH_CHECK("fifo parents");
    }
    timer.end(1, launches);
    if (!out_dev) {  // runs of consecutive caller rows become one copy each
      for (int j = 0; j < kb;) {
        const int64_t r0 = perm[k0 + j];
        int e = j + 1;
        while (e < kb && perm[k0 + e] == r0 + (e - j)) e++;
        const size_t bytes = sizeof(int32_t) * (size_t)(e - j) * (size_t)n;
        XB_CUDA(cudaMemcpyAsync(level_out + r0 * n, lv_base + (size_t)j * n, bytes, cudaMemcpyDeviceToHost,
                                c->stream));
        XB_CUDA(cudaMemcpyAsync(parent_out + r0 * n, pr_base + (size_t)j * n, bytes, cudaMemcpyDeviceToHost,
                                c->stream));
        j = e;
      }
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
xb_status dispatch_nw(xb_ctx* c, xb_graph* g, const int32_t* d_src, const int64_t* perm, int32_t k, int32_t* lv,
                      int32_t* pr, bool od, bool fifo, xb_stats* st) {
  switch (c->tuning.words) {
    case 1: return run_plain<W, 1, OffT>(c, g, d_src, perm, k, lv, pr, od, fifo, st);
    case 2: return run_plain<W, 2, OffT>(c, g, d_src, perm, k, lv, pr, od, fifo, st);
    case 4: return run_plain<W, 4, OffT>(c, g, d_src, perm, k, lv, pr, od, fifo, st);
    default: return fail(XB_ERR_ARG, "tuning.words must be 1, 2 or 4");
  }
}

}  // namespace xbe

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
  c->tuning.words = 4;  // 256 sources per pass: one gather of a whole 32-byte sector serves them all
  // pull unless the frontier's edges are under 1/256 of the unfinished edges:
  // pull steps record parents as they go, push steps leave them to a search;
  // a small source set's first level is still pushed (a pull there scans the
  // whole graph for a few frontier vertices)
  c->tuning.pull_alpha = 256.0f;
  c->tuning.heavy_degree = 256;
  c->tuning.timing = 0;
  c->tuning.chains = 4;
  *out = c.release();
  return XB_OK;
}

xb_status xb_ctx_destroy(xb_ctx* c) {
  xbi::clear_error();
  if (!c) return XB_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (xb_graph* g : c->graphs) g->ctx = nullptr;  // graphs outliving the context can still be freed
  xbe::batch_state_free(c->batch);
  if (c->ws) cudaFree(c->ws);
  if (c->d_src) cudaFree(c->d_src);
  if (c->d_stage) cudaFree(c->d_stage);
  if (c->d_rows) cudaFree(c->d_rows);
  if (c->d_fifo) cudaFree(c->d_fifo);
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
  if (t->chains < 0 || t->chains > 16) return fail(XB_ERR_ARG, "chains must be in [0, 16]");
  if (t->level_cap < 0 || t->workspace_cap < 0) return fail(XB_ERR_ARG, "level_cap and workspace_cap must be >= 0");
  if (t->tile != 0 && t->tile != 1) return fail(XB_ERR_ARG, "tile must be 0 or 1");
  if (!(t->push_beta >= 0)) return fail(XB_ERR_ARG, "push_beta must be >= 0");
  if (t->source_order != 0 && t->source_order != 1) return fail(XB_ERR_ARG, "source_order must be 0 or 1");
  c->tuning = *t;
  if (c->tuning.chains == 0) c->tuning.chains = 4;
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
  *bytes = (int64_t)(c->ws_bytes + c->stage_bytes + sizeof(int32_t) * c->src_cap + sizeof(int32_t*) * c->rows_cap);
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
  g->off64 = xbe::wide_offsets(m);
  for (int64_t v = 0; v < n; v++) g->max_deg = std::max(g->max_deg, ro[v + 1] - ro[v]);
  const size_t ro_bytes = (g->off64 ? 8 : 4) * (size_t)(n + 1);
  // colIndices carries kCiPad zero entries past the end: the 16-byte loads of
  // the per-lane pull read whole aligned groups of 4 entries
  g->store = std::make_shared<xb_csr_store>();
  g->store->device = c->device;
  if (cudaMalloc(&g->store->ro, ro_bytes) != cudaSuccess ||
      cudaMalloc(&g->store->ci, sizeof(int32_t) * (size_t)(m + xbe::kCiPad)) != cudaSuccess) {
    cudaGetLastError();
    return fail(XB_ERR_OOM, "graph allocation failed");
  }
  g->d_ro = g->store->ro;
  g->d_ci = g->store->ci;
  if (g->off64) {
    XB_CUDA(cudaMemcpy(g->d_ro, ro.data(), ro_bytes, cudaMemcpyHostToDevice));
  } else {
    std::vector<int32_t> r32((size_t)n + 1);
    for (int64_t i = 0; i <= n; i++) r32[i] = (int32_t)ro[i];
    XB_CUDA(cudaMemcpy(g->d_ro, r32.data(), ro_bytes, cudaMemcpyHostToDevice));
  }
  XB_CUDA(cudaMemset(g->d_ci + m, 0, sizeof(int32_t) * xbe::kCiPad));
  if (m > 0) XB_CUDA(cudaMemcpy(g->d_ci, col_indices, sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice));
  g->h_ro = std::move(ro);
  c->graphs.push_back(g.get());
  *out = g.release();
  return XB_OK;
}

xb_status xb_graph_upload_batch(xb_ctx* c, int32_t ninst, const int64_t* inst_n, const int64_t* row_offsets,
                                const int32_t* col_indices, xb_graph** out) {
  xbi::clear_error();
  if (!c || !out || !inst_n || ninst < 1) return fail(XB_ERR_ARG, "bad arguments");
  if (!row_offsets) return fail(XB_ERR_ARG, "null row offsets");
  for (int32_t i = 0; i < ninst; i++) out[i] = nullptr;
  // host-side offsets of every instance; validation per instance
  std::vector<int64_t> vtx_off((size_t)ninst + 1, 0), edge_src((size_t)ninst + 1, 0), edge_dev((size_t)ninst + 1, 0);
  bool off64 = false;
  for (int32_t i = 0; i < ninst; i++) {
    const int64_t n = inst_n[i];
    if (n < 1 || n >= INT32_MAX) return fail(XB_ERR_ARG, "instance " + std::to_string(i) + ": n out of range");
    const int64_t* ro = row_offsets + vtx_off[(size_t)i];
    const int64_t m = ro[n];
    xb_status s = xbi::validate_csr(n, ro, col_indices ? col_indices + edge_src[(size_t)i] : nullptr);
    if (s != XB_OK) return fail(s, "instance " + std::to_string(i) + ": " + xb_last_error());
    off64 = off64 || xbe::wide_offsets(m);
    vtx_off[(size_t)i + 1] = vtx_off[(size_t)i] + n + 1;
    edge_src[(size_t)i + 1] = edge_src[(size_t)i] + m;
    edge_dev[(size_t)i + 1] = edge_dev[(size_t)i] + ((m + 3) & ~(int64_t)3);  // instances start 16-byte aligned
  }
  XB_CUDA(cudaSetDevice(c->device));
  auto store = std::make_shared<xb_csr_store>();
  store->device = c->device;
  const size_t nro = (size_t)vtx_off[(size_t)ninst];
  const size_t ro_bytes = (off64 ? 8 : 4) * nro;
  const size_t nci = (size_t)edge_dev[(size_t)ninst] + (size_t)xbe::kCiPad;
  if (cudaMalloc(&store->ro, ro_bytes) != cudaSuccess || cudaMalloc(&store->ci, sizeof(int32_t) * nci) != cudaSuccess) {
    cudaGetLastError();
    return fail(XB_ERR_OOM, "batch graph allocation failed");
  }
  if (off64) {
    XB_CUDA(cudaMemcpy(store->ro, row_offsets, ro_bytes, cudaMemcpyHostToDevice));
  } else {
    std::vector<int32_t> r32(nro);
    for (size_t i = 0; i < nro; i++) r32[i] = (int32_t)row_offsets[i];
    XB_CUDA(cudaMemcpy(store->ro, r32.data(), ro_bytes, cudaMemcpyHostToDevice));
  }
  XB_CUDA(cudaMemset(store->ci, 0, sizeof(int32_t) * nci));
  std::vector<std::unique_ptr<xb_graph>> gs;
  for (int32_t i = 0; i < ninst; i++) {
    const int64_t n = inst_n[i];
    const int64_t* ro = row_offsets + vtx_off[(size_t)i];
    const int64_t m = ro[n];
    if (m > 0)
      XB_CUDA(cudaMemcpy(store->ci + edge_dev[(size_t)i], col_indices + edge_src[(size_t)i], sizeof(int32_t) * (size_t)m,
                         cudaMemcpyHostToDevice));
    std::unique_ptr<xb_graph> g(new xb_graph());
    g->ctx = c;
    g->n = n;
    g->m = m;
    g->off64 = off64;
    g->store = store;
    g->d_ro = (char*)store->ro + (off64 ? 8 : 4) * (size_t)vtx_off[(size_t)i];
    g->d_ci = store->ci + edge_dev[(size_t)i];
    g->h_ro.assign(ro, ro + n + 1);
    for (int64_t v = 0; v < n; v++) g->max_deg = std::max(g->max_deg, ro[v + 1] - ro[v]);
    gs.push_back(std::move(g));
  }
  for (int32_t i = 0; i < ninst; i++) {
    c->graphs.push_back(gs[(size_t)i].get());
    out[i] = gs[(size_t)i].release();
  }
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
  if (g->ctx) {
    xb_ctx* c = g->ctx;
    cudaSetDevice(c->device);
    xbe::batch_forget_graph(c, g);
    c->graphs.erase(std::remove(c->graphs.begin(), c->graphs.end(), g), c->graphs.end());
  } else if (g->store) {
    cudaSetDevice(g->store->device);
  }
  g->store.reset();  // frees the CSR arrays with the last graph viewing them
  if (g->d_heavy) cudaFree(g->d_heavy);
  if (g->d_hpar) cudaFree(g->d_hpar);
  if (g->d_hitems) cudaFree(g->d_hitems);
  if (g->d_hub_items) cudaFree(g->d_hub_items);
  if (g->d_hidx_of) cudaFree(g->d_hidx_of);
  if (g->d_lorder) cudaFree(g->d_lorder);
  if (g->d_lchunk) cudaFree(g->d_lchunk);
  if (g->d_w) cudaFree(g->d_w);
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

xb_status xb_graph_offset_bytes(const xb_graph* g, int32_t* bytes) {
  xbi::clear_error();
  if (!g || !bytes) return fail(XB_ERR_ARG, "null argument");
  *bytes = g->off64 ? 8 : 4;
  return XB_OK;
}

xb_status xb_select_sources(const xb_graph* g, uint64_t seed, int32_t k, int32_t* out) {
  xbi::clear_error();
  if (!g) return fail(XB_ERR_ARG, "null graph");
  return xbi::select_sources(g->n, g->h_ro.data(), seed, k, out);
}

xb_status xb_graph_source_order(const xb_graph* gc, const int32_t* sources, int32_t k, int32_t* order) {
  xbi::clear_error();
  xb_graph* g = const_cast<xb_graph*>(gc);  // the neighbour degree sums are cached on first use
  if (!g) return fail(XB_ERR_ARG, "null graph");
  if (k < 0) return fail(XB_ERR_ARG, "negative source count");
  if (k > 0 && (!sources || !order)) return fail(XB_ERR_ARG, "null sources or order");
  for (int32_t i = 0; i < k; i++)
    if (sources[i] < 0 || sources[i] >= g->n) return fail(XB_ERR_ARG, "source " + std::to_string(i) + " out of range");
  std::vector<int64_t> perm((size_t)k);
  for (int32_t i = 0; i < k; i++) perm[i] = i;
  if (k > 0) {
    const xb_status s = xbe::order_by_degree(g, perm, [&](int64_t i) { return (int64_t)sources[i]; });
    if (s != XB_OK) return s;
  }
  for (int32_t i = 0; i < k; i++) order[i] = (int32_t)perm[i];
  return XB_OK;
}

xb_status xb_traverse(xb_ctx* c, const xb_graph* gc, const int32_t* sources, int32_t k, int32_t mode,
                      const int32_t* matching, int32_t* level, int32_t* parent, int32_t* owner, uint32_t flags,
                      xb_stats* st) {
  xbi::clear_error();
  xb_graph* g = const_cast<xb_graph*>(gc);
  if (!c || !g) return fail(XB_ERR_ARG, "null context or graph");
  if (!g->ctx) return fail(XB_ERR_STATE, "the graph's context was destroyed");
  if (g->ctx->device != c->device) return fail(XB_ERR_ARG, "graph lives on another device");
  if (mode == XB_MODE_ALTERNATING) {
    if (st) std::memset(st, 0, sizeof(*st));
    XB_CUDA(cudaSetDevice(c->device));
    return xbe::traverse_alternating(c, g, matching, level, parent, owner, flags, st);
  }
  if (mode != XB_MODE_PLAIN) return fail(XB_ERR_ARG, "unknown traversal mode");
  if (matching || owner) return fail(XB_ERR_ARG, "matching/owner must be NULL in plain mode");
  if (k < 0) return fail(XB_ERR_ARG, "negative source count");
  if (k > 0 && (!sources || !level || !parent)) return fail(XB_ERR_ARG, "null sources or output tables");
  if (st) std::memset(st, 0, sizeof(*st));
  if (k == 0) return XB_OK;
  XB_CUDA(cudaSetDevice(c->device));
  const bool src_dev = (flags & XB_SOURCES_DEVICE) != 0;
  const bool out_dev = (flags & XB_OUT_DEVICE) != 0;
  const bool fifo = (flags & XB_PARENT_FIFO) != 0;
  // validate sources (host copy)
  std::vector<int32_t> hs((size_t)k);
  if (src_dev) {
    XB_CUDA(cudaMemcpy(hs.data(), sources, sizeof(int32_t) * k, cudaMemcpyDeviceToHost));
  } else {
    std::memcpy(hs.data(), sources, sizeof(int32_t) * k);
  }
  for (int32_t i = 0; i < k; i++)
    if (hs[i] < 0 || hs[i] >= g->n) return fail(XB_ERR_ARG, "source " + std::to_string(i) + " out of range");
  xb_status s = xbe::ensure_sources(c, k);
  if (s != XB_OK) return s;
  // pass grouping: perm[i] = the caller's row of the i-th source traversed
  std::vector<int64_t> perm((size_t)k);
  for (int32_t i = 0; i < k; i++) perm[i] = i;
  if (c->tuning.source_order == 0 && k > c->tuning.word_bits * c->tuning.words) {
    s = xbe::order_by_degree(g, perm, [&](int64_t i) { return (int64_t)hs[i]; });
    if (s != XB_OK) return s;
    std::vector<int32_t> ps((size_t)k);
    for (int32_t i = 0; i < k; i++) ps[i] = hs[perm[i]];
    hs.swap(ps);
  }
  XB_CUDA(cudaMemcpyAsync(c->d_src, hs.data(), sizeof(int32_t) * k, cudaMemcpyHostToDevice, c->stream));
  XB_CUDA(cudaEventRecord(c->ev0, c->stream));
  const int64_t* pm = perm.data();
  if (c->tuning.word_bits == 64) {
    s = g->off64
            ? xbe::dispatch_nw<unsigned long long, int64_t>(c, g, c->d_src, pm, k, level, parent, out_dev, fifo, st)
            : xbe::dispatch_nw<unsigned long long, int32_t>(c, g, c->d_src, pm, k, level, parent, out_dev, fifo, st);
  } else {
    s = g->off64 ? xbe::dispatch_nw<unsigned int, int64_t>(c, g, c->d_src, pm, k, level, parent, out_dev, fifo, st)
                 : xbe::dispatch_nw<unsigned int, int32_t>(c, g, c->d_src, pm, k, level, parent, out_dev, fifo, st);
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
