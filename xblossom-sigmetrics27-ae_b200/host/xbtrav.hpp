// xbtrav.hpp -- C++ host API over the C ABI of libxbtrav.so, mirroring the
// reference engine's host interface for the traversal path.
//
// Reference (X-Blossom project paths)        here
//   zblossom::HGraph(row_path, col_path)      xbtrav::HGraph(row_path, col_path)
//     apps/xb/src/include/graph/hgraph.h:37-48  (same text format, nnodes/nedges
//                                                with nedges = entries / 2)
//   zblossom::DGraph(const HGraph&)           xbtrav::DGraph(Context&, const HGraph&)
//     apps/xb/src/include/graph/dgraph.h:50-63
//   Engine(const HGraph&, ratio) +            xbtrav::TraversalEngine(const DGraph&)
//   ExpandAlternatingForest (the expand           .Traverse(sources) -> Tables
//   phase, xblossom_gpu_engine_10.cu:270-359)
//
// Error behaviour: the reference aborts the process (CUDA_CHECK ->
// std::terminate, apps/xb/src/include/utils/utils_gpu.h:54-63); this layer
// throws xbtrav::Error carrying the xb_status and message instead, which a
// caller that wants the old behaviour can leave uncaught.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "xbtrav.h"

namespace xbtrav {

struct Error : std::runtime_error {
  xb_status status;
  Error(xb_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(xb_status s) {
  if (s != XB_OK) {
    const char* m = xb_last_error();
    throw Error(s, std::string(xb_status_str(s)) + ": " + (m ? m : ""));
  }
}

// Host CSR; nnodes / nedges follow HGraph (nedges = directed entries / 2).
class HGraph {
 public:
  HGraph(const std::string& row_offsets_path, const std::string& col_indices_path) {
    check(xb_csr_load_text(row_offsets_path.c_str(), col_indices_path.c_str(), &h_));
    bind();
  }
  static HGraph Rmat(int scale, int edge_factor, uint64_t seed, double a = 0.57, double b = 0.19,
                     double c = 0.19) {
    xb_host_csr* h = nullptr;
    check(xb_csr_gen_rmat(scale, edge_factor, a, b, c, seed, 0, &h));
    return HGraph(h);
  }
  HGraph(HGraph&& o) noexcept { *this = std::move(o); }
  HGraph& operator=(HGraph&& o) noexcept {
    std::swap(h_, o.h_);
    bind();
    o.bind();
    return *this;
  }
  HGraph(const HGraph&) = delete;
  HGraph& operator=(const HGraph&) = delete;
  ~HGraph() { xb_csr_free(h_); }

  size_t nnodes = 0, nedges = 0;
  const int64_t* row_offsets = nullptr;
  const int32_t* col_indices = nullptr;
  const xb_host_csr* handle() const { return h_; }

  std::vector<int32_t> SelectSources(uint64_t seed, int32_t k) const {
    std::vector<int32_t> s((size_t)k);
    check(xb_select_sources_csr((int64_t)nnodes, row_offsets, seed, k, s.data()));
    return s;
  }

 private:
  explicit HGraph(xb_host_csr* h) : h_(h) { bind(); }
  void bind() {
    if (!h_) {
      nnodes = nedges = 0;
      row_offsets = nullptr;
      col_indices = nullptr;
      return;
    }
    int64_t n = 0, m = 0;
    check(xb_csr_info(h_, &n, &m, nullptr, nullptr));
    nnodes = (size_t)n;
    nedges = (size_t)m / 2;
    check(xb_csr_arrays(h_, &row_offsets, &col_indices));
  }
  xb_host_csr* h_ = nullptr;
};

class Context {
 public:
  explicit Context(int device = 0) { check(xb_ctx_create(device, &c_)); }
  ~Context() { xb_ctx_destroy(c_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  xb_ctx* get() const { return c_; }
  void SetTuning(const xb_tuning& t) { check(xb_ctx_set_tuning(c_, &t)); }
  xb_tuning Tuning() const {
    xb_tuning t{};
    check(xb_ctx_get_tuning(c_, &t));
    return t;
  }

 private:
  xb_ctx* c_ = nullptr;
};

// Device-resident CSR (DGraph).
class DGraph {
 public:
  DGraph(Context& ctx, const HGraph& g) : ctx_(&ctx) { check(xb_graph_from_host_csr(ctx.get(), g.handle(), &g_)); }
  ~DGraph() { xb_graph_free(g_); }
  DGraph(const DGraph&) = delete;
  DGraph& operator=(const DGraph&) = delete;
  const xb_graph* get() const { return g_; }
  Context& ctx() const { return *ctx_; }
  // The engine's pass grouping of `sources` (xb_graph_source_order): indices
  // into sources by degree, highest first, ties by the neighbours' degree sum.
  std::vector<int32_t> SourceOrder(const std::vector<int32_t>& sources) const {
    std::vector<int32_t> order(sources.size());
    check(xb_graph_source_order(g_, sources.data(), (int32_t)sources.size(), order.data()));
    return order;
  }

 private:
  Context* ctx_;
  xb_graph* g_ = nullptr;
};

// Host tables of one traversal: level / parent, k x n, source-major.
struct Tables {
  int64_t n = 0;
  int32_t k = 0;
  std::vector<int32_t> level, parent;
  xb_stats stats{};
  int32_t Level(int32_t s, int64_t v) const { return level[(size_t)s * (size_t)n + (size_t)v]; }
  int32_t Parent(int32_t s, int64_t v) const { return parent[(size_t)s * (size_t)n + (size_t)v]; }
};

class TraversalEngine {
 public:
  explicit TraversalEngine(const DGraph& g) : g_(&g) {
    check(xb_graph_info(g.get(), &n_, nullptr, nullptr));
  }
  // Plain multi-source traversal into host tables (the drop-in path).
  Tables Traverse(const std::vector<int32_t>& sources) const {
    Tables t;
    t.n = n_;
    t.k = (int32_t)sources.size();
    t.level.resize((size_t)t.k * (size_t)n_);
    t.parent.resize((size_t)t.k * (size_t)n_);
    check(xb_traverse(g_->ctx().get(), g_->get(), sources.data(), t.k, XB_MODE_PLAIN, nullptr, t.level.data(),
                      t.parent.data(), nullptr, 0u, &t.stats));
    return t;
  }

 private:
  const DGraph* g_;
  int64_t n_ = 0;
};

// Many source sets -- on one graph or several -- traversed in ONE launch
// (xb_traverse_batched; no counterpart in the reference, whose engine runs
// one source set per host-driven loop).  Tables come back on the host.
class BatchedEngine {
 public:
  explicit BatchedEngine(Context& ctx) : ctx_(&ctx) {}
  struct Query {
    const DGraph* graph;
    std::vector<int32_t> sources;
  };
  std::vector<Tables> Traverse(const std::vector<Query>& queries, xb_stats* stats = nullptr) const {
    std::vector<xb_batch_item> items(queries.size());
    std::vector<Tables> out(queries.size());
    std::vector<int32_t*> bufs;  // page-locked: the copies run inside the launch
    struct Free {
      std::vector<int32_t*>& b;
      ~Free() {
        for (int32_t* p : b) xb_host_free(p);
      }
    } guard{bufs};
    for (size_t i = 0; i < queries.size(); i++) {
      int64_t n = 0;
      check(xb_graph_info(queries[i].graph->get(), &n, nullptr, nullptr));
      const int64_t k = (int64_t)queries[i].sources.size();
      out[i].n = n;
      out[i].k = (int32_t)k;
      void* p = nullptr;
      check(xb_host_alloc(sizeof(int32_t) * 2 * k * n, &p));
      bufs.push_back((int32_t*)p);
      items[i] = xb_batch_item{queries[i].graph->get(), queries[i].sources.data(), (int32_t)k, 0u, (int32_t*)p,
                               (int32_t*)p + k * n};
    }
    xb_stats st{};
    check(xb_traverse_batched(ctx_->get(), items.data(), (int32_t)items.size(), &st));
    for (size_t i = 0; i < queries.size(); i++) {
      const size_t kn = (size_t)out[i].k * (size_t)out[i].n;
      out[i].level.assign(items[i].level, items[i].level + kn);
      out[i].parent.assign(items[i].parent, items[i].parent + kn);
      out[i].stats = st;
    }
    if (stats) *stats = st;
    return out;
  }

 private:
  Context* ctx_;
};

// Maximum matching with the reference engine's interface
// (AbstractMaximumMatchingEngine, apps/xb/src/include/xbsm_gpu/max_match_engine.h:8-15):
// Matching[v] = the mate of v, nnodes for an exposed vertex.
using Matching = std::vector<int32_t>;

class MaximumMatchingEngine {
 public:
  explicit MaximumMatchingEngine(const DGraph& g) : g_(&g) { check(xb_graph_info(g.get(), &n_, nullptr, nullptr)); }
  // From the empty matching.
  Matching FindMaximumMatch(xb_stats* stats = nullptr) const {
    return FindMaximumMatch(Matching((size_t)n_, (int32_t)n_), stats);
  }
  // From an initial matching (xb_max_match; XB_ERR_ARG if it is not one).
  Matching FindMaximumMatch(const Matching& initial, xb_stats* stats = nullptr) const {
    if ((int64_t)initial.size() != n_) check(XB_ERR_ARG);
    std::vector<int32_t> mate(initial.size());
    for (size_t v = 0; v < initial.size(); v++) mate[v] = initial[v] == (int32_t)n_ ? -1 : initial[v];
    xb_stats st{};
    check(xb_max_match(g_->ctx().get(), g_->get(), mate.data(), 0u, &st));
    if (stats) *stats = st;
    Matching out(mate.size());
    for (size_t v = 0; v < mate.size(); v++) out[v] = mate[v] < 0 ? (int32_t)n_ : mate[v];
    return out;
  }

 private:
  const DGraph* g_;
  int64_t n_ = 0;
};

}  // namespace xbtrav
