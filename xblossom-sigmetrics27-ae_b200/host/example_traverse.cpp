// example_traverse.cpp -- reference-style C++ caller of libxbtrav.so.
//
//   example_traverse <row_offsets.txt> <col_indices.txt> <k> <seed> [--batched | --match]
//   example_traverse --rmat <scale> <edge_factor> <k> <seed> [--batched | --match]
//
// Loads (or generates) a CSR the way the reference runners do (HGraph from
// two text files, apps/xb/runner/xblsm_gpu/run_xb_pp_by_dataset.cu:7-40),
// uploads it, traverses k seeded sources and prints one summary line plus a
// checksum of both tables.  --batched splits the sources into three queries
// run in one launch (BatchedEngine); the tables, and so the checksum, are the
// same.  --match runs FindMaximumMatch (MaximumMatchingEngine) from the empty
// matching instead and prints its size.  Exit status 0 on success.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "xbtrav.hpp"

int main(int argc, char** argv) {
  try {
    if (argc < 5) {
      std::fprintf(stderr, "usage: %s <row.txt> <col.txt> <k> <seed> | --rmat <scale> <ef> <k> <seed>\n", argv[0]);
      return 2;
    }
    const bool rmat = std::strcmp(argv[1], "--rmat") == 0;
    xbtrav::HGraph g = rmat ? xbtrav::HGraph::Rmat(std::atoi(argv[2]), std::atoi(argv[3]), 0x5EED)
                            : xbtrav::HGraph(argv[1], argv[2]);
    const int k = std::atoi(argv[rmat ? 4 : 3]);
    const uint64_t seed = std::strtoull(argv[rmat ? 5 : 4], nullptr, 0);
    xbtrav::Context ctx(0);
    xbtrav::DGraph dg(ctx, g);
    xbtrav::TraversalEngine eng(dg);
    if (std::strcmp(argv[argc - 1], "--match") == 0) {
      xb_stats st{};
      const xbtrav::Matching mt = xbtrav::MaximumMatchingEngine(dg).FindMaximumMatch(&st);
      size_t matched = 0;
      for (size_t v = 0; v < mt.size(); v++) {
        if (mt[v] == (int32_t)g.nnodes) continue;
        if (mt[(size_t)mt[v]] != (int32_t)v) throw xbtrav::Error(XB_ERR_STATE, "matching not symmetric");
        matched++;
      }
      std::printf("nnodes=%zu nedges=%zu matching_size=%zu phases=%d\n", g.nnodes, g.nedges, matched / 2, st.batches);
      return 0;
    }
    const auto sources = g.SelectSources(seed, k);
    const bool batched = std::strcmp(argv[argc - 1], "--batched") == 0;
    xbtrav::Tables t;
    if (!batched) {
      t = eng.Traverse(sources);
    } else {
      // three queries of the same graph: k/3, k/3 and the rest of the sources
      std::vector<xbtrav::BatchedEngine::Query> qs;
      const int cut[4] = {0, k / 3, 2 * k / 3, k};
      for (int q = 0; q < 3; q++)
        qs.push_back({&dg, std::vector<int32_t>(sources.begin() + cut[q], sources.begin() + cut[q + 1])});
      const auto parts = xbtrav::BatchedEngine(ctx).Traverse(qs, &t.stats);
      t.n = (int64_t)g.nnodes;
      t.k = k;
      for (const auto& p : parts) {
        t.level.insert(t.level.end(), p.level.begin(), p.level.end());
        t.parent.insert(t.parent.end(), p.parent.begin(), p.parent.end());
      }
    }
    uint64_t h = 1469598103934665603ull;  // FNV-1a over both tables
    for (int32_t x : t.level) h = (h ^ (uint32_t)x) * 1099511628211ull;
    for (int32_t x : t.parent) h = (h ^ (uint32_t)x) * 1099511628211ull;
    std::printf("nnodes=%zu nedges=%zu k=%d edges_traversed=%lld levels=%d checksum=%016llx\n", g.nnodes, g.nedges,
                k, (long long)t.stats.edges_traversed, t.stats.levels, (unsigned long long)h);
    return 0;
  } catch (const xbtrav::Error& e) {
    std::fprintf(stderr, "xbtrav error %d: %s\n", e.status, e.what());
    return 1;
  }
}
