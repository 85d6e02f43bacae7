// ligra_msssp_ref.cpp -- C-ABI wrapper that runs the reference's own CPU
// multi-source SSSP.
//
// TEST INFRASTRUCTURE ONLY (never linked into the product).
//
// Compiled by oracle/Makefile against the unmodified Ligra sources vendored in
// the X-Blossom project (apps/ligra/ligra/*.h and apps/ligra/apps/MultiSSSP.C,
// which defines WEIGHTED).  The search is Ligra's: the SSSP_F functor
// (writeMin on the shared float distance, CAS on Visited) and Reset_F of
// MultiSSSP.C, driven by edgeMap / vertexMap exactly as the loop of its
// Compute (the round loop, with the round == n guard that sets every
// distance to -infinity).  The glue here builds Ligra's in-memory weighted
// symmetric graph from a CSR plus int32 weights (interleaved (neighbour,
// weight) pairs, the layout readGraphFromFile produces for weighted files,
// apps/ligra/ligra/IO.h:200-230) and seeds the frontier from a source array
// instead of the command line.
#include "parallel.h"
#undef parallel_main
#define parallel_main ligra_unused_cli_main
#include "MultiSSSP.C"

#include <cstdint>

namespace {
struct NoopDeletable : public Deletable {
  void del() override {}
};
}  // namespace

extern "C" {

// dist: n floats (unreached: the reference's infinity, FLT_MAX / 4).
// Returns 0, or -1 on a bad argument.
int ligra_ref_msssp(int64_t n, const int64_t* row_offsets, const int32_t* col_indices, const int32_t* weights,
                    const int32_t* sources, int32_t k, float* dist, int32_t threads) {
  if (n <= 0 || k <= 0 || !dist) return -1;
  for (int32_t q = 0; q < k; q++)
    if (sources[q] < 0 || sources[q] >= n) return -1;
  if (threads > 0) setWorkers(threads);
  const int64_t m = row_offsets[n];
  intE* edges = newA(intE, 2 * (m > 0 ? m : 1));
  for (int64_t i = 0; i < m; i++) {
    edges[2 * i] = (intE)col_indices[i];
    edges[2 * i + 1] = (intE)weights[i];
  }
  symmetricVertex* V = newA(symmetricVertex, n);
  for (int64_t i = 0; i < n; i++) {
    V[i].setOutDegree((uintT)(row_offsets[i + 1] - row_offsets[i]));
    V[i].setOutNeighbors(edges + 2 * row_offsets[i]);
  }
  NoopDeletable* D = new NoopDeletable();
  graph<symmetricVertex> G(V, n, m, D);

  weightT* Dist = newA(weightT, n);
  const weightT infinity = std::numeric_limits<weightT>::max() / 4;
  parallel_for(long i = 0; i < n; i++) Dist[i] = infinity;
  bool* src = newA(bool, n);
  parallel_for(long i = 0; i < n; i++) src[i] = false;
  long count = 0;
  for (int32_t q = 0; q < k; q++) {
    if (!src[sources[q]]) {
      src[sources[q]] = true;
      Dist[sources[q]] = 0;
      count++;
    }
  }
  vertexSubset Frontier(n, count, src);
  int* Visited = newA(int, n);
  parallel_for(long i = 0; i < n; i++) Visited[i] = 0;
  long round = 0;
  while (!Frontier.isEmpty()) {
    if (round == n) {
      parallel_for(long i = 0; i < n; i++) Dist[i] = -infinity;
      break;
    }
    vertexSubset output = edgeMap(G, Frontier, SSSP_F(Dist, Visited));
    vertexMap(output, Reset_F(Visited));
    Frontier.del();
    Frontier = output;
    round++;
  }
  Frontier.del();
  for (long i = 0; i < n; i++) dist[i] = Dist[i];
  free(Dist);
  free(Visited);
  free(V);
  free(edges);
  delete D;
  return 0;
}

}  // extern "C"
