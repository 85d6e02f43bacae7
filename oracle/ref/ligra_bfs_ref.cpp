// ligra_bfs_ref.cpp -- C-ABI wrapper that runs the reference's own CPU BFS.
//
// TEST / BASELINE INFRASTRUCTURE ONLY (never linked into the product).
//
// Compiled by oracle/Makefile against the unmodified Ligra sources vendored in
// the X-Blossom project (apps/ligra/ligra/*.h and apps/ligra/apps/BFS.C).  The
// search itself is Ligra's: the BFS_F functor of apps/ligra/apps/BFS.C:26-37
// (CAS parent claim) driven by Ligra's edgeMap with its dense/sparse
// (pull/push) switch, exactly the loop of apps/ligra/apps/BFS.C:42-53.  The
// only code here is the glue a caller needs: building Ligra's in-memory
// symmetric graph from an int64/int32 CSR (the in-memory equivalent of
// readGraphFromFile, apps/ligra/ligra/IO.h:163-240) and returning the Parents
// array instead of freeing it.
//
// Used for (1) pinning the oracle's level rule: the depth of every Ligra
// parent chain must equal the oracle level, and every Ligra parent must be a
// valid predecessor; (2) the timed reference CPU arm of bench.py.
#include "parallel.h"
// ligra.h defines the command-line main() through the parallel_main macro;
// this wrapper is a library, so that function is renamed out of the way.
#undef parallel_main
#define parallel_main ligra_unused_cli_main
#include "BFS.C"

#include <chrono>
#include <cstdint>

namespace {
struct NoopDeletable : public Deletable {
  void del() override {}
};
}  // namespace

extern "C" {

// Runs Ligra BFS from each of the k sources.  parents may be NULL (timing
// only); else it is k*n uint32 (UINT_E_MAX = unreached), source-major.
// Returns the wall time in seconds of the k searches (graph build excluded),
// or a negative value on a bad argument.
double ligra_ref_bfs(int64_t n, const int64_t* row_offsets, const int32_t* col_indices,
                     const int32_t* sources, int32_t k, uint32_t* parents,
                     int64_t* edges_traversed, int32_t threads) {
  if (n <= 0 || k < 0) return -1.0;
  if (threads > 0) setWorkers(threads);
  const int64_t m = row_offsets[n];
  uintE* edges = newA(uintE, m > 0 ? m : 1);
  for (int64_t i = 0; i < m; i++) edges[i] = (uintE)col_indices[i];
  symmetricVertex* V = newA(symmetricVertex, n);
  for (int64_t i = 0; i < n; i++) {
    V[i].setOutDegree((uintT)(row_offsets[i + 1] - row_offsets[i]));
    V[i].setOutNeighbors(edges + row_offsets[i]);
  }
  NoopDeletable* D = new NoopDeletable();
  graph<symmetricVertex> G(V, n, m, D);

  uintE* Parents = newA(uintE, n);
  int64_t edges_total = 0;
  double seconds = 0.0;
  for (int32_t q = 0; q < k; q++) {
    long start = sources[q];
    auto t0 = std::chrono::high_resolution_clock::now();
    // apps/ligra/apps/BFS.C:42-53 (the Compute body), Parents kept.
    parallel_for(long i = 0; i < n; i++) Parents[i] = UINT_E_MAX;
    Parents[start] = start;
    vertexSubset Frontier(n, start);
    while (!Frontier.isEmpty()) {
      vertexSubset output = edgeMap(G, Frontier, BFS_F(Parents));
      Frontier.del();
      Frontier = output;
    }
    Frontier.del();
    auto t1 = std::chrono::high_resolution_clock::now();
    seconds += std::chrono::duration<double>(t1 - t0).count();
    if (edges_traversed) {
      for (long i = 0; i < n; i++)
        if (Parents[i] != UINT_E_MAX) edges_total += row_offsets[i + 1] - row_offsets[i];
    }
    if (parents) {
      uint32_t* row = parents + (size_t)q * (size_t)n;
      for (long i = 0; i < n; i++) row[i] = (uint32_t)Parents[i];
    }
  }
  free(Parents);
  free(V);
  free(edges);
  delete D;
  if (edges_traversed) *edges_traversed = edges_total;
  return seconds;
}

int32_t ligra_ref_workers(void) { return (int32_t)getWorkers(); }

}  // extern "C"
