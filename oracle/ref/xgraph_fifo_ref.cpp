// xgraph_fifo_ref.cpp -- C-ABI wrapper around the reference's deterministic
// sequential BFS with predecessors.
//
// TEST INFRASTRUCTURE ONLY (never linked into the product).
//
// Compiled by oracle/Makefile against the unmodified header
// apps/xb/src/include/graph/xgraph.h of the X-Blossom project.  The graph is
// built with the reference's own CSR constructor and adjacency builder
// (xblossom::Graph(rowOffsets, colIndices) + buildAdjListFromCSR,
// xgraph.h:341-356) and every path comes from
// xblossom::Graph::findShortestPath (xgraph.h:155-191): a FIFO queue whose
// neighbours are visited in CSR order, first discoverer = predecessor.
//
// For each (source, destination) pair the wrapper records the path length
// (= the level) and the second-to-last vertex (= the FIFO parent).  The caller
// passes only destinations it knows to be reachable: findShortestPath's
// predecessor walk does not terminate for an unreachable destination whose
// default predecessor entry (0) is itself unvisited.
#include "graph/xgraph.h"

#include <cstdint>
#include <vector>

extern "C" {

// n vertices, int32 CSR.  For q in [0, npairs): runs findShortestPath(src[q],
// dst[q]) and writes out_level[q] = |path|-1 and out_parent[q] = the vertex
// before dst on the path (src itself for dst == src; -1 when the reference
// returns an empty path, e.g. for a vertex without edges).
int32_t xgraph_ref_paths(int32_t n, const int32_t* row_offsets, const int32_t* col_indices,
                         const int32_t* src, const int32_t* dst, int64_t npairs,
                         int32_t* out_level, int32_t* out_parent) {
  if (n <= 0 || npairs < 0) return -1;
  std::vector<int> ro(row_offsets, row_offsets + n + 1);
  std::vector<int> ci(col_indices, col_indices + ro[n]);
  xblossom::Graph g(ro, ci);
  g.buildAdjListFromCSR();
  for (int64_t q = 0; q < npairs; q++) {
    std::list<int> path = g.findShortestPath(src[q], dst[q]);
    if (path.empty()) {
      out_level[q] = -1;
      out_parent[q] = -1;
      continue;
    }
    out_level[q] = (int32_t)path.size() - 1;
    if (path.size() == 1) {
      out_parent[q] = path.back();
    } else {
      auto it = path.rbegin();
      ++it;
      out_parent[q] = *it;
    }
  }
  return 0;
}

}  // extern "C"
