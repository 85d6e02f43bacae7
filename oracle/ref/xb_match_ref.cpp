// xb_match_ref.cpp -- C-ABI wrapper that runs the reference's own CPU
// maximum-matching engine (X-Blossom, per-node parallel variant).
//
// TEST INFRASTRUCTURE ONLY (never linked into the product).
//
// Compiled by oracle/Makefile from the unmodified X-Blossom sources where
// they lie: apps/xb/src/xblsm_cpu/par_pro_pernode.cu (included below as a
// C++ translation unit) and functions.cu / functions_for_par_{1,2}.cu
// (compiled beside it as C++).  The matcher is
// parFindMaximumMatchingNoRecursionUpdatePathTable_pro_pernode
// (par_pro_pernode.cu:42-90): repeated forest searches from all exposed
// vertices with blossom handling and path-table reuse, flipping the
// vertex-disjoint augmenting paths found, until none is left.  Its
// configuration globals live in xblsm_cpu_config.cu, which needs glog, so
// they are defined here instead (same names and types).
#include <chrono>
#include <climits>
#include <cstdint>
#include <vector>

namespace xblossom {
int nodes, num_of_threads, count;
std::chrono::microseconds duration_blossom, duration_augmenting_path, duration_expand, duration_edge,
    duration_prepare, duration_update;
uint64_t num_aug_path_discovery_iterations = 0, num_edges_processed = 0, num_expand_edges_processed = 0,
         cur_num_edges_processed = 0, num_blossom = 0, num_blossom_edges_processed = 0, num_reset_tree_nodes = 0,
         num_reused_tree_nodes = 0, num_aug_path = 0, num_aug_path_edges_processed = 0,
         num_search_phase_iterations = 0, max_num_edges_processed = 0;
bool stop_immediately = false;
}  // namespace xblossom

#include "xblsm_cpu/par_pro_pernode.cu"

extern "C" {

// match: n ints in/out (-1 unmatched); on entry the initial matching.
// Returns the matching size (edges), or -1 on a bad argument or an invalid
// result.
int64_t xb_ref_max_match(int64_t n, const int64_t* row_offsets, const int32_t* col_indices, int32_t threads,
                         int32_t* match) {
  if (n <= 0 || n > INT_MAX || !row_offsets || !match) return -1;
  std::vector<int> ro((size_t)n + 1), ci((size_t)row_offsets[n]);
  for (int64_t i = 0; i <= n; i++) ro[(size_t)i] = (int)row_offsets[i];
  for (int64_t e = 0; e < row_offsets[n]; e++) ci[(size_t)e] = col_indices[e];
  xblossom::Graph G(ro, ci);
  xblossom::nodes = (int)n;
  xblossom::num_of_threads = threads > 0 ? threads : 1;
  xblossom::count = 0;
  std::vector<int> M(match, match + n);
  bool valid = true;
  xblossom::parFindMaximumMatchingNoRecursionUpdatePathTable_pro_pernode(G, M, valid, INT_MAX);
  if (!valid) return -1;
  int64_t size = 0;
  for (int64_t i = 0; i < n; i++) {
    match[i] = M[(size_t)i];
    if (M[(size_t)i] >= 0) size++;
  }
  return size / 2;
}

}  // extern "C"
