/*
 * xbtrav.h -- C ABI of the B200 multi-source traversal engine (libxbtrav.so).
 *
 * The engine traverses an undirected CSR graph from many sources at once and
 * returns, per source, an int32 level table and an int32 parent table
 * (k x n, source-major: level[s*n + v]).  Every call returns an xb_status
 * (0 = OK, negative = error; xb_status_str / xb_last_error explain it).
 * Buffers are caller-owned unless a function says otherwise.  No torch or C++
 * types cross this boundary.
 *
 * Reference interfaces these entry points replace (paths relative to the
 * X-Blossom project):
 *   CSR load            zblossom::HGraph(row_path, col_path)
 *                       apps/xb/src/include/graph/hgraph.h:37-48, text format
 *                       one int per line apps/xb/src/include/common/utils_cpu.h:9-23
 *   device graph        zblossom::DGraph(const HGraph&)
 *                       apps/xb/src/include/graph/dgraph.h:50-63
 *   source set          exposed-vertex roots
 *                       apps/xb/src/xblsm_gpu/xblossom_gpu_engine_10.cu:119-144;
 *                       experiment source lists scripts/2-datasets/src_nodes/generate_src_lists.py
 *   traversal           Engine::ExpandAlternatingForest
 *                       apps/xb/src/xblsm_gpu/xblossom_gpu_engine_10.cu:270-359 and
 *                       parExpand_pro_all apps/xb/src/xblsm_cpu/par_pro_pernode.cu:178-234;
 *                       plain BFS semantics apps/ligra/apps/BFS.C:26-53
 *   level / parent      PathTable root_distance_ / ExpandTwoNodes
 *                       apps/xb/src/include/path_table/path_table.h:222,256-271
 */
#ifndef XBTRAV_H
#define XBTRAV_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XB_ABI_VERSION 3

typedef int32_t xb_status;
#define XB_OK 0
#define XB_ERR_ARG (-1)      /* bad argument (null pointer, out-of-range id, size) */
#define XB_ERR_OOM (-2)      /* device or host allocation failed */
#define XB_ERR_CAPACITY (-3) /* a table or queue would overflow its fixed capacity */
#define XB_ERR_TIMEOUT (-4)  /* a bounded device-side wait gave up */
#define XB_ERR_CUDA (-5)     /* a CUDA runtime call failed */
#define XB_ERR_IO (-6)       /* file could not be read or written */
#define XB_ERR_NODEV (-7)    /* no usable CUDA device */
#define XB_ERR_STATE (-8)    /* object used in the wrong state */

#define XB_MODE_PLAIN 0       /* independent BFS per source */
#define XB_MODE_ALTERNATING 1 /* alternating forest of a matching from its exposed vertices */

/* xb_traverse flags */
#define XB_OUT_DEVICE 1u     /* level/parent are device pointers (else host) */
#define XB_SOURCES_DEVICE 2u /* sources is a device pointer (else host) */
#define XB_PARENT_FIFO 4u    /* xb_traverse only: parents by the FIFO rule (see xb_traverse) */

typedef struct xb_host_csr xb_host_csr; /* host-resident CSR (int64 offsets) */
typedef struct xb_ctx xb_ctx;           /* device, stream, workspace */
typedef struct xb_graph xb_graph;       /* device-resident CSR */

/* Counters of one traversal call.  edges_traversed is the work unit of the
 * GTEPS metric: sum over sources of sum over reached vertices of deg(v), the
 * "Processed Edges" of apps/ligra/apps/BFS_Throughput.C:42-63. */
typedef struct xb_stats {
  int64_t edges_traversed;  /* GTEPS numerator */
  int64_t reached;          /* sum over sources of reached vertices */
  int64_t edges_scanned;    /* CSR entries read by the level steps */
  int64_t vertices_scanned; /* vertices whose adjacency the level steps read */
  int64_t vertices_swept;   /* vertex state words swept by the level steps */
  int64_t parent_edges_scanned; /* CSR entries read by the parent pass */
  int64_t algo_bytes;       /* algorithmic HBM bytes of the whole call */
  int32_t levels;           /* max depth + 1 over all sources */
  int32_t push_levels;
  int32_t pull_levels;
  int32_t batches;          /* source words processed */
  double device_ms;         /* device time of the call (CUDA events) */
  /* per kernel class (0 = level steps, 1 = parent/table pass, 2 = other):
   * launches, device ms (events; only when timing is enabled) and
   * algorithmic bytes. */
  int64_t class_launches[3];
  double class_ms[3];
  int64_t class_bytes[3];
} xb_stats;

/* Tunables of the engine (the autotuner's search space). */
typedef struct xb_tuning {
  int32_t word_bits;       /* sources per word: 32 or 64 */
  int32_t words;           /* words per vertex traversed together: 1, 2 or 4 */
  float pull_alpha;        /* pull when frontier_edges*alpha > unfinished_edges */
  int32_t heavy_degree;    /* vertices above this degree get block-wide passes */
  int32_t timing;          /* 1 = record per-class CUDA events into xb_stats */
  int32_t chains;          /* xb_traverse_batched: passes in flight at once, each with its
                              own workspace (1..16; 0 = default 4) */
  /* Limits for exercising the error paths without faulting anything (0 =
   * off, the default).  level_cap: a pass whose frontier is still alive at
   * this level stops there, as a pass beyond the structural bound (levels <
   * 2^planes, which a correct traversal never reaches) does, and the call
   * returns XB_ERR_STATE.  workspace_cap: a working-memory allocation of the
   * traversal paths (plain workspace and staging, batched chain workspaces,
   * serving slot workspaces, SSSP / matching scratch) above this many bytes
   * fails with XB_ERR_OOM before cudaMalloc is called. */
  int32_t level_cap;
  /* Launch tile of the pull and table kernels (the autotuner's tile axis):
   * 0 (default) = heavy-vertex pull with one 32-edge round in flight per warp
   * at four words per vertex (four rounds otherwise) and 4-warp table blocks;
   * 1 = two rounds in flight at every layout and 8-warp table blocks. */
  int32_t tile;
  int64_t workspace_cap;
  /* After a pull step, push when the frontier holds fewer than n/push_beta
   * vertices (the traversal's tail); 0 = never. */
  float push_beta;
  /* How a call's sources are grouped into passes: 0 (default) = by source
   * degree, highest first, equal degrees by their neighbours' degree sum
   * (xb_graph_source_order; sources whose traversals grow alike share a
   * pass's level steps: fewer steps with few live lanes); 1 = in the order
   * given.  Output rows stay where the caller asked for them either way.
   * xb_traverse_batched with host output tables keys its captured copies
   * on the grouping, so a stream of calls with host tables and new source
   * lists recaptures under 0 and reuses one graph under 1. */
  int32_t source_order;
} xb_tuning;

/* ---- status ------------------------------------------------------------ */
const char* xb_status_str(xb_status s);
/* Message of the last error raised on the calling thread ("" if none). */
const char* xb_last_error(void);
int32_t xb_abi_version(void);

/* ---- host CSR (no GPU needed) ------------------------------------------ */
/* Seeded undirected R-MAT: n = 2^scale, n*edge_factor sampled pairs with
 * quadrant probabilities a, b, c (d = 1-a-b-c); symmetrised, self-loops and
 * duplicates removed, adjacency sorted ascending.  threads <= 0: all cores. */
xb_status xb_csr_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                          uint64_t seed, int32_t threads, xb_host_csr** out);
/* Seeded Erdos-Renyi style graph: m_pairs uniform vertex pairs, same cleaning. */
xb_status xb_csr_gen_er(int64_t n, int64_t m_pairs, uint64_t seed, int32_t threads,
                        xb_host_csr** out);
/* Copies and validates a CSR (ids in range; offsets non-decreasing). */
xb_status xb_csr_from_arrays(int64_t n, const int64_t* row_offsets, const int32_t* col_indices,
                             xb_host_csr** out);
/* Reference text format: one integer per line, row offsets file and column
 * indices file (HGraph(row_path, col_path), hgraph.h:37-48). */
xb_status xb_csr_load_text(const char* row_path, const char* col_path, xb_host_csr** out);
xb_status xb_csr_save_text(const xb_host_csr* g, const char* row_path, const char* col_path);
/* Native binary CSR: 8-byte magic "XBCSR\0\1\0", int64 n, int64 m, int64
 * row offsets (n+1), int32 column indices (m), little-endian. */
xb_status xb_csr_save_binary(const xb_host_csr* g, const char* path);
xb_status xb_csr_load_binary(const char* path, xb_host_csr** out);
/* Source-list files of the reference's experiment scripts
 * (scripts/2-datasets/src_nodes/generate_src_lists.py writes them,
 * source_nodes_from_file in scripts/4-expr/common.sh reads them): "#" starts
 * a comment (whole line or trailing), ids are separated by white space.
 * Load writes up to capacity ids and sets *count to the number in the file
 * (XB_ERR_CAPACITY if that is more). */
xb_status xb_sources_load(const char* path, int32_t* out, int32_t capacity, int32_t* count);
xb_status xb_sources_save(const char* path, const int32_t* sources, int32_t k, const char* comment);
/* Exports for cross-checks with other engines: Ligra "AdjacencyGraph" text
 * (n, m, n offsets, m targets) and Matrix Market coordinate pattern
 * symmetric, one 1-based (i < j) entry per undirected edge in ascending
 * order -- the entry lines of scripts/2-datasets/gunrock/csr_to_gunrock_mm.py.
 * A Matrix Market coordinate file (any field; values ignored) loads as the
 * symmetric, loop-free, duplicate-free pattern graph. */
xb_status xb_csr_save_ligra(const xb_host_csr* g, const char* path);
xb_status xb_csr_save_mtx(const xb_host_csr* g, const char* path);
xb_status xb_csr_load_mtx(const char* path, xb_host_csr** out);
xb_status xb_csr_info(const xb_host_csr* g, int64_t* n, int64_t* m, int64_t* max_degree,
                      int64_t* isolated);
/* Borrowed pointers, valid until xb_csr_free. */
xb_status xb_csr_arrays(const xb_host_csr* g, const int64_t** row_offsets,
                        const int32_t** col_indices);
void xb_csr_free(xb_host_csr* g);
/* k distinct sources drawn uniformly without replacement from the vertices of
 * non-zero degree, splitmix64 stream seeded by seed. */
xb_status xb_select_sources_csr(int64_t n, const int64_t* row_offsets, uint64_t seed, int32_t k,
                                int32_t* out);

/* ---- device context and graphs ----------------------------------------- */
xb_status xb_ctx_create(int32_t device, xb_ctx** out);
xb_status xb_ctx_destroy(xb_ctx* ctx);
xb_status xb_ctx_set_tuning(xb_ctx* ctx, const xb_tuning* t);
xb_status xb_ctx_get_tuning(const xb_ctx* ctx, xb_tuning* t);
/* Device workspace bytes currently held by the context. */
xb_status xb_ctx_workspace_bytes(const xb_ctx* ctx, int64_t* bytes);
/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or timing events against the engine's launches. */
xb_status xb_ctx_get_stream(const xb_ctx* ctx, void** stream);

/* Uploads a CSR (row offsets int32 or int64 as offsets_are_64bit says; host
 * pointers) and keeps it resident. */
xb_status xb_graph_upload(xb_ctx* ctx, int64_t n, const void* row_offsets,
                          int32_t offsets_are_64bit, int64_t m, const int32_t* col_indices,
                          xb_graph** out);
xb_status xb_graph_from_host_csr(xb_ctx* ctx, const xb_host_csr* g, xb_graph** out);
/* Uploads ninst independent graphs stored back to back as ONE device CSR with
 * per-instance offsets: instance i has inst_n[i] vertices; its row offsets
 * (inst_n[i] + 1 entries, local, starting at 0) follow those of instance i-1
 * in row_offsets, and its column indices (local ids, row_offsets[..][n]
 * entries) follow those of instance i-1 in col_indices.  out[i] receives a
 * graph handle per instance (views of the shared arrays; each is freed with
 * xb_graph_free, the arrays with the last of them).  Offsets are stored as
 * int32 unless an instance has 2^31-1 or more entries. */
xb_status xb_graph_upload_batch(xb_ctx* ctx, int32_t ninst, const int64_t* inst_n,
                                const int64_t* row_offsets, const int32_t* col_indices,
                                xb_graph** out);
xb_status xb_graph_load_csr_text(xb_ctx* ctx, const char* row_path, const char* col_path,
                                 xb_graph** out);
xb_status xb_graph_free(xb_graph* g);
/* Row offsets live on the device as int32 when the graph has fewer than
 * 2^31 - 1 entries, else as int64.  Setting XB_OFFSETS64=1 in the
 * environment keeps int64 offsets for every graph uploaded meanwhile (tests
 * of the int64 kernels on small graphs). */
xb_status xb_graph_info(const xb_graph* g, int64_t* n, int64_t* m, int64_t* max_degree);
/* Width of the graph's device row offsets: 4 or 8 bytes. */
xb_status xb_graph_offset_bytes(const xb_graph* g, int32_t* bytes);
xb_status xb_select_sources(const xb_graph* g, uint64_t seed, int32_t k, int32_t* out);
/* The pass grouping of tuning.source_order 0: order[i] = the index (into
 * sources) of the i-th source to traverse, by out-degree, highest first,
 * ties in the given order.  For host schedulers that split a query over
 * several passes themselves (xb_slot_launch).  No reference counterpart. */
xb_status xb_graph_source_order(const xb_graph* g, const int32_t* sources, int32_t k, int32_t* order);

/* ---- traversal ---------------------------------------------------------- */
/* Plain per-call path (the drop-in).  k sources; level and parent receive
 * k*n int32 each, source-major.  level = hop distance (-1 unreached); parent =
 * the smallest-id neighbour one level closer to the source (the source's own
 * parent is itself; -1 unreached).  Sources are processed in passes of
 * tuning.word_bits * tuning.words sources (64-bit words, four per vertex by
 * default: 256 sources per pass), one pass per launch sequence, with a
 * host-side level loop; with more sources than one pass holds, they are
 * grouped into passes as tuning.source_order says (by degree by default) and
 * every source's rows still land at its index in `sources`.
 * In plain mode matching and owner must be NULL.
 * XB_MODE_ALTERNATING: the alternating forest of `matching` (n ints, -1 =
 * exposed) grown from every exposed vertex, the expansion of the reference's
 * alternating mode (ExpandAlternatingForest, xblossom_gpu_engine_10.cu:270-359;
 * ExpandTwoNodes records, path_table.h:256-271); sources and k are ignored.
 * level, parent, owner: n ints each -- exposed vertices level 0 and their own
 * parent and owner; an inner vertex w at level 2d+1 has parent = its
 * smallest outer neighbour of level 2d; its mate is outer at level 2d+2 with
 * parent w; owner = the tree's root; -1 unreached.  When both ends of a
 * matched pair qualify at one level, the end with the smaller such
 * neighbour (then the smaller id) is the inner one.  Edges between outer
 * vertices label nothing.  XB_OUT_DEVICE: matching and the three outputs
 * are device pointers.  stats.levels = expansion rounds, stats.reached =
 * labeled vertices (host outputs).  XB_ERR_ARG if matching is not a
 * matching of the graph.
 * With XB_PARENT_FIFO the parents follow the reference's sequential FIFO
 * search instead (xblossom::Graph::findShortestPath, xgraph.h:155-191): a
 * vertex's parent is the first vertex of the BFS queue adjacent to it, the
 * queue of a level ordered by (parent's place, place in the parent's
 * adjacency); levels are the same.  The graph must hold no duplicate
 * adjacency entries for this rule. */
xb_status xb_traverse(xb_ctx* ctx, const xb_graph* g, const int32_t* sources, int32_t k,
                      int32_t mode, const int32_t* matching, int32_t* level, int32_t* parent,
                      int32_t* owner, uint32_t flags, xb_stats* stats);

/* Page-locked host memory (for host tables of the batched call). */
xb_status xb_host_alloc(int64_t bytes, void** out);
xb_status xb_host_free(void* p);

/* ---- batched traversal ------------------------------------------------- */
/* One query of a batch: k sources on a resident graph, tables k*n int32 each
 * (source-major), with the same meaning as xb_traverse's.  flags:
 * XB_SOURCES_DEVICE (sources is a device pointer) and XB_OUT_DEVICE (level /
 * parent are device pointers; otherwise they must be page-locked host memory,
 * from cudaHostAlloc or cudaHostRegister, so the copies can run inside the
 * launch). */
typedef struct xb_batch_item {
  const xb_graph* graph;
  const int32_t* sources;
  int32_t k;
  uint32_t flags;
  int32_t* level;
  int32_t* parent;
} xb_batch_item;

/* Batched path (the reference has none: its engine runs one source set per
 * host-driven loop, xblossom_gpu_engine_10.cu:72-185).  All queries of the
 * batch -- on one graph or several, of any sizes -- run as ONE CUDA-graph
 * launch: the sources of queries on the same graph are packed into passes of
 * tuning.word_bits * tuning.words regardless of which query they come from
 * (grouped by degree under tuning.source_order 0), the passes are
 * spread over tuning.chains concurrent chains, and each pass's level loop runs
 * on the device (conditional WHILE / SWITCH nodes pick push or pull per level
 * from the frontier counters; no host round trip per level).  The launch is
 * cached: calls with the same queries shape (graphs, k per query, flags and,
 * for host outputs, the output pointers and the sources' grouping) reuse it;
 * sources and device output pointers may change freely between such calls.  Results are identical to
 * xb_traverse's.  stats (may be NULL) sums over the whole batch. */
xb_status xb_traverse_batched(xb_ctx* ctx, const xb_batch_item* items, int32_t nitems,
                              xb_stats* stats);

/* ---- serving slots ------------------------------------------------------ */
/* Summary of one source's tables, for serving clients that need no full
 * tables: reached = vertices with level >= 0, level_sum over them, depth =
 * the largest level, and row_hash = the wrapping 64-bit sum over reached
 * vertices v of h(v, level[v], parent[v]), where h is the splitmix64
 * finalizer of (v * 0x9E3779B97F4A7C15) XOR ((uint32 level << 32) | uint32
 * parent) -- position-sensitive (a parent moved between vertices changes it)
 * and independent of the order the entries are summed in.  Stored as the
 * int64 with the same bits. */
typedef struct xb_row_digest {
  int64_t reached;
  int64_t level_sum;
  int64_t row_hash;
  int32_t depth; /* -1 for a row written to a caller buffer (no digest taken) */
  int32_t pad;
} xb_row_digest;

#define XB_MAX_SLOTS 16
/* Asynchronous passes for a serving loop (no counterpart in the reference,
 * which has no serving path).  A slot (0..XB_MAX_SLOTS-1) runs one pass of up
 * to word_bits*words sources of ONE graph at a time, on its own stream and
 * workspace, so passes on different slots overlap on the device; a host
 * scheduler packs the sources of whatever queries are waiting into each pass.
 * level_rows[j] / parent_rows[j] are device pointers to the n-entry rows of
 * source j (sources is a host array); a NULL pair sends both rows to the
 * slot's scratch and only their digest comes back.  The slot must be idle
 * (XB_ERR_STATE otherwise); the call returns once the pass is queued.
 * Results match xb_traverse's for the same sources. */
xb_status xb_slot_launch(xb_ctx* ctx, int32_t slot, const xb_graph* g, const int32_t* sources,
                         int32_t kb, int32_t* const* level_rows, int32_t* const* parent_rows);
/* Non-blocking: *done = 0 while the slot's pass runs; *done = 1 once it has
 * finished, with its counters in stats and kb digests in digests (either may
 * be NULL); the slot is then idle.  XB_ERR_STATE for an idle slot. */
xb_status xb_slot_poll(xb_ctx* ctx, int32_t slot, int32_t* done, xb_stats* stats,
                       xb_row_digest* digests);
/* Blocking form of xb_slot_poll. */
xb_status xb_slot_wait(xb_ctx* ctx, int32_t slot, xb_stats* stats, xb_row_digest* digests);
/* Frees every slot's device memory (all slots must be idle). */
xb_status xb_slots_release(xb_ctx* ctx);
/* Stream priority of a slot: 0 = default, 1 = the device's greatest; an
 * idle slot only.  Passes on a priority-1 slot have their kernels scheduled
 * ahead of the other slots' (a serving loop's express lane for small
 * queries).  Kept across xb_slots_release.  No counterpart in the
 * reference (it has no serving path). */
xb_status xb_slot_set_priority(xb_ctx* ctx, int32_t slot, int32_t priority);

/* ---- weighted: multi-source shortest paths ------------------------------ */
/* Attaches int32 edge weights to a resident graph, one per column index
 * (weights[e] belongs to col_indices[e]; an undirected edge carries its
 * weight in both directions).  Host pointer. */
xb_status xb_graph_set_weights(xb_graph* g, const int32_t* weights, int64_t m);
/* Multi-source shortest-path distances: dist[v] (n floats) = the smallest
 * float sum of weights over paths from any of the k sources to v, the
 * semantics of Ligra's MultiSSSP in the reference's baselines
 * (apps/ligra/apps/MultiSSSP.C): unreached vertices get FLT_MAX / 4, and every
 * vertex -FLT_MAX / 4 when the distances still change after n rounds (a
 * negative cycle -- in an undirected graph, any reachable negative weight).
 * flags: XB_OUT_DEVICE (dist is a device pointer), XB_SOURCES_DEVICE.  Uses
 * the context's workspace (a later xb_traverse rebuilds its state). */
xb_status xb_multi_sssp(xb_ctx* ctx, const xb_graph* g, const int32_t* sources, int32_t k, float* dist,
                        uint32_t flags, xb_stats* stats);

/* ---- alternating mode: maximum matching --------------------------------- */
/* Maximum-cardinality matching of a resident graph (undirected: symmetric
 * CSR), replacing the reference's FindMaximumMatch(const Matching&)
 * (apps/xb/src/include/xbsm_gpu/max_match_engine.h:93-113, engine
 * apps/xb/src/xblsm_gpu/xblossom_gpu_engine_10.cu:72-80): repeated forest
 * searches from all exposed vertices, augmenting along vertex-disjoint
 * paths, blossoms contracted, until a search finds no augmenting path.
 * mate: n ints, in = the initial matching (-1 = exposed; the reference's
 * engines use nnodes as that value), out = a maximum matching.  Host
 * pointer, or device pointer with XB_OUT_DEVICE.  An initial mate array
 * that is not a matching of the graph gives XB_ERR_ARG.  stats: batches =
 * search phases, levels = forest levels, pull_levels = levels that
 * contracted blossoms, vertices_scanned = augmenting paths flipped,
 * edges_scanned = adjacency entries expanded, reached = matching size (host
 * mate only).  Graphs of up to 2^29 - 1 vertices; uses the context's
 * workspace (a later xb_traverse rebuilds its state). */
xb_status xb_max_match(xb_ctx* ctx, const xb_graph* g, int32_t* mate, uint32_t flags, xb_stats* stats);

/* ---- traversal without device allocation -------------------------------- */
/* No counterpart in the reference (whose engine allocates all its device
 * buffers itself): an entry point for callers that may not allocate device
 * memory -- a plugin whose host owns the GPU's memory through its own pool,
 * or a latency-critical path where cudaMalloc/cudaFree and their implicit
 * device synchronisation are not allowed.  Same results as xb_traverse in
 * plain mode (64 sources per word).  Every pointer is a device pointer the
 * caller owns: int32 CSR (row_offsets n+1, col_indices row_offsets[n]),
 * k sources, level and parent tables k*n each, source-major.  stream is a
 * cudaStream_t (NULL = the legacy default stream); the call returns after
 * the work on it has finished.  Working state lives in one fixed array of
 * about 32 MiB compiled into the library, held by every GPU that loads the
 * library until exit; graphs above XB_NOALLOC_MAX_VERTICES vertices are
 * rejected with XB_ERR_CAPACITY.  The first call on a device looks up the
 * array's address (do it before any stream capture on that device); the
 * address is kept per device context, so after cudaDeviceReset the next call
 * looks it up again.  Every call first checks the CSR and the sources on the
 * device (one read of row_offsets, col_indices and sources, two short host
 * waits) before it traverses.  Calls share the array: calls that overlap on
 * the GPU race and must be serialised by the caller; a call that fails after
 * queuing work waits for that work before it returns.  stats may be NULL. */
#define XB_NOALLOC_MAX_VERTICES 131072
xb_status xb_traverse_noalloc(int64_t n, const int32_t* row_offsets, const int32_t* col_indices,
                              const int32_t* sources, int32_t k, int32_t* level, int32_t* parent,
                              void* stream, xb_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* XBTRAV_H */
