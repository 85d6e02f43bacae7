/*
 * msbfs_oracle.c -- CPU oracle for the multi-source traversal path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference legs
 * load it.  The product (libxbtrav.so) never links or calls it.
 *
 * What it restates (reference paths are relative to the X-Blossom project):
 *
 *  - Plain multi-source BFS.  One independent breadth-first search per source
 *    over an undirected CSR graph, producing an int32 level table and an int32
 *    parent table per source (k x n, source-major).
 *      * level[s][v]  = hop distance from source s, -1 if unreached.
 *      * parent[s][s] = s: the root convention of
 *        apps/ligra/apps/BFS.C:47 (Parents[start] = start) and of the
 *        reference's root initialisation apps/xb/src/xblsm_gpu/xblossom_gpu_engine_10.cu:119-144.
 *      * parent rule ORACLE_RULE_MINID: parent[s][v] = the smallest vertex id u
 *        adjacent to v with level[s][u] == level[s][v]-1.  This is the
 *        deterministic rule the GPU engine implements.  The reference's own
 *        parents (Ligra CAS, apps/ligra/apps/BFS.C:33-35; XB-Pro CAS claims,
 *        apps/xb/src/xblsm_cpu/par_pro_pernode.cu:203-215) are first-writer-wins
 *        and schedule dependent, so every one of them is merely *a* valid
 *        predecessor at level-1; the min-id rule picks one of those.
 *      * parent rule ORACLE_RULE_FIFO: the first discoverer in a FIFO queue
 *        whose neighbours are visited in CSR order.  This is the rule of the
 *        reference's only deterministic BFS with predecessors,
 *        xblossom::Graph::findShortestPath, apps/xb/src/include/graph/xgraph.h:155-191
 *        (adjacency built in CSR order by buildAdjListFromCSR, xgraph.h:347-356).
 *  - The work unit: edges traversed = sum over sources of sum over reached
 *    vertices of deg(v), the "Processed Edges" count of
 *    apps/ligra/apps/BFS_Throughput.C:42-63,77 and
 *    apps/xb/runner/xblsm_gpu/run_xb_pp_by_dataset.cu:117,152.
 *  - Work split over host threads: the chunked fetch_add idiom of the
 *    reference CPU engine (apps/xb/src/xblsm_cpu/par_pro_pernode.cu:111-118),
 *    here over sources instead of frontier vertices.
 *
 * Parity pinning: the level rule and the FIFO parent rule are checked against
 * the reference's own code (xgraph.h findShortestPath and Ligra BFS_F/edgeMap,
 * compiled from the reference sources by oracle/Makefile into oracle/_ref/)
 * through the fixtures in tests/golden/.
 */
#include <float.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <stdatomic.h>

#define ORACLE_RULE_MINID 0
#define ORACLE_RULE_FIFO 1

typedef struct {
    int64_t n;
    const int64_t *ro;
    const int32_t *ci;
    const int32_t *src;
    int32_t k;
    int32_t rule;
    int32_t *level;   /* k*n or NULL */
    int32_t *parent;  /* k*n or NULL */
    atomic_long next; /* next source index to claim */
    atomic_llong edges;
    atomic_llong reached;
    int chunk;
} job_t;

/* One BFS from s.  lvl/par are the rows for this source (n entries). */
static void bfs_one(const job_t *j, int32_t s, int32_t *lvl, int32_t *par,
                    int32_t *queue, long long *edges_out, long long *reached_out) {
    const int64_t n = j->n;
    for (int64_t v = 0; v < n; v++) { lvl[v] = -1; par[v] = -1; }
    int64_t head = 0, tail = 0;
    queue[tail++] = s;
    lvl[s] = 0;
    par[s] = s;
    long long edges = 0;
    while (head < tail) {
        int32_t u = queue[head++];
        int64_t b = j->ro[u], e = j->ro[u + 1];
        edges += (long long)(e - b);
        for (int64_t p = b; p < e; p++) {
            int32_t w = j->ci[p];
            if (lvl[w] < 0) {
                lvl[w] = lvl[u] + 1;
                par[w] = u; /* FIFO first discoverer */
                queue[tail++] = w;
            }
        }
    }
    if (j->rule == ORACLE_RULE_MINID) {
        /* parent = smallest adjacent id one level up */
        for (int64_t q = 0; q < tail; q++) {
            int32_t v = queue[q];
            if (v == s) continue;
            int32_t best = -1;
            for (int64_t p = j->ro[v]; p < j->ro[v + 1]; p++) {
                int32_t u = j->ci[p];
                if (lvl[u] == lvl[v] - 1 && (best < 0 || u < best)) best = u;
            }
            par[v] = best;
        }
    }
    *edges_out = edges;
    *reached_out = tail;
}

static void *worker(void *arg) {
    job_t *j = (job_t *)arg;
    int32_t *queue = (int32_t *)malloc(sizeof(int32_t) * (size_t)(j->n > 0 ? j->n : 1));
    int32_t *lvl_tmp = NULL, *par_tmp = NULL;
    if (!j->level) lvl_tmp = (int32_t *)malloc(sizeof(int32_t) * (size_t)(j->n > 0 ? j->n : 1));
    if (!j->parent) par_tmp = (int32_t *)malloc(sizeof(int32_t) * (size_t)(j->n > 0 ? j->n : 1));
    for (;;) {
        long b = atomic_fetch_add(&j->next, j->chunk);
        if (b >= j->k) break;
        long e = b + j->chunk < j->k ? b + j->chunk : j->k;
        for (long i = b; i < e; i++) {
            int32_t *lvl = j->level ? j->level + (size_t)i * (size_t)j->n : lvl_tmp;
            int32_t *par = j->parent ? j->parent + (size_t)i * (size_t)j->n : par_tmp;
            long long ed = 0, rc = 0;
            bfs_one(j, j->src[i], lvl, par, queue, &ed, &rc);
            atomic_fetch_add(&j->edges, ed);
            atomic_fetch_add(&j->reached, rc);
        }
    }
    free(queue);
    free(lvl_tmp);
    free(par_tmp);
    return NULL;
}

/*
 * Plain multi-source BFS.  Returns 0 on success, -1 on a bad argument.
 * level/parent may be NULL (then the search runs but the table is dropped,
 * used by the timed CPU baseline).  edges_traversed/reached may be NULL.
 */
int oracle_msbfs(int64_t n, const int64_t *row_offsets, const int32_t *col_indices,
                 const int32_t *sources, int32_t k, int32_t rule,
                 int32_t *level, int32_t *parent,
                 long long *edges_traversed, long long *reached, int32_t threads) {
    if (n < 0 || k < 0 || (k > 0 && (!sources || !row_offsets))) return -1;
    if (rule != ORACLE_RULE_MINID && rule != ORACLE_RULE_FIFO) return -1;
    for (int32_t i = 0; i < k; i++)
        if (sources[i] < 0 || sources[i] >= n) return -1;
    job_t j;
    memset(&j, 0, sizeof(j));
    j.n = n; j.ro = row_offsets; j.ci = col_indices; j.src = sources; j.k = k;
    j.rule = rule; j.level = level; j.parent = parent;
    atomic_init(&j.next, 0);
    atomic_init(&j.edges, 0);
    atomic_init(&j.reached, 0);
    j.chunk = 1;
    if (threads < 1) threads = 1;
    if (threads > k) threads = k > 0 ? k : 1;
    if (threads == 1) {
        worker(&j);
    } else {
        pthread_t *tid = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)threads);
        for (int t = 0; t < threads; t++) pthread_create(&tid[t], NULL, worker, &j);
        for (int t = 0; t < threads; t++) pthread_join(tid[t], NULL);
        free(tid);
    }
    if (edges_traversed) *edges_traversed = atomic_load(&j.edges);
    if (reached) *reached = atomic_load(&j.reached);
    return 0;
}

/*
 * Checks that parent[] (one source row) is a valid BFS predecessor table for
 * level[] (same row): parent[s]==s at level 0, every other reached v has an
 * edge (parent[v], v) with level[parent[v]] == level[v]-1, unreached vertices
 * carry -1.  Returns the number of violations.  This is the acceptance rule
 * for schedule-dependent reference parents (Ligra CAS, XB-Pro claims).
 */
long long oracle_check_parents(int64_t n, const int64_t *ro, const int32_t *ci,
                               int32_t s, const int32_t *level, const int32_t *parent) {
    long long bad = 0;
    for (int64_t v = 0; v < n; v++) {
        int32_t L = level[v], p = parent[v];
        if (L < 0) { if (p != -1) bad++; continue; }
        if (v == s) { if (L != 0 || p != s) bad++; continue; }
        if (p < 0 || p >= n || level[p] != L - 1) { bad++; continue; }
        int found = 0;
        for (int64_t q = ro[v]; q < ro[v + 1]; q++)
            if (ci[q] == p) { found = 1; break; }
        if (!found) bad++;
    }
    return bad;
}

/* Multi-source single-shortest-path distances (one shared distance array,
 * every source at distance 0), restating Ligra's MultiSSSP
 * (apps/ligra/apps/MultiSSSP.C: SSSP_F, Reset_F and the round loop of
 * Compute): rounds of relaxation of the frontier's edges with float
 * distances dist[v] = min(dist[v], dist[u] + (float)w); a vertex whose
 * distance dropped joins the next frontier; unreached vertices keep
 * FLT_MAX / 4; if the frontier is still non-empty after n rounds (a negative
 * cycle; in an undirected graph any negative edge) every distance becomes
 * -FLT_MAX / 4.  Sequential; the fixed point -- the minimum over paths of the
 * path's float sum taken from the source -- does not depend on the order.
 * Returns 0, or -1 on a bad argument. */
int oracle_msssp(int64_t n, const int64_t *row_offsets, const int32_t *col_indices, const int32_t *weights,
                 const int32_t *sources, int32_t k, float *dist) {
  if (n <= 0 || k <= 0 || !dist || !row_offsets) return -1;
  for (int32_t q = 0; q < k; q++)
    if (sources[q] < 0 || sources[q] >= n) return -1;
  const float inf = FLT_MAX / 4;
  int32_t *cur = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  int32_t *nxt = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  char *in_next = (char *)calloc((size_t)n, 1);
  if (!cur || !nxt || !in_next) {
    free(cur);
    free(nxt);
    free(in_next);
    return -1;
  }
  for (int64_t v = 0; v < n; v++) dist[v] = inf;
  int64_t nc = 0;
  for (int32_t q = 0; q < k; q++)
    if (dist[sources[q]] != 0.0f) {
      dist[sources[q]] = 0.0f;
      cur[nc++] = sources[q];
    }
  int64_t round = 0;
  while (nc > 0) {
    if (round == n) {
      for (int64_t v = 0; v < n; v++) dist[v] = -inf;
      break;
    }
    int64_t nn = 0;
    for (int64_t i = 0; i < nc; i++) {
      const int32_t u = cur[i];
      for (int64_t e = row_offsets[u]; e < row_offsets[u + 1]; e++) {
        const int32_t v = col_indices[e];
        const float nd = dist[u] + (float)weights[e];
        if (nd < dist[v]) {
          dist[v] = nd;
          if (!in_next[v]) {
            in_next[v] = 1;
            nxt[nn++] = v;
          }
        }
      }
    }
    for (int64_t i = 0; i < nn; i++) in_next[nxt[i]] = 0;
    int32_t *t = cur;
    cur = nxt;
    nxt = t;
    nc = nn;
    round++;
  }
  free(cur);
  free(nxt);
  free(in_next);
  return 0;
}

/* Maximum-cardinality matching in a general graph: Edmonds' blossom
 * algorithm (J. Edmonds, "Paths, trees, and flowers", Canad. J. Math. 17,
 * 1965), restated as the checker of the matching path.  The reference's
 * engines (apps/xb/src/xblsm_cpu/par_pro_pernode.cu:42-90, the GPU engine
 * apps/xb/src/xblsm_gpu/xblossom_gpu_engine_10.cu:72-80) compute a maximum
 * matching of the same graph; matchings are not unique, so the checks are
 * validity and size.
 *
 * One alternating tree per exposed root, grown breadth first; a blossom is
 * an edge between two outer vertices of the tree, contracted by pointing the
 * base of every vertex on its cycle to the cycle's top and making its inner
 * vertices outer; `pred` is rerouted along the cycle so an augmenting path
 * can be read back through blossoms.  Exposed roots are tried once each: an
 * exposed vertex without an augmenting path keeps none after augmentations
 * elsewhere.  mate: n ints in/out (-1 exposed).  Returns the matching size
 * or -1 on a bad argument. */
struct mm_state {
  int64_t n;
  const int64_t *ro;
  const int32_t *ci;
  int32_t *mate, *base, *pred, *queue, *stamp;
  char *outer, *cyc;
  int32_t tick;
};

static int32_t mm_top(struct mm_state *S, int32_t a, int32_t b) {
  S->tick++;
  for (;;) { /* up from a to the root, stamping the bases */
    a = S->base[a];
    S->stamp[a] = S->tick;
    if (S->mate[a] < 0) break;
    a = S->pred[S->mate[a]];
  }
  for (;;) { /* up from b to the first stamped base */
    b = S->base[b];
    if (S->stamp[b] == S->tick) return b;
    b = S->pred[S->mate[b]];
  }
}

static void mm_cycle_side(struct mm_state *S, int32_t v, int32_t top, int32_t across) {
  while (S->base[v] != top) {
    const int32_t m = S->mate[v];
    S->cyc[S->base[v]] = 1;
    S->cyc[S->base[m]] = 1;
    S->pred[v] = across;  /* leave v through the cycle edge instead */
    across = m;
    v = S->pred[m];
  }
}

static int32_t mm_search(struct mm_state *S, int32_t root) {
  const int64_t n = S->n;
  for (int64_t v = 0; v < n; v++) {
    S->base[v] = (int32_t)v;
    S->pred[v] = -1;
    S->outer[v] = 0;
  }
  int64_t qh = 0, qt = 0;
  S->outer[root] = 1;
  S->queue[qt++] = root;
  while (qh < qt) {
    const int32_t v = S->queue[qh++];
    for (int64_t e = S->ro[v]; e < S->ro[v + 1]; e++) {
      const int32_t w = S->ci[e];
      if (S->base[v] == S->base[w] || S->mate[v] == w) continue;
      const int w_outer = w == root || (S->mate[w] >= 0 && S->pred[S->mate[w]] >= 0);
      if (w_outer) {
        const int32_t top = mm_top(S, v, w);
        memset(S->cyc, 0, (size_t)n);
        mm_cycle_side(S, v, top, w);
        mm_cycle_side(S, w, top, v);
        for (int64_t x = 0; x < n; x++) {
          if (!S->cyc[S->base[x]]) continue;
          S->base[x] = top;
          if (!S->outer[x]) {
            S->outer[x] = 1;
            S->queue[qt++] = (int32_t)x;
          }
        }
      } else if (S->pred[w] < 0) {
        S->pred[w] = v;
        if (S->mate[w] < 0) return w;
        S->outer[S->mate[w]] = 1;
        S->queue[qt++] = S->mate[w];
      }
    }
  }
  return -1;
}

int64_t oracle_max_match(int64_t n, const int64_t *row_offsets, const int32_t *col_indices, int32_t *mate) {
  if (n <= 0 || n > INT32_MAX || !row_offsets || !mate) return -1;
  for (int64_t v = 0; v < n; v++) {
    const int32_t m = mate[v];
    if (m < -1 || m >= n || (m >= 0 && mate[m] != v)) return -1;
  }
  struct mm_state S;
  S.n = n;
  S.ro = row_offsets;
  S.ci = col_indices;
  S.mate = mate;
  S.base = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  S.pred = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  S.queue = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  S.stamp = (int32_t *)calloc((size_t)n, sizeof(int32_t));
  S.outer = (char *)malloc((size_t)n);
  S.cyc = (char *)malloc((size_t)n);
  S.tick = 0;
  if (!S.base || !S.pred || !S.queue || !S.stamp || !S.outer || !S.cyc) {
    free(S.base); free(S.pred); free(S.queue); free(S.stamp); free(S.outer); free(S.cyc);
    return -1;
  }
  for (int64_t r = 0; r < n; r++) {
    if (mate[r] >= 0) continue;
    int32_t u = mm_search(&S, (int32_t)r);
    while (u >= 0) { /* flip the path from u back to r */
      const int32_t p = S.pred[u], next = mate[p];
      mate[u] = p;
      mate[p] = u;
      u = next;
    }
  }
  int64_t size = 0;
  for (int64_t v = 0; v < n; v++) size += mate[v] >= 0;
  free(S.base); free(S.pred); free(S.queue); free(S.stamp); free(S.outer); free(S.cyc);
  return size / 2;
}

/* Alternating forest of a matching (the expansion of the reference's
 * alternating mode, ExpandAlternatingForest in
 * apps/xb/src/xblsm_gpu/xblossom_gpu_engine_10.cu:270-359 and
 * ExpandTwoNodes in apps/xb/src/include/path_table/path_table.h:256-271),
 * grown level by level from every exposed vertex (mate -1), with a
 * deterministic rule where the reference's claims race:
 *   level 0: exposed vertices, parent = owner = itself;
 *   level 2d+1 (inner): an unlabeled matched vertex w next to an outer vertex
 *     of level 2d; parent = the smallest such neighbour, owner = its owner;
 *   level 2d+2 (outer): the mate of that inner vertex; parent = the inner.
 * When both ends of a matched pair qualify at the same level, the end whose
 * smallest outer neighbour is smaller (then the smaller id) is the inner
 * one.  Edges between outer vertices (augmenting paths, blossoms) do not
 * label anything.  Unreached vertices: -1 in all three arrays.  Returns the
 * number of expansion rounds, or -1 on a bad argument. */
int64_t oracle_alt_forest(int64_t n, const int64_t *row_offsets, const int32_t *col_indices, const int32_t *mate,
                          int32_t *level, int32_t *parent, int32_t *owner) {
  if (n <= 0 || n > INT32_MAX || !row_offsets || !mate || !level || !parent || !owner) return -1;
  int32_t *front = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  int32_t *next = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  int32_t *cand = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  int32_t *touched = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  if (!front || !next || !cand || !touched) {
    free(front); free(next); free(cand); free(touched);
    return -1;
  }
  int64_t nf = 0;
  for (int64_t v = 0; v < n; v++) {
    cand[v] = INT32_MAX;
    if (mate[v] < 0) {
      level[v] = 0;
      parent[v] = owner[v] = (int32_t)v;
      front[nf++] = (int32_t)v;
    } else {
      level[v] = parent[v] = owner[v] = -1;
    }
  }
  int64_t rounds = 0;
  for (int32_t d = 0; nf > 0; d++) {
    rounds++;
    int64_t nt = 0, nn = 0;
    for (int64_t i = 0; i < nf; i++) {
      const int32_t v = front[i];
      for (int64_t e = row_offsets[v]; e < row_offsets[v + 1]; e++) {
        const int32_t w = col_indices[e];
        if (level[w] != -1 || mate[w] < 0) continue;
        if (cand[w] == INT32_MAX) touched[nt++] = w;
        if (v < cand[w]) cand[w] = v;
      }
    }
    for (int64_t i = 0; i < nt; i++) {
      const int32_t w = touched[i], x = mate[w];
      const int32_t cw = cand[w], cx = cand[x];
      const int inner = cx == INT32_MAX || cw < cx || (cw == cx && w < x);
      if (!inner) continue;
      level[w] = 2 * d + 1;
      parent[w] = cw;
      owner[w] = owner[cw];
      level[x] = 2 * d + 2;
      parent[x] = w;
      owner[x] = owner[w];
      next[nn++] = x;
    }
    for (int64_t i = 0; i < nt; i++) cand[touched[i]] = INT32_MAX;
    int32_t *t = front;
    front = next;
    next = t;
    nf = nn;
  }
  free(front); free(next); free(cand); free(touched);
  return rounds;
}
