// xb_sssp.cu -- multi-source single-shortest-path distances on a weighted
// resident graph (xb_graph_set_weights, xb_multi_sssp).
//
// Same semantics as Ligra's MultiSSSP, the weighted multi-source app of the
// reference's baselines (apps/ligra/apps/MultiSSSP.C): one shared float
// distance array, every source at 0, rounds that relax the edges of the
// vertices whose distance dropped in the previous round (SSSP_F: write-min on
// the distance, then a claim of the vertex for the next frontier; Reset_F
// clears the claims), unreached vertices at FLT_MAX / 4, and every distance
// at -FLT_MAX / 4 when the frontier is still alive after n rounds.  The
// result -- the minimum over paths of the path's float sum from a source --
// does not depend on the order of the relaxations, so it is bit-exact
// against the reference.
//
// Device layout: distances as order-preserving int32 images of the floats
// (atomicMin on them is a float min for every sign), claim flags, two
// frontier lists, and the per-round edge partition of the frontier: an
// exclusive scan of the frontier's degrees (eoff) and, per chunk of kChunk
// consecutive frontier edges, the frontier index that owns the chunk's first
// edge (chunk_first).  Each round relaxes the frontier's edges in equal
// chunks, whatever the degrees -- a hub's adjacency is spread over many
// blocks -- with a plain read of the target's distance before the atomic.
#include <cfloat>

#include "xb_engine_common.cuh"
#include "xb_partition.cuh"

using xbi::fail;

namespace {

using xbp::kChunk;
using xbp::kItems;
using xbp::kThreads;
using xbp::kTile;
constexpr int kRelaxWarps = 4;                // warps per relax block
constexpr int kAppCap = 2 * kChunk;           // per-warp buffer of new frontier vertices
__device__ __forceinline__ int32_t float_key(float f) {
  const int32_t b = __float_as_int(f);
  return b >= 0 ? b : (b ^ 0x7FFFFFFF);
}

__device__ __forceinline__ float key_float(int32_t k) { return __int_as_float(k >= 0 ? k : (k ^ 0x7FFFFFFF)); }

template <typename OffT>
__global__ void k_sssp_init(const OffT* __restrict__ ro, int32_t* dkey, int32_t* claim, int64_t n) {
  const int32_t inf = float_key(FLT_MAX / 4);
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    dkey[v] = inf;
    claim[v] = ro[v + 1] > ro[v] ? 0 : 2;
  }
}

// Sources (distinct) get distance 0; those with edges form the first
// frontier, the others are only counted (*zero): a frontier vertex without
// edges relaxes nothing but still keeps the round loop alive, as in the
// reference's frontier.
template <typename OffT>
__global__ void k_sssp_sources(const int32_t* src, int32_t k, const OffT* ro, int32_t* dkey, int32_t* list,
                               int32_t* count, int32_t* zero) {
  for (int32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < k; q += gridDim.x * blockDim.x) {
    const int32_t s = src[q];
    dkey[s] = 0;
    if (ro[s + 1] > ro[s]) list[atomicAdd(count, 1)] = s;
    else atomicAdd(zero, 1);
  }
}

// One round: the frontier's edges in chunks of kChunk, one chunk per warp
// iteration; in step `it` lane l takes chunk edge 32 * it + l, so the
// column-index and weight reads of a warp are consecutive.  The owner of an
// edge is found from a bitmask of the edges where a spanned vertex starts
// (popcount of the bits up to the edge).  Warps run independently (tables
// and append buffer per warp, no block barrier).  Every frontier vertex has
// at least one edge, so a chunk spans at most kChunk + 1 of them.  claim[v]:
// 0 free, 1 already in the next frontier, 2 the vertex has no edges.  New
// frontier vertices gather in the warp's buffer and go out with one atomic
// per flush.
template <typename OffT>
__global__ void __launch_bounds__(32 * kRelaxWarps, 10) k_sssp_relax(
    const int32_t* __restrict__ list, const int32_t* __restrict__ count, const int64_t* __restrict__ eoff,
    const int64_t* __restrict__ ebase, const int32_t* __restrict__ chunk_first, const int64_t* __restrict__ edges_p,
    const int64_t* __restrict__ nchunks_p, const int32_t* __restrict__ ci, const int32_t* __restrict__ w,
    int32_t* dkey, int32_t* claim, int32_t* next, int32_t* next_count, int32_t* next_zero) {
  // spanned vertex: column-index position minus eoff (fits OffT: both lie in [0, m])
  __shared__ OffT s_base_all[kRelaxWarps][kChunk + 1];
  __shared__ float s_du_all[kRelaxWarps][kChunk + 1];      // spanned vertex: its distance
  __shared__ uint32_t s_mask_all[kRelaxWarps][kItems];     // bit e: a spanned vertex starts at chunk edge e
  __shared__ int32_t s_app_all[kRelaxWarps][kAppCap];      // vertices for the next frontier
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  OffT* s_base = s_base_all[wib];
  float* s_du = s_du_all[wib];
  uint32_t* s_mask = s_mask_all[wib];
  int32_t* s_app = s_app_all[wib];
  const uint32_t le_mask = (2u << lane) - 1u;  // lanes 0..lane
  const int32_t cnt = *count;
  const int64_t E = *edges_p, nchunks = *nchunks_p;
  const int64_t gw = (int64_t)blockIdx.x * kRelaxWarps + wib, nw = (int64_t)gridDim.x * kRelaxWarps;
  int32_t napp = 0;  // warp-uniform
  for (int64_t c = gw; c < nchunks; c += nw) {
    const int64_t E0 = c * kChunk;
    const int32_t len = (int32_t)min((int64_t)kChunk, E - E0);
    const int32_t vlo = chunk_first[c];
    const int32_t vhi = c + 1 < nchunks ? chunk_first[c + 1] : cnt - 1;
    const int32_t nv = vhi - vlo + 1;
    __syncwarp();  // the previous chunk is done with the tables
    if (lane < kItems) s_mask[lane] = 0u;
    __syncwarp();
    int32_t rel0 = 0;
    for (int32_t j = lane; j < nv; j += 32) {
      const int32_t u = list[vlo + j];
      const int64_t rel = __ldcs(&eoff[vlo + j]) - E0;
      s_base[j] = (OffT)__ldcs(&ebase[vlo + j]);
      s_du[j] = key_float(__ldcg(&dkey[u]));
      if (j == 0) rel0 = (int32_t)max(rel, (int64_t)-1);
      if (rel >= 0 && rel < kChunk) atomicOr(&s_mask[rel >> 5], 1u << (rel & 31));
    }
    __syncwarp();
    // owner of chunk edge e: (starts at or before e) - 1, plus one if vertex 0 began before the chunk
    int32_t run = (__shfl_sync(0xffffffffu, rel0, 0) < 0 ? 1 : 0) - 1;
    int64_t idx[kItems];
    float du[kItems];
#pragma unroll
    for (int it = 0; it < kItems; it++) {
      const uint32_t m = s_mask[it];
      const int32_t e = 32 * it + lane;
      const int32_t j = run + __popc(m & le_mask);
      run += __popc(m);
      idx[it] = -1;
      du[it] = 0.f;
      if (e < len) {
        idx[it] = (int64_t)s_base[j] + E0 + e;
        du[it] = s_du[j];
      }
    }
    int32_t v[kItems], key[kItems], cur[kItems];
#pragma unroll
    for (int it = 0; it < kItems; it++) {
      v[it] = idx[it] >= 0 ? __ldcs(&ci[idx[it]]) : 0;
      key[it] = idx[it] >= 0 ? __ldcs(&w[idx[it]]) : 0;
    }
#pragma unroll
    for (int it = 0; it < kItems; it++) {
      key[it] = float_key(du[it] + (float)key[it]);
      cur[it] = idx[it] >= 0 ? __ldcg(&dkey[v[it]]) : INT32_MIN;
    }
#pragma unroll
    for (int it = 0; it < kItems; it++) {
      bool add = false;
      // distances only fall: a stale read can only send an extra atomic
      if (key[it] < cur[it] && key[it] < atomicMin(&dkey[v[it]], key[it])) {
        const int32_t old = atomicCAS(&claim[v[it]], 0, 1);
        add = old == 0;
        if (old == 2) atomicAdd(next_zero, 1);
      }
      const unsigned bal = __ballot_sync(0xffffffffu, add);
      if (add) s_app[napp + __popc(bal & (le_mask >> 1))] = v[it];
      napp += __popc(bal);
    }
    if (napp > kAppCap - kChunk || c + nw >= nchunks) {  // room for one more chunk, or the warp's last chunk
      __syncwarp();
      int32_t base = 0;
      if (lane == 0 && napp) base = atomicAdd(next_count, napp);
      base = __shfl_sync(0xffffffffu, base, 0);
      for (int32_t i = lane; i < napp; i += 32) next[base + i] = s_app[i];
      napp = 0;
    }
  }
}

__global__ void k_sssp_unclaim(const int32_t* __restrict__ list, const int32_t* __restrict__ count, int32_t* claim) {
  const int32_t cnt = *count;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x)
    claim[list[i]] = 0;
}

__global__ void k_sssp_out(const int32_t* __restrict__ dkey, int64_t n, float* dist, int negative) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
    dist[v] = negative ? -FLT_MAX / 4 : key_float(dkey[v]);
}

struct SsspWork {
  int32_t *dkey, *claim, *list[2], *cnt;  // cnt[0], cnt[1]: list lengths; cnt[2]: edgeless vertices that improved
  int64_t *eoff, *ebase, *tsum, *scal;    // scal: edges, chunks
  int32_t* chunk_first;
  unsigned long long* relaxed;
};

// Workspace for n vertices, m edges and k sources, in int64 units.
int64_t sssp_work_words(int64_t n, int64_t m, int64_t k) {
  const int64_t i32 = 4 * n + k + 4 + (m / kChunk + 2);  // dkey, claim, lists, sources, counters, chunk_first
  return (i32 + 1) / 2 + 2 * n + (n / kTile + 2) + 4;    // + eoff, ebase, tile sums, scalars / relaxed
}

SsspWork carve(void* ws, int64_t n, int64_t m, int32_t k, int32_t** d_src) {
  SsspWork wk;
  int64_t* q = (int64_t*)ws;
  wk.eoff = q;
  q += n;
  wk.ebase = q;
  q += n;
  wk.tsum = q;
  q += n / kTile + 2;
  wk.scal = q;
  wk.relaxed = (unsigned long long*)(q + 2);
  q += 4;
  int32_t* p = (int32_t*)q;
  wk.dkey = p;
  wk.claim = p + n;
  wk.list[0] = p + 2 * n;
  wk.list[1] = p + 3 * n;
  *d_src = p + 4 * n;
  wk.cnt = *d_src + k;
  wk.chunk_first = wk.cnt + 4;
  return wk;
}

template <typename OffT>
xb_status run_sssp(xb_ctx* c, xb_graph* g, const int32_t* d_src, int32_t k, float* dist, bool out_dev,
                   const SsspWork& wk, int32_t* h_cnt /* 4 pinned ints */, xb_stats* st) {
  cudaStream_t s = c->stream;
  const int64_t n = g->n;
  const int sms = c->num_sms;
  const OffT* ro = (const OffT*)g->d_ro;
  const int vgrid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8));
  XB_CUDA(cudaMemsetAsync(wk.cnt, 0, 4 * sizeof(int32_t), s));
  XB_CUDA(cudaMemsetAsync(wk.relaxed, 0, sizeof(unsigned long long), s));
  k_sssp_init<OffT><<<vgrid, 256, 0, s>>>(ro, wk.dkey, wk.claim, n);
  k_sssp_sources<OffT><<<(k + 255) / 256, 256, 0, s>>>(d_src, k, ro, wk.dkey, wk.list[0], wk.cnt, wk.cnt + 2);
  XB_LAUNCH_CHECK("sssp init");
  XB_CUDA(cudaMemcpyAsync(h_cnt, wk.cnt, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  XB_CUDA(cudaStreamSynchronize(s));
  int32_t fcount = h_cnt[0], zero = h_cnt[2];
  int64_t rounds = 0;
  int cur = 0, negative = 0;
  // classes: 0 = relax rounds, 1 = frontier partition (scan, offsets, unclaim), 2 = init and output
  xbe::ClassTimer timer{c, st, c->tuning.timing != 0};
  if (st) st->class_launches[2] += 2;
  int relax_per_sm = 0;  // resident blocks of 4 warps (about 20 KB of tables each)
  XB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&relax_per_sm, k_sssp_relax<OffT>, 32 * kRelaxWarps, 0));
  const int relax_grid = sms * std::max(relax_per_sm, 1);
  while (fcount > 0 || zero > 0) {
    if (rounds == n) {  // still changing after n rounds: a negative cycle
      negative = 1;
      break;
    }
    rounds++;
    if (fcount == 0) break;  // only edgeless vertices: this round relaxes nothing
    const int32_t ntiles = (fcount + kTile - 1) / kTile;
    XB_CUDA(cudaMemsetAsync(wk.cnt + (cur ^ 1), 0, sizeof(int32_t), s));
    XB_CUDA(cudaMemsetAsync(wk.cnt + 2, 0, sizeof(int32_t), s));
    timer.begin();
    if (ntiles == 1) {
      xbp::k_lb_single<OffT><<<1, kThreads, 0, s>>>(wk.list[cur], wk.cnt + cur, ro, wk.eoff, wk.ebase, wk.chunk_first,
                                                    wk.scal, wk.scal + 1, wk.relaxed);
      timer.end(1, 1);
    } else {
      xbp::k_lb_tile_sums<OffT><<<ntiles, kThreads, 0, s>>>(wk.list[cur], wk.cnt + cur, ro, wk.tsum);
      xbp::k_lb_tile_scan<<<1, 1024, 0, s>>>(wk.tsum, wk.cnt + cur, wk.scal, wk.scal + 1, wk.relaxed);
      xbp::k_lb_offsets<OffT><<<ntiles, kThreads, 0, s>>>(wk.list[cur], wk.cnt + cur, ro, wk.tsum, wk.eoff, wk.ebase,
                                                          wk.chunk_first);
      timer.end(1, 3);
    }
    timer.begin();
    k_sssp_relax<OffT><<<relax_grid, 32 * kRelaxWarps, 0, s>>>(wk.list[cur], wk.cnt + cur, wk.eoff, wk.ebase,
                                                               wk.chunk_first, wk.scal, wk.scal + 1, g->d_ci,
                                                               g->d_w, wk.dkey, wk.claim, wk.list[cur ^ 1],
                                                               wk.cnt + (cur ^ 1), wk.cnt + 2);
    timer.end(0, 1);
    k_sssp_unclaim<<<vgrid, 256, 0, s>>>(wk.list[cur ^ 1], wk.cnt + (cur ^ 1), wk.claim);
    XB_LAUNCH_CHECK("sssp round");
    if (st) st->class_launches[1] += 1;
    XB_CUDA(cudaMemcpyAsync(h_cnt, wk.cnt, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    XB_CUDA(cudaStreamSynchronize(s));
    cur ^= 1;
    fcount = h_cnt[cur];
    zero = h_cnt[2];
  }
  float* out = dist;
  if (!out_dev) out = (float*)c->d_stage;  // sized by the caller
  k_sssp_out<<<vgrid, 256, 0, s>>>(wk.dkey, n, out, negative);
  XB_LAUNCH_CHECK("sssp out");
  if (st) st->class_launches[2] += 1;
  if (!out_dev) XB_CUDA(cudaMemcpyAsync(dist, out, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, s));
  unsigned long long relaxed = 0;
  XB_CUDA(cudaMemcpyAsync(&relaxed, wk.relaxed, sizeof(relaxed), cudaMemcpyDeviceToHost, s));
  XB_CUDA(cudaStreamSynchronize(s));
  if (st) {
    st->edges_scanned = (int64_t)relaxed;
    st->levels = (int32_t)rounds;
    // algorithmic bytes of the relax rounds: a column index and a weight per relaxation
    // (the distance array is read at random but stays in L2 up to about 2^24 vertices)
    st->class_bytes[0] = (int64_t)relaxed * 8;
    st->algo_bytes = st->class_bytes[0];
  }
  return XB_OK;
}

}  // namespace

extern "C" {

xb_status xb_graph_set_weights(xb_graph* g, const int32_t* weights, int64_t m) {
  xbi::clear_error();
  if (!g || (m > 0 && !weights)) return fail(XB_ERR_ARG, "null argument");
  if (m != g->m) return fail(XB_ERR_ARG, "weights must have one entry per column index");
  if (!g->ctx) return fail(XB_ERR_STATE, "the graph's context was destroyed");
  XB_CUDA(cudaSetDevice(g->ctx->device));
  if (g->d_w) cudaFree(g->d_w);
  g->d_w = nullptr;
  if (cudaMalloc(&g->d_w, sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1)) != cudaSuccess) {
    cudaGetLastError();
    return fail(XB_ERR_OOM, "weight allocation failed");
  }
  if (m > 0) XB_CUDA(cudaMemcpy(g->d_w, weights, sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice));
  return XB_OK;
}

xb_status xb_multi_sssp(xb_ctx* c, const xb_graph* gc, const int32_t* sources, int32_t k, float* dist,
                        uint32_t flags, xb_stats* st) {
  xbi::clear_error();
  xb_graph* g = const_cast<xb_graph*>(gc);
  if (!c || !g || !dist) return fail(XB_ERR_ARG, "null argument");
  if (!g->ctx) return fail(XB_ERR_STATE, "the graph's context was destroyed");
  if (g->ctx->device != c->device) return fail(XB_ERR_ARG, "graph lives on another device");
  if (!g->d_w && g->m > 0) return fail(XB_ERR_STATE, "the graph has no weights (xb_graph_set_weights)");
  if (k < 1 || !sources) return fail(XB_ERR_ARG, "at least one source is needed");
  if (st) std::memset(st, 0, sizeof(*st));
  XB_CUDA(cudaSetDevice(c->device));
  std::vector<int32_t> hs((size_t)k);
  if (flags & XB_SOURCES_DEVICE) {
    XB_CUDA(cudaMemcpy(hs.data(), sources, sizeof(int32_t) * k, cudaMemcpyDeviceToHost));
  } else {
    std::memcpy(hs.data(), sources, sizeof(int32_t) * k);
  }
  for (int32_t i = 0; i < k; i++)
    if (hs[(size_t)i] < 0 || hs[(size_t)i] >= g->n) return fail(XB_ERR_ARG, "source " + std::to_string(i) + " out of range");
  std::sort(hs.begin(), hs.end());  // the first frontier holds each source once
  hs.erase(std::unique(hs.begin(), hs.end()), hs.end());
  const int32_t kd = (int32_t)hs.size();
  const int64_t n = g->n;
  const size_t bytes = sizeof(int64_t) * (size_t)sssp_work_words(n, g->m, kd);
  {
    const xb_status ws = xbe::ensure_scratch(c, bytes, "SSSP");
    if (ws != XB_OK) return ws;
  }
  const bool out_dev = (flags & XB_OUT_DEVICE) != 0;
  if (!out_dev) {
    if (c->stage_bytes < sizeof(float) * (size_t)n) {
      if (c->d_stage) cudaFree(c->d_stage);
      c->d_stage = nullptr;
      c->stage_bytes = 0;
      if (cudaMalloc(&c->d_stage, sizeof(float) * (size_t)n) != cudaSuccess) {
        cudaGetLastError();
        return fail(XB_ERR_OOM, "SSSP staging allocation failed");
      }
      c->stage_bytes = sizeof(float) * (size_t)n;
    }
  }
  int32_t* d_src = nullptr;
  const SsspWork wk = carve(c->ws, n, g->m, kd, &d_src);
  XB_CUDA(cudaMemcpyAsync(d_src, hs.data(), sizeof(int32_t) * kd, cudaMemcpyHostToDevice, c->stream));
  XB_CUDA(cudaEventRecord(c->ev0, c->stream));
  // four pinned ints of host scratch: the counters of the first level record
  static_assert(sizeof(xbk::LevelCtr) >= 4 * sizeof(int32_t), "pinned scratch too small");
  int32_t* h4 = reinterpret_cast<int32_t*>(&c->h_ctr->lv[0]);
  xb_status s = g->off64 ? run_sssp<int64_t>(c, g, d_src, kd, dist, out_dev, wk, h4, st)
                         : run_sssp<int32_t>(c, g, d_src, kd, dist, out_dev, wk, h4, st);
  if (s != XB_OK) {
    cudaStreamSynchronize(c->stream);
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
