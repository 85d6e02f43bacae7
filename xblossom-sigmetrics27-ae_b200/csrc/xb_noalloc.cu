// xb_noalloc.cu -- xb_traverse_noalloc: the plain multi-source traversal for
// callers that must not allocate device memory.
//
// Who needs it: a host that owns all of the GPU's memory through its own pool
// (a plugin inside a database or analytics engine, a framework with a caching
// allocator that hands out every byte) may not call cudaMalloc behind that
// pool's back, and a latency-critical serving path may forbid cudaMalloc and
// cudaFree because they can synchronise the device and stall other streams.
// Such a caller already holds the graph, the sources and the output tables in
// memory it owns; this entry point takes only device pointers to those and
// keeps its own working state in one fixed array compiled into the library.
//
// The array (g_noalloc_scratch, about 32 MiB) lives in every GPU that loads
// the library until the process exits.  It bounds the graph to
// XB_NOALLOC_MAX_VERTICES vertices; larger graphs are rejected with
// XB_ERR_CAPACITY.  Every call on a device shares the one array and leaves
// its contents behind; each call clears what must start at zero before it
// uses it.  Calls whose work overlaps on the GPU (two host threads, or two
// streams, at once on the same device) race on the array and give wrong
// results: serialise them.
//
// The device address of the array is looked up once per device context, on
// the first call made with that device current (cudaGetSymbolAddress); make
// that first call before any stream capture begins on the device.  The
// address is cached under the context's unique id, so a host that resets the
// device (cudaDeviceReset) or otherwise replaces its context gets a fresh
// lookup on its next call instead of a pointer into the old context.
//
// No cudaMalloc, cudaFree, cudaMallocHost or allocating library routine is
// called here, on the host or the device.
#include <cuda.h>  // CUcontext and the prototypes of the two driver calls fetched below
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "xb_internal.h"
#include "xb_kernels.cuh"

using xbi::fail;

namespace {

constexpr int64_t kMaxN = XB_NOALLOC_MAX_VERTICES;  // 131072
constexpr int kPlanes = 17;                          // levels < kMaxN <= 2^17
constexpr size_t kW = (size_t)kMaxN;                 // 8-byte words per state array
// layout in 8-byte words
constexpr size_t kSeenOff = 0;
constexpr size_t kFOff = kSeenOff + kW;
constexpr size_t kNOff = kFOff + kW;
constexpr size_t kPlanesOff = kNOff + kW;
constexpr size_t kPushedOff = kPlanesOff + (size_t)kPlanes * kW;  // bits reached by push steps
constexpr size_t kP8Off = kPushedOff + kW;                        // 64 parent-index bytes per vertex
constexpr size_t kListsOff = kP8Off + 8 * kW;                     // 6 int32 lists of kMaxN
constexpr size_t kCtrOff = kListsOff + 3 * kW;
constexpr size_t kCtrWords = (sizeof(xbk::Ctrs) + 7) / 8;
constexpr size_t kMiscOff = kCtrOff + kCtrWords;  // int32 heavy count, int32 error flag
constexpr size_t kRowsOff = kMiscOff + 4;          // 2 x 64 row pointers of the table pass
constexpr size_t kTotalWords = kRowsOff + 128;

constexpr int kHeavy = 2048;
constexpr float kAlpha = 4.0f;
constexpr int kMaxDevices = 64;

}  // namespace

static __device__ __align__(256) unsigned long long g_noalloc_scratch[kTotalWords];

namespace {

std::mutex g_setup_mu;
struct ScratchSlot {
  unsigned long long ctx_id = 0;  // unique id of the context the address belongs to (0: none yet)
  unsigned long long* ptr = nullptr;
};
ScratchSlot g_scratch[kMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique id of the context current on the calling thread (0 when none is).
// The two driver calls are fetched through the runtime, so the library needs
// no link against libcuda.
xb_status current_context_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  if (!get_current || !get_id) {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = cudaDriverEntryPointSymbolNotFound;
    const cudaError_t e1 = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1);
    const cudaError_t e2 = cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2);
    if (e1 != cudaSuccess || e2 != cudaSuccess || q1 != cudaDriverEntryPointSuccess ||
        q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
      return fail(XB_ERR_CUDA, "driver entry points cuCtxGetCurrent / cuCtxGetId are unavailable");
    get_current = (CtxGetCurrentFn)f1;
    get_id = (CtxGetIdFn)f2;
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS) return fail(XB_ERR_CUDA, "cuCtxGetCurrent failed");
  *id = 0;
  if (ctx && get_id(ctx, id) != CUDA_SUCCESS) return fail(XB_ERR_CUDA, "cuCtxGetId failed");
  return XB_OK;
}

// Set-up: the array's device address in the current device's context, looked
// up with cudaGetSymbolAddress once per context and cached under its id.
xb_status scratch_for_current_device(unsigned long long** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(XB_ERR_NODEV, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(XB_ERR_ARG, "device index beyond the supported range");
  std::lock_guard<std::mutex> lock(g_setup_mu);
  unsigned long long id = 0;
  xb_status s = current_context_id(&id);
  if (s != XB_OK) return s;
  ScratchSlot& slot = g_scratch[dev];
  if (id == 0 || slot.ctx_id != id || !slot.ptr) {
    // cudaGetSymbolAddress makes the device's primary context current when
    // none is, so the id is read again after it
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(XB_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    s = current_context_id(&id);
    if (s != XB_OK) return s;
    slot.ctx_id = id;
    slot.ptr = (unsigned long long*)p;
  }
  *out = slot.ptr;
  return XB_OK;
}

// Checks the caller's CSR and sources on the device; sets *err on the first
// violation: 1 = offsets, 2 = column index, 3 = source id.
__global__ void k_validate(int64_t n, const int32_t* __restrict__ ro, const int32_t* __restrict__ ci,
                           const int32_t* __restrict__ src, int32_t k, int32_t* err) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t m = ro[n];
  if (tid == 0 && (ro[0] != 0 || m < 0)) atomicCAS(err, 0, 1);
  for (int64_t v = tid; v < n; v += stride)
    if (ro[v + 1] < ro[v]) atomicCAS(err, 0, 1);
  for (int64_t i = tid; i < (int64_t)k; i += stride)
    if (src[i] < 0 || src[i] >= n) atomicCAS(err, 0, 3);
  if (m < 0) return;
  for (int64_t e = tid; e < m; e += stride)
    if (ci[e] < 0 || ci[e] >= n) atomicCAS(err, 0, 2);
}

// Vertices of degree > thr, appended in any order (the kernels that read the
// list reduce per vertex, so the order does not matter).
__global__ void k_heavy_list(int64_t n, const int32_t* __restrict__ ro, int thr, int32_t* list, int32_t* count) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
    const int64_t v = base + threadIdx.x;
    const bool hv = v < n && ro[v + 1] - ro[v] > thr;
    xbk::warp_append(hv, (int32_t)v, list, count);
  }
}

// Error exits of the entry point once it may have queued work on the caller's
// stream: the stream is drained first (its result ignored), so no kernel or
// copy of this call is still using the shared array when the call returns.
xb_status drained(cudaStream_t sm, xb_status s) {
  cudaStreamSynchronize(sm);
  cudaGetLastError();
  return s;
}

#define NA_CUDA(call)                                                                                 \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess)                                                                            \
      return drained(sm, fail(XB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)));      \
  } while (0)

}  // namespace

extern "C" xb_status xb_traverse_noalloc(int64_t n, const int32_t* row_offsets, const int32_t* col_indices,
                                         const int32_t* sources, int32_t k, int32_t* level, int32_t* parent,
                                         void* stream_handle, xb_stats* st) {
  using W = unsigned long long;
  constexpr int B = 64;
  xbi::clear_error();
  if (st) std::memset(st, 0, sizeof(*st));
  if (n < 1) return fail(XB_ERR_ARG, "n must be at least 1");
  if (n > kMaxN)
    return fail(XB_ERR_CAPACITY, "graph has " + std::to_string(n) + " vertices; xb_traverse_noalloc holds at most " +
                                     std::to_string(kMaxN) + " (its scratch array is fixed at build time)");
  if (k < 0) return fail(XB_ERR_ARG, "negative source count");
  if (!row_offsets || (k > 0 && (!sources || !level || !parent)))
    return fail(XB_ERR_ARG, "null device pointer");
  if (k == 0) return XB_OK;
  cudaStream_t sm = (cudaStream_t)stream_handle;
  unsigned long long* scratch = nullptr;
  xb_status s = scratch_for_current_device(&scratch);
  if (s != XB_OK) return s;
  int dev = 0, sms = 148;
  NA_CUDA(cudaGetDevice(&dev));
  NA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));

  W* seen = scratch + kSeenOff;
  W* F = scratch + kFOff;
  W* N = scratch + kNOff;
  // planes 0-1 interleaved (2 words per vertex), planes 2.. separate
  const xbk::Planes<W, 1> pl{scratch + kPlanesOff, scratch + kPlanesOff + 2 * kW, (int64_t)kW};
  W* pushed = scratch + kPushedOff;
  W* ppos = scratch + kP8Off;  // 8 position planes per vertex
  int32_t* lists = (int32_t*)(scratch + kListsOff);
  xbk::Lists fl{lists + 0 * kW, lists + 1 * kW};
  xbk::Lists nl{lists + 2 * kW, lists + 3 * kW};
  int32_t* touched = lists + 4 * kW;
  int32_t* heavy_list = lists + 5 * kW;
  xbk::Ctrs* ctr = (xbk::Ctrs*)(scratch + kCtrOff);
  int32_t* misc = (int32_t*)(scratch + kMiscOff);  // [0] heavy count, [1] validation error
  int32_t** rows = (int32_t**)(scratch + kRowsOff);
  const size_t plane_bytes = sizeof(W) * kW;
  const size_t state_bytes = sizeof(W) * (size_t)n;

  // validate the caller's arrays on the device (a bad id would fault the kernels)
  int32_t m32 = 0;
  NA_CUDA(cudaMemcpyAsync(&m32, row_offsets + n, sizeof(int32_t), cudaMemcpyDeviceToHost, sm));
  NA_CUDA(cudaStreamSynchronize(sm));
  if (m32 < 0) return drained(sm, fail(XB_ERR_ARG, "row_offsets[n] is negative"));
  if (m32 > 0 && !col_indices) return drained(sm, fail(XB_ERR_ARG, "null column indices"));
  NA_CUDA(cudaMemsetAsync(misc, 0, 4 * sizeof(int32_t), sm));
  const int vgrid = sms * 4;
  k_validate<<<vgrid, 256, 0, sm>>>(n, row_offsets, col_indices, sources, k, misc + 1);
  NA_CUDA(cudaGetLastError());
  int32_t hmisc[2] = {0, 0};
  NA_CUDA(cudaMemcpyAsync(hmisc, misc, sizeof(hmisc), cudaMemcpyDeviceToHost, sm));
  NA_CUDA(cudaStreamSynchronize(sm));
  if (hmisc[1] == 1) return drained(sm, fail(XB_ERR_ARG, "row offsets must start at 0 and not decrease"));
  if (hmisc[1] == 2) return drained(sm, fail(XB_ERR_ARG, "a column index is out of range"));
  if (hmisc[1] == 3) return drained(sm, fail(XB_ERR_ARG, "a source id is out of range"));
  k_heavy_list<<<(int)std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8), 256, 0, sm>>>(n, row_offsets, kHeavy,
                                                                                        heavy_list, misc);
  NA_CUDA(cudaGetLastError());
  NA_CUDA(cudaMemcpyAsync(hmisc, misc, sizeof(int32_t), cudaMemcpyDeviceToHost, sm));
  NA_CUDA(cudaStreamSynchronize(sm));
  const int32_t n_heavy = hmisc[0];

  // F and N must start zero: the array keeps whatever the last call left
  NA_CUDA(cudaMemsetAsync(F, 0, state_bytes, sm));
  NA_CUDA(cudaMemsetAsync(N, 0, state_bytes, sm));

  const int64_t ntiles = (n + 31) / 32;
  constexpr int PULL_WARPS = 8, TAB_WARPS = 4, U = 4;
  constexpr int PUSH_CHUNK = 2048;
  const int pull_grid = (int)std::max<int64_t>(1, std::min<int64_t>((ntiles + PULL_WARPS - 1) / PULL_WARPS, (int64_t)sms * 8));
  const int tab_grid = (int)std::max<int64_t>(1, std::min<int64_t>((ntiles + TAB_WARPS - 1) / TAB_WARPS, (int64_t)sms * 16));
  xbk::Ctrs h{};
  int max_levels = 0;
  for (int64_t k0 = 0; k0 < k; k0 += B) {
    const int kb = (int)std::min<int64_t>(B, k - k0);
    xbk::Masks<W, 1> active{};
    active.w[0] = kb == 64 ? ~0ull : ((1ull << kb) - 1ull);
    NA_CUDA(cudaMemsetAsync(seen, 0, state_bytes, sm));
    NA_CUDA(cudaMemsetAsync(pl.p01, 0, 2 * plane_bytes, sm));
    NA_CUDA(cudaMemsetAsync(pl.ph, 0, plane_bytes, sm));
    NA_CUDA(cudaMemsetAsync(pushed, 0, state_bytes, sm));
    NA_CUDA(cudaMemsetAsync(ppos, 0, 8 * state_bytes, sm));
    xbk::k_pass_init<<<1, 1, 0, sm>>>(ctr, (long long)m32);
    xbk::k_init_batch<W, 1, int32_t><<<1, 256, 0, sm>>>(sources + k0, kb, row_offsets, F, seen, pl, active, kHeavy,
                                                         fl, ctr);
    NA_CUDA(cudaGetLastError());
    int cur = 0;
    for (;;) {
      // the device picks the step (push / pull / done); the host reads it back
      xbk::k_step_begin<<<1, 1, 0, sm>>>(ctr, cur, kAlpha, kPlanes, 1 << kPlanes, 0, 0);
      NA_CUDA(cudaMemcpyAsync(&h, ctr, sizeof(h), cudaMemcpyDeviceToHost, sm));
      NA_CUDA(cudaStreamSynchronize(sm));
      if (h.b.dir == 2) break;
      const xbk::LevelCtr lc = h.lv[cur];
      if (h.b.zero_plane >= 3)
        NA_CUDA(cudaMemsetAsync(pl.ph + (size_t)(h.b.zero_plane - 2) * kW, 0, plane_bytes, sm));
      if (h.b.dir == 0) {
        if (lc.n_light > 0)
          xbk::k_push_light<W, 1, int32_t><<<(int)std::min<int64_t>((lc.n_light + 7) / 8, (int64_t)sms * 16), 256, 0,
                                             sm>>>(fl.light, &ctr->lv[cur].n_light, row_offsets, col_indices, F, seen, N,
                                                   nullptr, touched, ctr, cur);
        if (lc.n_heavy > 0) {
          const dim3 hgrid((unsigned)std::max<int64_t>(1, std::min<int64_t>((n + PUSH_CHUNK - 1) / PUSH_CHUNK, 64)),
                           (unsigned)std::min<int64_t>(lc.n_heavy, 65535));
          xbk::k_push_heavy<W, 1, int32_t><<<hgrid, 256, 0, sm>>>(fl.heavy, &ctr->lv[cur].n_heavy, row_offsets,
                                                                  col_indices, F, seen, N, nullptr, touched, ctr, cur,
                                                                  PUSH_CHUNK);
          xbk::k_clear_list<W, 1><<<(int)std::min<int64_t>((lc.n_heavy + 255) / 256, (int64_t)sms * 8), 256, 0, sm>>>(
              fl.heavy, &ctr->lv[cur].n_heavy, F);
        }
        xbk::k_push_finalize<W, 1, int32_t><<<(int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8)),
                                              256, 0, sm>>>(touched, row_offsets, N, seen, pl, active, kHeavy, nl, ctr,
                                                            cur, pushed, nullptr, 0);
      } else {
        xbk::k_pull_tiles<W, 1, int32_t, PULL_WARPS, U><<<pull_grid, PULL_WARPS * 32, 0, sm>>>(
            n, row_offsets, col_indices, F, seen, N, pl, active, kHeavy, nl, ctr, cur, ppos);
        // one warp per heavy vertex; their parents are searched by the table pass
        if (n_heavy > 0) {
          // heavy vertices with wanted bits (listed into the push steps' touched list), then a warp per vertex
          xbk::k_heavy_want<W, 1, int32_t><<<(int)std::min<int64_t>((n_heavy + 255) / 256, (int64_t)sms * 4), 256, 0,
                                             sm>>>(heavy_list, n_heavy, row_offsets, seen, active, INT32_MAX, ctr, cur,
                                                   touched);
          xbk::k_pull_heavy<W, 1, int32_t, 4><<<(int)std::min<int64_t>((n_heavy + 7) / 8, (int64_t)sms * 16), 256, 0,
                                                sm>>>(heavy_list, touched, row_offsets, col_indices, F, seen, N, pl,
                                                      active, kHeavy, INT32_MAX, nl, ctr, cur, nullptr, n, nullptr);
        }
        // zero the consumed frontier: its listed vertices, or all of F when it is large
        xbk::k_clear_frontier<W, 1><<<(int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8)),
                                      256, 0, sm>>>(F, n, fl, ctr, cur);
      }
      NA_CUDA(cudaGetLastError());
      std::swap(F, N);
      std::swap(fl, nl);
      cur ^= 1;
    }
    if (h.b.err)
      return drained(sm, fail(XB_ERR_STATE, "the level loop ran past the level bound (corrupted traversal state)"));
    max_levels = std::max(max_levels, h.b.level);
    // every vertex takes the edge-flat table path here (no heavy-vertex staging)
    int32_t* hrows[2 * B];
    for (int j = 0; j < B; j++) {
      hrows[j] = j < kb ? level + (k0 + j) * n : nullptr;
      hrows[B + j] = j < kb ? parent + (k0 + j) * n : nullptr;
    }
    // pageable source: the copy has taken hrows by the time the call returns
    NA_CUDA(cudaMemcpyAsync(rows, hrows, sizeof(hrows), cudaMemcpyHostToDevice, sm));
    xbk::k_tables<W, 1, int32_t, TAB_WARPS, U><<<tab_grid, TAB_WARPS * 32, 0, sm>>>(
        n, row_offsets, col_indices, seen, pl, kb, INT32_MAX, rows, ctr, ppos, pushed, sources + k0, nullptr,
        nullptr);
    NA_CUDA(cudaGetLastError());
    NA_CUDA(cudaMemcpyAsync(&h, ctr, sizeof(h), cudaMemcpyDeviceToHost, sm));
    NA_CUDA(cudaStreamSynchronize(sm));
    if (st) {
      st->edges_traversed += (int64_t)h.b.edges_traversed;
      st->reached += (int64_t)h.b.reached;
      st->edges_scanned += (int64_t)h.b.edges_scanned;
      st->vertices_scanned += (int64_t)h.b.vertices_scanned;
      st->vertices_swept += (int64_t)h.b.vertices_swept;
      st->parent_edges_scanned += (int64_t)h.b.parent_edges;
      st->push_levels += h.b.push_levels;
      st->pull_levels += h.b.pull_levels;
      st->batches += 1;
    }
  }
  if (st) st->levels = max_levels;
  return XB_OK;
}
