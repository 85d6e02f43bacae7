// xb_host.cpp -- host side of libxbtrav.so: status strings and thread-local
// errors, seeded synthetic graph generators, the reference CSR text format,
// CSR validation and seeded source selection.  No CUDA here; every function
// in this file works on a machine without a GPU.
//
// Reference counterparts (X-Blossom project paths):
//   text CSR reader   ReadFileIntoHVector apps/xb/src/include/common/utils_cpu.h:9-23,
//                     HGraph(row, col) apps/xb/src/include/graph/hgraph.h:37-48
//                     (nedges = |col|/2: the CSR holds both directions)
//   source sets       exposed-vertex roots xblossom_gpu_engine_10.cu:119-144; the
//                     experiments sample sources from the non-trivial part of
//                     the graph (scripts/2-datasets/src_nodes/generate_src_lists.py);
//                     here: uniform without replacement over vertices of
//                     non-zero degree, seeded (the reference's sampler is unseeded).
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <unordered_map>

#include "xb_internal.h"

namespace xbi {

static thread_local std::string g_last_error;

xb_status fail(xb_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}
void clear_error() { g_last_error.clear(); }

int default_threads() {
  unsigned h = std::thread::hardware_concurrency();
  return h == 0 ? 1 : (int)h;
}

xb_status validate_csr(int64_t n, const int64_t* ro, const int32_t* ci) {
  if (n < 0) return fail(XB_ERR_ARG, "negative vertex count");
  if (n > INT32_MAX) return fail(XB_ERR_ARG, "vertex ids must fit int32");
  if (!ro) return fail(XB_ERR_ARG, "null row offsets");
  if (ro[0] != 0) return fail(XB_ERR_ARG, "row_offsets[0] must be 0");
  for (int64_t v = 0; v < n; v++)
    if (ro[v + 1] < ro[v]) return fail(XB_ERR_ARG, "row offsets decrease at vertex " + std::to_string(v));
  const int64_t m = ro[n];
  if (m > 0 && !ci) return fail(XB_ERR_ARG, "null column indices");
  for (int64_t e = 0; e < m; e++)
    if (ci[e] < 0 || (int64_t)ci[e] >= n)
      return fail(XB_ERR_ARG, "column index out of range at entry " + std::to_string(e));
  return XB_OK;
}

// Builds a symmetric, self-loop-free, duplicate-free CSR with ascending
// adjacency from a list of sampled pairs (u, v) packed as (u << 32) | v.
void csr_from_pairs(int64_t n, const std::vector<uint64_t>& pairs, int threads, xb_host_csr* out) {
  const int64_t np = (int64_t)pairs.size();
  std::vector<int64_t> deg(n + 1, 0);
  {
    std::unique_ptr<std::atomic<int64_t>[]> adeg(new std::atomic<int64_t>[n]);
    for (int64_t v = 0; v < n; v++) adeg[v].store(0, std::memory_order_relaxed);
    parallel_run(threads, [&](int t, int nt) {
      int64_t b = np * t / nt, e = np * (t + 1) / nt;
      for (int64_t i = b; i < e; i++) {
        uint32_t u = (uint32_t)(pairs[i] >> 32), v = (uint32_t)pairs[i];
        if (u == v) continue;
        adeg[u].fetch_add(1, std::memory_order_relaxed);
        adeg[v].fetch_add(1, std::memory_order_relaxed);
      }
    });
    for (int64_t v = 0; v < n; v++) deg[v] = adeg[v].load(std::memory_order_relaxed);
  }
  std::vector<int64_t> off(n + 1, 0);
  for (int64_t v = 0; v < n; v++) off[v + 1] = off[v] + deg[v];
  const int64_t mraw = off[n];
  std::vector<int32_t> tmp((size_t)std::max<int64_t>(mraw, 1));
  {
    std::unique_ptr<std::atomic<int64_t>[]> pos(new std::atomic<int64_t>[n]);
    for (int64_t v = 0; v < n; v++) pos[v].store(off[v], std::memory_order_relaxed);
    parallel_run(threads, [&](int t, int nt) {
      int64_t b = np * t / nt, e = np * (t + 1) / nt;
      for (int64_t i = b; i < e; i++) {
        uint32_t u = (uint32_t)(pairs[i] >> 32), v = (uint32_t)pairs[i];
        if (u == v) continue;
        tmp[pos[u].fetch_add(1, std::memory_order_relaxed)] = (int32_t)v;
        tmp[pos[v].fetch_add(1, std::memory_order_relaxed)] = (int32_t)u;
      }
    });
  }
  // sort + unique each adjacency list; dynamic chunks balance the hubs
  std::vector<int64_t> udeg(n, 0);
  {
    std::atomic<int64_t> next{0};
    const int64_t chunk = 256;
    parallel_run(threads, [&](int, int) {
      for (;;) {
        int64_t b = next.fetch_add(chunk);
        if (b >= n) break;
        int64_t e = std::min(n, b + chunk);
        for (int64_t v = b; v < e; v++) {
          int32_t* s = tmp.data() + off[v];
          int32_t* t2 = tmp.data() + off[v + 1];
          std::sort(s, t2);
          udeg[v] = std::unique(s, t2) - s;
        }
      }
    });
  }
  out->n = n;
  out->ro.assign(n + 1, 0);
  for (int64_t v = 0; v < n; v++) out->ro[v + 1] = out->ro[v] + udeg[v];
  out->ci.resize((size_t)out->ro[n]);
  parallel_run(threads, [&](int t, int nt) {
    int64_t b = n * t / nt, e = n * (t + 1) / nt;
    for (int64_t v = b; v < e; v++)
      std::memcpy(out->ci.data() + out->ro[v], tmp.data() + off[v], sizeof(int32_t) * udeg[v]);
  });
}

// Per-sample counter-based stream: sample i of a generator seeded by seed.
static inline uint64_t sample_state(uint64_t seed, uint64_t i) {
  uint64_t s = seed ^ 0x5851F42D4C957F2DULL;
  uint64_t h = splitmix64_next(s);
  uint64_t s2 = h + i * 0xD1342543DE82EF95ULL;
  return splitmix64_next(s2);
}

static inline double unit_double(uint64_t x) { return (double)(x >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace xbi

using namespace xbi;

extern "C" {

const char* xb_status_str(xb_status s) {
  switch (s) {
    case XB_OK: return "ok";
    case XB_ERR_ARG: return "invalid argument";
    case XB_ERR_OOM: return "out of memory";
    case XB_ERR_CAPACITY: return "capacity exceeded";
    case XB_ERR_TIMEOUT: return "device wait timed out";
    case XB_ERR_CUDA: return "CUDA error";
    case XB_ERR_IO: return "I/O error";
    case XB_ERR_NODEV: return "no CUDA device";
    case XB_ERR_STATE: return "invalid state";
    default: return "unknown status";
  }
}

const char* xb_last_error(void) { return g_last_error.c_str(); }

int32_t xb_abi_version(void) { return XB_ABI_VERSION; }

xb_status xb_csr_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                          uint64_t seed, int32_t threads, xb_host_csr** out) {
  clear_error();
  if (!out) return fail(XB_ERR_ARG, "null out");
  if (scale < 1 || scale > 30) return fail(XB_ERR_ARG, "scale must be in [1, 30]");
  if (edge_factor < 1 || edge_factor > 1024) return fail(XB_ERR_ARG, "edge_factor must be in [1, 1024]");
  if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0))
    return fail(XB_ERR_ARG, "R-MAT probabilities must be non-negative and sum to <= 1");
  const int64_t n = (int64_t)1 << scale;
  const int64_t ns = n * (int64_t)edge_factor;
  if (threads <= 0) threads = default_threads();
  std::vector<uint64_t> pairs;
  try {
    pairs.resize((size_t)ns);
  } catch (...) {
    return fail(XB_ERR_OOM, "host allocation of R-MAT samples failed");
  }
  const double ab = a + b, abc = a + b + c;
  parallel_run(threads, [&](int t, int nt) {
    int64_t lo = ns * t / nt, hi = ns * (t + 1) / nt;
    for (int64_t i = lo; i < hi; i++) {
      uint64_t s = sample_state(seed, (uint64_t)i);
      uint32_t u = 0, v = 0;
      for (int l = 0; l < scale; l++) {
        double r = unit_double(splitmix64_next(s));
        uint32_t bit = 1u << (scale - 1 - l);
        if (r < a) {
        } else if (r < ab) {
          v |= bit;
        } else if (r < abc) {
          u |= bit;
        } else {
          u |= bit;
          v |= bit;
        }
      }
      pairs[i] = ((uint64_t)u << 32) | v;
    }
  });
  std::unique_ptr<xb_host_csr> g(new xb_host_csr());
  try {
    csr_from_pairs(n, pairs, threads, g.get());
  } catch (...) {
    return fail(XB_ERR_OOM, "host allocation while building the CSR failed");
  }
  *out = g.release();
  return XB_OK;
}

xb_status xb_csr_gen_er(int64_t n, int64_t m_pairs, uint64_t seed, int32_t threads,
                        xb_host_csr** out) {
  clear_error();
  if (!out) return fail(XB_ERR_ARG, "null out");
  if (n < 1 || n > INT32_MAX) return fail(XB_ERR_ARG, "n must be in [1, 2^31)");
  if (m_pairs < 0) return fail(XB_ERR_ARG, "negative pair count");
  if (threads <= 0) threads = default_threads();
  std::vector<uint64_t> pairs;
  try {
    pairs.resize((size_t)m_pairs);
  } catch (...) {
    return fail(XB_ERR_OOM, "host allocation of samples failed");
  }
  parallel_run(threads, [&](int t, int nt) {
    int64_t lo = m_pairs * t / nt, hi = m_pairs * (t + 1) / nt;
    for (int64_t i = lo; i < hi; i++) {
      uint64_t s = sample_state(seed, (uint64_t)i);
      uint64_t u = splitmix64_next(s) % (uint64_t)n;
      uint64_t v = splitmix64_next(s) % (uint64_t)n;
      pairs[i] = (u << 32) | v;
    }
  });
  std::unique_ptr<xb_host_csr> g(new xb_host_csr());
  try {
    csr_from_pairs(n, pairs, threads, g.get());
  } catch (...) {
    return fail(XB_ERR_OOM, "host allocation while building the CSR failed");
  }
  *out = g.release();
  return XB_OK;
}

xb_status xb_csr_from_arrays(int64_t n, const int64_t* row_offsets, const int32_t* col_indices,
                             xb_host_csr** out) {
  clear_error();
  if (!out) return fail(XB_ERR_ARG, "null out");
  xb_status st = validate_csr(n, row_offsets, col_indices);
  if (st != XB_OK) return st;
  std::unique_ptr<xb_host_csr> g(new xb_host_csr());
  g->n = n;
  g->ro.assign(row_offsets, row_offsets + n + 1);
  g->ci.assign(col_indices, col_indices + row_offsets[n]);
  *out = g.release();
  return XB_OK;
}

// Reads whitespace-separated integers (the reference writes one per line).
static xb_status read_ints(const char* path, std::vector<int64_t>& vals) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(XB_ERR_IO, std::string("cannot open ") + path + ": " + std::strerror(errno));
  std::fseek(f, 0, SEEK_END);
  long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  std::string buf;
  buf.resize(sz > 0 ? (size_t)sz : 0);
  if (sz > 0 && std::fread(&buf[0], 1, (size_t)sz, f) != (size_t)sz) {
    std::fclose(f);
    return fail(XB_ERR_IO, std::string("short read on ") + path);
  }
  std::fclose(f);
  const char* p = buf.data();
  const char* e = p + buf.size();
  while (p < e) {
    while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) p++;
    if (p >= e) break;
    bool neg = false;
    if (*p == '-') {
      neg = true;
      p++;
    }
    if (p >= e || *p < '0' || *p > '9') return fail(XB_ERR_IO, std::string("non-integer token in ") + path);
    int64_t v = 0;
    while (p < e && *p >= '0' && *p <= '9') v = v * 10 + (*p++ - '0');
    vals.push_back(neg ? -v : v);
  }
  return XB_OK;
}

xb_status xb_csr_load_text(const char* row_path, const char* col_path, xb_host_csr** out) {
  clear_error();
  if (!row_path || !col_path || !out) return fail(XB_ERR_ARG, "null argument");
  std::vector<int64_t> ro, ci;
  xb_status st = read_ints(row_path, ro);
  if (st != XB_OK) return st;
  st = read_ints(col_path, ci);
  if (st != XB_OK) return st;
  if (ro.empty()) return fail(XB_ERR_IO, "row offsets file is empty");
  const int64_t n = (int64_t)ro.size() - 1;
  if (ro[n] != (int64_t)ci.size())
    return fail(XB_ERR_IO, "last row offset does not match the number of column indices");
  std::unique_ptr<xb_host_csr> g(new xb_host_csr());
  g->n = n;
  g->ro = std::move(ro);
  g->ci.resize(ci.size());
  for (size_t i = 0; i < ci.size(); i++) {
    if (ci[i] < 0 || ci[i] > INT32_MAX) return fail(XB_ERR_IO, "column index out of int32 range");
    g->ci[i] = (int32_t)ci[i];
  }
  st = validate_csr(n, g->ro.data(), g->ci.data());
  if (st != XB_OK) return st;
  *out = g.release();
  return XB_OK;
}

xb_status xb_csr_save_text(const xb_host_csr* g, const char* row_path, const char* col_path) {
  clear_error();
  if (!g || !row_path || !col_path) return fail(XB_ERR_ARG, "null argument");
  FILE* f = std::fopen(row_path, "wb");
  if (!f) return fail(XB_ERR_IO, std::string("cannot create ") + row_path);
  for (int64_t v : g->ro) std::fprintf(f, "%lld\n", (long long)v);
  std::fclose(f);
  f = std::fopen(col_path, "wb");
  if (!f) return fail(XB_ERR_IO, std::string("cannot create ") + col_path);
  for (int32_t v : g->ci) std::fprintf(f, "%d\n", v);
  std::fclose(f);
  return XB_OK;
}

xb_status xb_csr_info(const xb_host_csr* g, int64_t* n, int64_t* m, int64_t* max_degree,
                      int64_t* isolated) {
  clear_error();
  if (!g) return fail(XB_ERR_ARG, "null graph");
  if (n) *n = g->n;
  if (m) *m = g->ro[g->n];
  int64_t md = 0, iso = 0;
  for (int64_t v = 0; v < g->n; v++) {
    int64_t d = g->ro[v + 1] - g->ro[v];
    md = std::max(md, d);
    iso += d == 0;
  }
  if (max_degree) *max_degree = md;
  if (isolated) *isolated = iso;
  return XB_OK;
}

xb_status xb_csr_arrays(const xb_host_csr* g, const int64_t** row_offsets,
                        const int32_t** col_indices) {
  clear_error();
  if (!g) return fail(XB_ERR_ARG, "null graph");
  if (row_offsets) *row_offsets = g->ro.data();
  if (col_indices) *col_indices = g->ci.data();
  return XB_OK;
}

void xb_csr_free(xb_host_csr* g) { delete g; }

xb_status xb_select_sources_csr(int64_t n, const int64_t* row_offsets, uint64_t seed, int32_t k,
                                int32_t* out) {
  clear_error();
  return xbi::select_sources(n, row_offsets, seed, k, out);
}

}  // extern "C"

namespace xbi {

xb_status select_sources(int64_t n, const int64_t* ro, uint64_t seed, int32_t k, int32_t* out) {
  if (n < 0 || !ro || k < 0 || (k > 0 && !out)) return fail(XB_ERR_ARG, "bad source-selection argument");
  std::vector<int32_t> cand;
  cand.reserve((size_t)n);
  for (int64_t v = 0; v < n; v++)
    if (ro[v + 1] > ro[v]) cand.push_back((int32_t)v);
  const int64_t cnt = (int64_t)cand.size();
  if (k > cnt)
    return fail(XB_ERR_ARG, "asked for " + std::to_string(k) + " sources but only " +
                                std::to_string(cnt) + " vertices have edges");
  // partial Fisher-Yates over the candidate list
  uint64_t s = seed;
  for (int32_t i = 0; i < k; i++) {
    uint64_t r = splitmix64_next(s);
    int64_t j = i + (int64_t)(r % (uint64_t)(cnt - i));
    std::swap(cand[i], cand[j]);
    out[i] = cand[i];
  }
  return XB_OK;
}

}  // namespace xbi
