// xb_internal.h -- definitions shared by the host part (xb_host.cpp) and the
// device part (xb_engine.cu) of libxbtrav.so.  Not part of the public ABI.
#pragma once

#include <cstdint>
#include <string>
#include <thread>
#include <vector>

#include "xbtrav.h"

struct xb_host_csr {
  int64_t n = 0;
  std::vector<int64_t> ro;  // n+1
  std::vector<int32_t> ci;  // ro[n]
};

namespace xbi {

// Records msg as the calling thread's last error and returns s.
xb_status fail(xb_status s, const std::string& msg);
void clear_error();

int default_threads();

// Runs fn(t, nthreads) on nthreads host threads (t = 0..nthreads-1).
template <class F>
void parallel_run(int nthreads, F fn) {
  if (nthreads <= 1) {
    fn(0, 1);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(nthreads);
  for (int t = 0; t < nthreads; t++) pool.emplace_back([&fn, t, nthreads] { fn(t, nthreads); });
  for (auto& th : pool) th.join();
}

// Counter-based splitmix64 (Steele, Lea, Flood 2014): state advances by the
// golden gamma, output is the mix13 finaliser.
inline uint64_t splitmix64_next(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// Validates a CSR: offsets start at 0, non-decreasing, ids in [0, n).
xb_status validate_csr(int64_t n, const int64_t* ro, const int32_t* ci);

// Builds a symmetric, self-loop-free, duplicate-free CSR with ascending
// adjacency from pairs (u, v) packed as (u << 32) | v.
void csr_from_pairs(int64_t n, const std::vector<uint64_t>& pairs, int threads, xb_host_csr* out);

// Source selection over vertices of non-zero degree (host).
xb_status select_sources(int64_t n, const int64_t* ro, uint64_t seed, int32_t k, int32_t* out);

}  // namespace xbi
