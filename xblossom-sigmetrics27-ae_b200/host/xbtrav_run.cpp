// xbtrav_run.cpp -- command-line runner with the reference runners' flags.
//
// The reference's runners (apps/xb/runner/xblsm_gpu/run_xb_pp_by_dataset.cu,
// flags in apps/xb/src/flag/flag.cc) load a text CSR, run the engine
// --rounds times and print per-round and average runtimes plus work counters.
// This runner takes the same flags (gflags syntax: --name=value or
// --name value) and prints the same summary lines for the engine here:
//
//   --dataset=NAME          label only
//   --row_offsets=PATH      text CSR row offsets (one integer per line)
//   --col_indices=PATH      text CSR column indices
//   --rounds=N              timed repetitions after one untimed warm-up
//   --num_threads=N         accepted (the reference's CPU-engine thread count; unused here)
//   --path_buffer_ratio=N   accepted (sizes the reference GPU engine's path buffer; this
//                           engine sizes its buffers itself)
//   --max_cuda_sms=N        accepted (0 = default launch sizing, the only sizing here)
// and, for this library's other paths:
//   --mode=match|traverse|sssp   default match (FindMaximumMatch from the empty matching)
//   --rmat=SCALE:EF         generate the seeded R-MAT graph instead of reading files
//   --src_count=K --seed=S  sources for traverse / sssp (xb_select_sources)
//   --weight_max=W          sssp: seeded symmetric weights in [1, W]
//
// Average runtime drops the fastest and slowest round when there are three
// or more, as the reference's AvgRuntime does (apps/xb/src/include/common/timing_guard.h:43-70).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "xbtrav.hpp"

namespace {

struct Flags {
  std::map<std::string, std::string> kv;
  std::string get(const std::string& k, const std::string& dflt) const {
    auto it = kv.find(k);
    return it == kv.end() ? dflt : it->second;
  }
  long long num(const std::string& k, long long dflt) const {
    auto it = kv.find(k);
    return it == kv.end() ? dflt : std::strtoll(it->second.c_str(), nullptr, 0);
  }
};

bool parse(int argc, char** argv, Flags* f) {
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a.rfind("--", 0) != 0) return false;
    a = a.substr(2);
    const size_t eq = a.find('=');
    if (eq != std::string::npos) {
      f->kv[a.substr(0, eq)] = a.substr(eq + 1);
    } else if (i + 1 < argc && std::strncmp(argv[i + 1], "--", 2) != 0) {
      f->kv[a] = argv[++i];
    } else {
      f->kv[a] = "1";
    }
  }
  return true;
}

double avg_runtime(const std::vector<double>& t) {
  double total = 0, mn = t[0], mx = t[0];
  for (double x : t) {
    total += x;
    mn = std::min(mn, x);
    mx = std::max(mx, x);
  }
  size_t count = t.size();
  if (count >= 3) {
    total -= mn + mx;
    count -= 2;
  }
  return total / (double)count;
}

// Seeded weight of the unordered pair {a, b} in [1, wmax]: both directions of an edge agree.
int32_t pair_weight(int64_t a, int64_t b, int64_t seed, int64_t wmax) {
  const int64_t lo = std::min(a, b), hi = std::max(a, b);
  return (int32_t)((lo * 1000003 + hi * 7919 + seed) % wmax) + 1;
}

void usage(const char* prog) {
  std::fprintf(stderr,
               "usage: %s --row_offsets=PATH --col_indices=PATH | --rmat=SCALE:EF\n"
               "       [--mode=match|traverse|sssp] [--rounds=N] [--dataset=NAME]\n"
               "       [--src_count=K] [--seed=S] [--weight_max=W]\n"
               "       [--num_threads=N] [--path_buffer_ratio=N] [--max_cuda_sms=N]  (accepted, unused)\n",
               prog);
}

}  // namespace

int main(int argc, char** argv) {
  Flags f;
  if (!parse(argc, argv, &f) || f.kv.count("help")) {
    usage(argv[0]);
    return f.kv.count("help") ? 0 : 2;
  }
  try {
    const std::string mode = f.get("mode", "match");
    const std::string rmat = f.get("rmat", "");
    if (rmat.empty() && (f.get("row_offsets", "").empty() || f.get("col_indices", "").empty())) {
      usage(argv[0]);
      return 2;
    }
    if (mode != "match" && mode != "traverse" && mode != "sssp") {
      usage(argv[0]);
      return 2;
    }
    const long long rounds = std::max(1LL, f.num("rounds", 1));
    const std::string dataset = f.get("dataset", rmat.empty() ? "Amazon" : "rmat" + rmat);
    std::printf("Run xbtrav (%s) on Dataset %s\n", mode.c_str(), dataset.c_str());
    std::printf("Run xbtrav for %lld times\n", rounds);
    xbtrav::HGraph g = rmat.empty()
                           ? xbtrav::HGraph(f.get("row_offsets", ""), f.get("col_indices", ""))
                           : xbtrav::HGraph::Rmat(std::atoi(rmat.c_str()),
                                                  std::atoi(rmat.substr(rmat.find(':') + 1).c_str()), 0x5EED);
    xbtrav::Context ctx(0);
    xbtrav::DGraph dg(ctx, g);
    int64_t n = 0, m = 0, max_degree = 0;
    xbtrav::check(xb_graph_info(dg.get(), &n, &m, &max_degree));
    const int k = (int)f.num("src_count", 64);
    const uint64_t seed = (uint64_t)f.num("seed", 0x5EED + 1);
    std::vector<int32_t> sources;
    if (mode != "match") sources = g.SelectSources(seed, k);
    if (mode == "sssp") {
      const int64_t wmax = std::max(1LL, f.num("weight_max", 100));
      std::vector<int32_t> w((size_t)m);
      for (int64_t v = 0; v < n; v++)
        for (int64_t e = g.row_offsets[v]; e < g.row_offsets[v + 1]; e++)
          w[(size_t)e] = pair_weight(v, g.col_indices[e], (int64_t)seed, wmax);
      xbtrav::check(xb_graph_set_weights(const_cast<xb_graph*>(dg.get()), w.data(), m));
    }
    std::vector<double> times;
    double work = 0, levels = 0, phases = 0;
    size_t result = 0;
    std::vector<float> dist((size_t)(mode == "sssp" ? n : 0));
    xbtrav::Tables tables;
    for (long long r = -1; r < rounds; r++) {  // round -1: untimed warm-up
      xb_stats st{};
      const auto t0 = std::chrono::steady_clock::now();
      if (mode == "match") {
        const xbtrav::Matching mt = xbtrav::MaximumMatchingEngine(dg).FindMaximumMatch(&st);
        result = 0;
        for (size_t v = 0; v < mt.size(); v++) result += mt[v] != (int32_t)n;
        result /= 2;
      } else if (mode == "traverse") {
        tables = xbtrav::TraversalEngine(dg).Traverse(sources);
        st = tables.stats;
        result = (size_t)st.reached;
      } else {
        xbtrav::check(xb_multi_sssp(ctx.get(), dg.get(), sources.data(), k, dist.data(), 0u, &st));
        result = 0;
        for (float d : dist) result += d < 3.0e37f;
      }
      const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (r < 0) continue;
      times.push_back(secs);
      work += (double)(mode == "traverse" ? st.edges_traversed : st.edges_scanned);
      levels += st.levels;
      phases += st.batches;
      std::printf("Round runtime: %.6f\n", secs);
    }
    const double avg = avg_runtime(times);
    const double nedges = (double)m / 2.0;
    std::printf("Average runtime: %.6f\n", avg);
    std::printf("Num of Nodes: %lld\n", (long long)n);
    std::printf("Num of Edges: %.0f\n", nedges);
    if (mode == "match") {
      std::printf("Matching Size: %zu\n", result);
      std::printf("Number of Phases: %.1f\n", phases / (double)rounds);
    } else if (mode == "traverse") {
      std::printf("Sources: %d\n", k);
      std::printf("Reached (source, vertex) pairs: %zu\n", result);
    } else {
      std::printf("Sources: %d\n", k);
      std::printf("Reached Vertices: %zu\n", result);
    }
    std::printf("Number of Levels: %.1f\n", levels / (double)rounds);
    std::printf("Number of Processed Edges: %.0f\n", work / (double)rounds);
    std::printf("Max Degree: %lld\n", (long long)max_degree);
    std::printf("Avg Degree: %.6f\n", nedges / (double)n);
    std::printf("Processed Edges per Second: %.6e\n", work / (double)rounds / avg);
    return 0;
  } catch (const xbtrav::Error& e) {
    std::fprintf(stderr, "xbtrav error %d: %s\n", e.status, e.what());
    return 1;
  }
}
