// xb_formats.cpp -- on-disk formats of libxbtrav.so (host only, no GPU):
//   binary CSR       the native fast format: magic, n, m, int64 row offsets,
//                    int32 column indices (little-endian)
//   source lists     "#" comments (whole line or trailing), vertex ids
//                    separated by white space: the files of
//                    scripts/2-datasets/src_nodes/generate_src_lists.py, read
//                    by source_nodes_from_file in scripts/4-expr/common.sh
//   Ligra adjacency  "AdjacencyGraph", n, m, n offsets, m targets
//                    (the target of scripts/2-datasets/ligra/csr_to_ligra_adj.py)
//   Matrix Market    coordinate pattern symmetric, one 1-based (i < j) entry
//                    per undirected edge in ascending order (the entry lines of
//                    scripts/2-datasets/gunrock/csr_to_gunrock_mm.py)
#include <cctype>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "xb_internal.h"

using xbi::clear_error;
using xbi::fail;

namespace {

constexpr char kMagic[8] = {'X', 'B', 'C', 'S', 'R', '\0', '\1', '\0'};

struct File {
  FILE* f = nullptr;
  File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

// Reads one line (without the newline); false at end of file with nothing read.
bool read_line(FILE* f, std::string& line) {
  line.clear();
  int c;
  bool any = false;
  while ((c = std::fgetc(f)) != EOF) {
    any = true;
    if (c == '\n') break;
    line.push_back((char)c);
  }
  return any;
}

}  // namespace

extern "C" {

xb_status xb_csr_save_binary(const xb_host_csr* g, const char* path) {
  clear_error();
  if (!g || !path) return fail(XB_ERR_ARG, "null argument");
  File f(path, "wb");
  if (!f.f) return fail(XB_ERR_IO, std::string("cannot create ") + path);
  const int64_t n = g->n, m = g->ro[g->n];
  const bool ok = std::fwrite(kMagic, 1, 8, f.f) == 8 && std::fwrite(&n, 8, 1, f.f) == 1 &&
                  std::fwrite(&m, 8, 1, f.f) == 1 &&
                  std::fwrite(g->ro.data(), 8, (size_t)n + 1, f.f) == (size_t)n + 1 &&
                  (m == 0 || std::fwrite(g->ci.data(), 4, (size_t)m, f.f) == (size_t)m);
  if (!ok) return fail(XB_ERR_IO, std::string("write failed: ") + path);
  return XB_OK;
}

xb_status xb_csr_load_binary(const char* path, xb_host_csr** out) {
  clear_error();
  if (!path || !out) return fail(XB_ERR_ARG, "null argument");
  *out = nullptr;
  File f(path, "rb");
  if (!f.f) return fail(XB_ERR_IO, std::string("cannot open ") + path);
  char magic[8];
  int64_t n = 0, m = 0;
  if (std::fread(magic, 1, 8, f.f) != 8 || std::memcmp(magic, kMagic, 8) != 0)
    return fail(XB_ERR_IO, std::string("not a binary CSR file: ") + path);
  if (std::fread(&n, 8, 1, f.f) != 1 || std::fread(&m, 8, 1, f.f) != 1 || n < 0 || n >= INT32_MAX || m < 0)
    return fail(XB_ERR_IO, std::string("bad header: ") + path);
  std::unique_ptr<xb_host_csr> g(new xb_host_csr());
  g->n = n;
  g->ro.resize((size_t)n + 1);
  g->ci.resize((size_t)m);
  if (std::fread(g->ro.data(), 8, (size_t)n + 1, f.f) != (size_t)n + 1 ||
      (m > 0 && std::fread(g->ci.data(), 4, (size_t)m, f.f) != (size_t)m))
    return fail(XB_ERR_IO, std::string("truncated file: ") + path);
  if (g->ro[(size_t)n] != m) return fail(XB_ERR_IO, std::string("row offsets do not end at m: ") + path);
  xb_status s = xbi::validate_csr(n, g->ro.data(), g->ci.data());
  if (s != XB_OK) return s;
  *out = g.release();
  return XB_OK;
}

xb_status xb_sources_load(const char* path, int32_t* out, int32_t capacity, int32_t* count) {
  clear_error();
  if (!path || !count || capacity < 0 || (capacity > 0 && !out)) return fail(XB_ERR_ARG, "bad argument");
  *count = 0;
  File f(path, "rb");
  if (!f.f) return fail(XB_ERR_IO, std::string("cannot open ") + path);
  std::string line;
  int32_t k = 0;
  while (read_line(f.f, line)) {
    const size_t hash = line.find('#');
    if (hash != std::string::npos) line.resize(hash);
    size_t i = 0;
    while (i < line.size()) {
      while (i < line.size() && std::isspace((unsigned char)line[i])) i++;
      if (i >= line.size()) break;
      size_t j = i;
      while (j < line.size() && !std::isspace((unsigned char)line[j])) j++;
      const std::string tok = line.substr(i, j - i);
      char* end = nullptr;
      const long long v = std::strtoll(tok.c_str(), &end, 10);
      if (!end || *end != '\0' || v < 0 || v >= INT32_MAX)
        return fail(XB_ERR_IO, std::string("not a vertex id: '") + tok + "' in " + path);
      if (k < capacity) out[k] = (int32_t)v;
      k++;
      i = j;
    }
  }
  *count = k;
  if (k > capacity) return fail(XB_ERR_CAPACITY, "the file lists " + std::to_string(k) + " sources");
  return XB_OK;
}

xb_status xb_sources_save(const char* path, const int32_t* sources, int32_t k, const char* comment) {
  clear_error();
  if (!path || k < 0 || (k > 0 && !sources)) return fail(XB_ERR_ARG, "bad argument");
  File f(path, "wb");
  if (!f.f) return fail(XB_ERR_IO, std::string("cannot create ") + path);
  if (comment && *comment) {
    const std::string c(comment);
    size_t b = 0;
    while (b < c.size()) {  // one "# " line per line of the comment
      size_t e = c.find('\n', b);
      if (e == std::string::npos) e = c.size();
      std::fprintf(f.f, "# %s\n", c.substr(b, e - b).c_str());
      b = e + 1;
    }
  }
  for (int32_t i = 0; i < k; i++) std::fprintf(f.f, "%d\n", sources[i]);
  return XB_OK;
}

xb_status xb_csr_save_ligra(const xb_host_csr* g, const char* path) {
  clear_error();
  if (!g || !path) return fail(XB_ERR_ARG, "null argument");
  File f(path, "wb");
  if (!f.f) return fail(XB_ERR_IO, std::string("cannot create ") + path);
  std::fprintf(f.f, "AdjacencyGraph\n%lld\n%lld\n", (long long)g->n, (long long)g->ro[(size_t)g->n]);
  for (int64_t v = 0; v < g->n; v++) std::fprintf(f.f, "%lld\n", (long long)g->ro[(size_t)v]);
  for (int32_t w : g->ci) std::fprintf(f.f, "%d\n", w);
  return XB_OK;
}

xb_status xb_csr_save_mtx(const xb_host_csr* g, const char* path) {
  clear_error();
  if (!g || !path) return fail(XB_ERR_ARG, "null argument");
  int64_t entries = 0;
  for (int64_t v = 0; v < g->n; v++)
    for (int64_t e = g->ro[(size_t)v]; e < g->ro[(size_t)v + 1]; e++) entries += g->ci[(size_t)e] > v;
  File f(path, "wb");
  if (!f.f) return fail(XB_ERR_IO, std::string("cannot create ") + path);
  std::fprintf(f.f, "%%%%MatrixMarket matrix coordinate pattern symmetric\n");
  std::fprintf(f.f, "%% undirected graph, one (i < j) entry per edge, 1-based\n");
  std::fprintf(f.f, "%lld %lld %lld\n", (long long)g->n, (long long)g->n, (long long)entries);
  // rows ascending, each adjacency ascending: the (i, j) pairs come out sorted
  for (int64_t v = 0; v < g->n; v++)
    for (int64_t e = g->ro[(size_t)v]; e < g->ro[(size_t)v + 1]; e++)
      if (g->ci[(size_t)e] > v) std::fprintf(f.f, "%lld %d\n", (long long)v + 1, g->ci[(size_t)e] + 1);
  return XB_OK;
}

xb_status xb_csr_load_mtx(const char* path, xb_host_csr** out) {
  clear_error();
  if (!path || !out) return fail(XB_ERR_ARG, "null argument");
  *out = nullptr;
  File f(path, "rb");
  if (!f.f) return fail(XB_ERR_IO, std::string("cannot open ") + path);
  std::string line;
  if (!read_line(f.f, line) || line.compare(0, 14, "%%MatrixMarket") != 0)
    return fail(XB_ERR_IO, std::string("not a Matrix Market file: ") + path);
  for (auto& ch : line) ch = (char)std::tolower((unsigned char)ch);
  if (line.find("coordinate") == std::string::npos) return fail(XB_ERR_IO, "only coordinate Matrix Market files are read");
  long long rows = 0, cols = 0, nnz = 0;
  for (;;) {
    if (!read_line(f.f, line)) return fail(XB_ERR_IO, "missing size line");
    if (line.empty() || line[0] == '%') continue;
    if (std::sscanf(line.c_str(), "%lld %lld %lld", &rows, &cols, &nnz) != 3) return fail(XB_ERR_IO, "bad size line");
    break;
  }
  if (rows != cols || rows < 1 || rows >= INT32_MAX || nnz < 0) return fail(XB_ERR_IO, "need a square matrix");
  std::vector<uint64_t> pairs;
  pairs.reserve((size_t)nnz);
  for (long long i = 0; i < nnz;) {
    if (!read_line(f.f, line)) return fail(XB_ERR_IO, "truncated entries");
    if (line.empty() || line[0] == '%') continue;
    long long a = 0, b = 0;
    if (std::sscanf(line.c_str(), "%lld %lld", &a, &b) != 2) return fail(XB_ERR_IO, "bad entry line");
    if (a < 1 || a > rows || b < 1 || b > rows) return fail(XB_ERR_IO, "entry index out of range");
    pairs.push_back(((uint64_t)(a - 1) << 32) | (uint64_t)(b - 1));  // values, if any, are ignored
    i++;
  }
  std::unique_ptr<xb_host_csr> g(new xb_host_csr());
  xbi::csr_from_pairs((int64_t)rows, pairs, xbi::default_threads(), g.get());
  *out = g.release();
  return XB_OK;
}

}  // extern "C"
