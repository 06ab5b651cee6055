// gcl_dimacs.h -- the DIMACS graph reader shared by the file pipeline
// (gcl_files.cu) and the command-line front-end (host code, no CUDA).
//
// It reads what CSRGraph::fromDIMACS (CSRGraph.cpp:40-119) reads.  That
// function takes the file line by line with std::getline and extracts from
// each line with std::istringstream:
//   * an empty line or one whose first character is 'c' is skipped;
//   * the first non-blank character is the line type;
//   * 'p <word> <n> <m>' sets the vertex count (m is ignored);
//   * 'n <v> <colour>' colours vertex v (1-based; v = 0 or v > n ignored);
//   * 'e <u> <v>' adds an undirected edge (1-based), self loops dropped, both
//     directions stored; rows come out sorted;
//   * any other type is ignored.
// Numbers follow the stream extraction rules: blanks skipped, an optional
// sign, decimal digits up to the first non-digit; no digits stores 0 and an
// overflow the type's limit, and either stops the rest of the line, whose
// targets keep their values ('-k' read as unsigned wraps modulo 2^32).
//
// Where the reference has undefined behaviour this reader rejects the file:
// an edge endpoint of 0 or above the current n (the reference indexes out of
// bounds; also an endpoint that a later 'p' line puts out of range) and a
// repeated edge (the reference keeps the multi-edge, which its refinement
// does not support).  A vertex count above max_n is rejected too.
// The file is read in one piece and scanned in place, without a stream object
// per line.
#pragma once
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

namespace gcl {

struct DimacsGraph {
  int n = 0;
  std::vector<int32_t> rowptr;  // n + 1 offsets
  std::vector<int32_t> col;     // both directions, each row sorted
  std::vector<int32_t> color;   // n colours (0 where the file sets none)
  bool colored = false;         // some colour is nonzero
};

enum DimacsStatus : int {
  kDimacsOk = 0,
  kDimacsOpenFailed = 1,
  kDimacsBadEndpoint = 2,
  kDimacsDuplicateEdge = 3,
  kDimacsTooLarge = 4,
};

namespace dimacs_detail {

inline bool blank(char c) {
  return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f' || c == '\n';
}

// Extractions from one line with the rules of std::istringstream >> x.
struct LineReader {
  const char* p;
  const char* end;
  bool failed = false;

  // The stream sentry: skip blanks; at the end of the line the extraction
  // fails and leaves its target alone.
  bool sentry() {
    if (failed) return false;
    while (p < end && blank(*p)) ++p;
    if (p == end) {
      failed = true;
      return false;
    }
    return true;
  }
  void get_char(char* c) {
    if (sentry()) *c = *p++;
  }
  void skip_word() {
    if (sentry())
      while (p < end && !blank(*p)) ++p;
  }
  // Sign and digits; false when there were no digits or the magnitude passed `limit`.
  bool digits(uint64_t limit, bool* neg, uint64_t* mag) {
    *neg = false;
    *mag = 0;
    if (*p == '+' || *p == '-') *neg = *p++ == '-';
    bool any = false, over = false;
    while (p < end && *p >= '0' && *p <= '9') {
      any = true;
      if (!over) {
        *mag = *mag * 10 + (uint64_t)(*p - '0');
        over = *mag > limit;
      }
      ++p;
    }
    if (!any) return false;
    return !over;
  }
  void get_uint(unsigned* out) {
    if (!sentry()) return;
    bool neg;
    uint64_t mag;
    if (!digits(UINT_MAX, &neg, &mag)) {
      failed = true;
      *out = mag > UINT_MAX ? UINT_MAX : 0u;  // overflow, or no digits
      return;
    }
    *out = neg ? (unsigned)(0u - (unsigned)mag) : (unsigned)mag;
  }
  void get_int(int* out) {
    if (!sentry()) return;
    bool neg;
    uint64_t mag;
    if (!digits((uint64_t)INT_MAX + 1, &neg, &mag)) {
      failed = true;
      *out = mag == 0 ? 0 : (neg ? INT_MIN : INT_MAX);
      return;
    }
    if (!neg && mag > (uint64_t)INT_MAX) {
      failed = true;
      *out = INT_MAX;
      return;
    }
    *out = neg ? (int)(-(int64_t)mag) : (int)mag;
  }
};

}  // namespace dimacs_detail

// Parses DIMACS text (len bytes at text) into g.
inline int parse_dimacs_text(const char* text, size_t len, int64_t max_n, DimacsGraph* g) {
  using dimacs_detail::LineReader;
  unsigned n = 0;
  std::vector<std::pair<unsigned, unsigned>> edges;  // one entry per undirected edge
  std::vector<std::pair<unsigned, int>> colors;
  const char* end = text + len;
  for (const char* line = text; line < end;) {
    const char* nl = (const char*)std::memchr(line, '\n', (size_t)(end - line));
    const char* le = nl ? nl : end;
    const char* cur = line;
    line = nl ? nl + 1 : end;
    if (cur == le || *cur == 'c') continue;
    LineReader r{cur, le};
    char type = 0;
    r.get_char(&type);
    if (type == 'p') {
      unsigned m = 0;
      r.skip_word();
      r.get_uint(&n);
      r.get_uint(&m);
    } else if (type == 'n') {
      unsigned vid = 0;
      int c = 0;
      r.get_uint(&vid);
      r.get_int(&c);
      if (vid != 0) colors.emplace_back(vid - 1, c);
    } else if (type == 'e') {
      unsigned u = 0, v = 0;
      r.get_uint(&u);
      r.get_uint(&v);
      if (u == v) continue;
      if (u == 0 || v == 0 || u > n || v > n) return kDimacsBadEndpoint;
      edges.emplace_back(u - 1, v - 1);
    }
  }
  if ((int64_t)n > max_n) return kDimacsTooLarge;
  // a later 'p' line may have lowered n below an endpoint accepted earlier
  for (const auto& e : edges)
    if (e.first >= n || e.second >= n) return kDimacsBadEndpoint;
  // CSR by counting, then each row sorted: the layout of sorting the
  // (u, v) and (v, u) pairs together, which the reference does
  g->n = (int)n;
  g->rowptr.assign((size_t)n + 1, 0);
  for (const auto& e : edges) {
    g->rowptr[e.first + 1]++;
    g->rowptr[e.second + 1]++;
  }
  for (unsigned i = 0; i < n; ++i) g->rowptr[i + 1] += g->rowptr[i];
  g->col.resize(2 * edges.size());
  {
    std::vector<int32_t> fill(g->rowptr.begin(), g->rowptr.end() - (n ? 1 : 0));
    for (const auto& e : edges) {
      g->col[(size_t)fill[e.first]++] = (int32_t)e.second;
      g->col[(size_t)fill[e.second]++] = (int32_t)e.first;
    }
  }
  for (unsigned i = 0; i < n; ++i) {
    int32_t* b = g->col.data() + g->rowptr[i];
    int32_t* e = g->col.data() + g->rowptr[i + 1];
    std::sort(b, e);
    if (std::adjacent_find(b, e) != e) return kDimacsDuplicateEdge;
  }
  g->color.assign(n, 0);
  for (const auto& kv : colors)
    if (kv.first < n) g->color[kv.first] = kv.second;
  g->colored = std::any_of(g->color.begin(), g->color.end(), [](int32_t c) { return c != 0; });
  return kDimacsOk;
}

// Reads and parses the file at `path`.
inline int read_dimacs_file(const char* path, int64_t max_n, DimacsGraph* g) {
  std::FILE* f = std::fopen(path, "rb");
  if (!f) return kDimacsOpenFailed;
  std::string buf;
  char chunk[1 << 16];
  size_t k;
  while ((k = std::fread(chunk, 1, sizeof chunk, f)) > 0) buf.append(chunk, k);
  std::fclose(f);
  return parse_dimacs_text(buf.data(), buf.size(), max_n, g);
}

}  // namespace gcl
