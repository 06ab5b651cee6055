// ref_shim.cpp -- TEST INFRASTRUCTURE ONLY (never linked into the product).
//
// A C-ABI shim around the reference's own sequential canonical labeler so
// tests, the golden-fixture script and bench.py's CPU baseline can call it
// in-process.  The reference sources are compiled unchanged from where they
// lie (src/sequential.cpp, src/partition_refinement.cpp, src/perm_group.cpp,
// src/CSRGraph.cpp); this file only adds:
//   * a stub Nauty_Parallel (the GPU entry point, never called on the
//     --sequential path; nauty_parallel.h:9-13),
//   * gcl_ref_canon(): builds a CSRGraph from plain arrays, runs
//     Nauty_Sequential (sequential.cpp:13-88) and copies best_leaf out,
//     the same copy main.cpp:133-144 performs.
//
// The reference constructor prints three lines per graph to std::cout
// (sequential.cpp:73-85); gcl_ref_quiet() sends std::cout to a null buffer
// so batch timing is not dominated by terminal I/O.
#include <cstdint>
#include <cstring>
#include <iostream>
#include <stdexcept>
#include <streambuf>
#include <string>
#include <vector>

#include "CSRGraph.h"
#include "nauty_parallel.h"
// node_counter / num_aut are private members of Nauty_Sequential; the shim
// reads them for the node and automorphism counts the reference prints.
#define private public
#include "sequential.h"
#undef private

std::vector<unsigned char> Nauty_Parallel(CSRGraph&, int, unsigned int*,
                                          const std::string&) {
  return {};
}

namespace {
struct NullBuf : std::streambuf {
  int overflow(int c) override { return c; }
  std::streamsize xsputn(const char*, std::streamsize n) override { return n; }
};
NullBuf g_null;
}  // namespace

extern "C" {

struct gcl_ref_stats {
  int64_t num_aut;  // "Total automorphisms discovered" (sequential.cpp:83)
  int64_t nodes;    // "Total search tree nodes created" (sequential.cpp:85)
};

void gcl_ref_quiet(int on) {
  static std::streambuf* saved = nullptr;
  if (on) {
    if (!saved) saved = std::cout.rdbuf(&g_null);
  } else if (saved) {
    std::cout.rdbuf(saved);
    saved = nullptr;
  }
}

// rowptr[n+1], col[rowptr[n]] (both directions, rows sorted, no self loops,
// no duplicates -- the shape CSRGraph::fromDIMACS builds, CSRGraph.cpp:40-119),
// color[n] or NULL.  out_nxn receives best_leaf.hash_of_perm_graph (n*n bytes,
// 0/1), label_out (may be NULL) receives best_leaf.label (position -> vertex).
int gcl_ref_canon(int n, const int32_t* rowptr, const int32_t* col,
                  const int32_t* color, unsigned max_aut, uint8_t* out_nxn,
                  int32_t* label_out, gcl_ref_stats* st) {
  if (n < 0 || max_aut == 0) return -1;
  const unsigned m2 = n ? (unsigned)rowptr[n] : 0u;
  CSRGraph g((unsigned)n, m2);  // new[] arrays; ~Nauty_Sequential frees them
  for (int i = 0; i <= n; ++i) g.srcPtr[i] = (unsigned)rowptr[i];
  for (unsigned e = 0; e < m2; ++e) g.dst[e] = (unsigned)col[e];
  for (int i = 0; i < n; ++i) {
    g.degree[i] = rowptr[i + 1] - rowptr[i];
    g.color[i] = color ? color[i] : 0;
  }
  {
    Nauty_Sequential nauty(g, max_aut);
    for (long i = 0; i < (long)n * n; ++i)
      out_nxn[i] = (uint8_t)nauty.best_leaf.hash_of_perm_graph[i];
    if (label_out)
      for (int i = 0; i < n; ++i) label_out[i] = nauty.best_leaf.label[i];
    if (st) {
      st->num_aut = nauty.num_aut;
      st->nodes = nauty.node_counter;
    }
    // The reference never frees its per-level target cells
    // (sequential.cpp:39-46); free them here so long batch runs stay bounded.
    if (nauty.target_cell_at_level) {
      for (int i = 0; i <= n; ++i) delete[] nauty.target_cell_at_level[i].elems;
      delete[] nauty.target_cell_at_level;
      nauty.target_cell_at_level = nullptr;
    }
  }
  return 0;
}

// Batched form over a ragged arena: graph g has vertices
// [voff[g], voff[g+1]) and CSR entries [eoff[g], eoff[g+1]); rowptr for graph
// g is local (starts at 0) and stored at rowptr_arena[voff[g] + g ...]
// (n_g + 1 entries per graph).  Outputs go to out_arena at ooff[g] (n_g^2
// bytes) and stats[g].
int gcl_ref_canon_batch(int count, const int64_t* voff, const int64_t* eoff,
                        const int32_t* rowptr_arena, const int32_t* col_arena,
                        const int32_t* color_arena, unsigned max_aut,
                        uint8_t* out_arena, const int64_t* ooff,
                        gcl_ref_stats* stats) {
  for (int gi = 0; gi < count; ++gi) {
    const int n = (int)(voff[gi + 1] - voff[gi]);
    const int32_t* rp = rowptr_arena + voff[gi] + gi;
    const int32_t* cl = col_arena + eoff[gi];
    const int32_t* co = color_arena ? color_arena + voff[gi] : nullptr;
    int rc = gcl_ref_canon(n, rp, cl, co, max_aut, out_arena + ooff[gi],
                           nullptr, stats ? stats + gi : nullptr);
    if (rc) return rc;
  }
  return 0;
}

// The reference's own DIMACS reader, CSRGraph::fromDIMACS
// (CSRGraph.cpp:40-119), for checking other readers.  Only files on which it
// is well defined may be given: every edge endpoint within 1..n of the last
// 'p' line before it, and every 'e' line with two numbers.  Returns 0 with n,
// the CSR and the colours copied out; 1 when the file cannot be opened; 2
// when n > cap_n or the entries > cap_m.
int gcl_ref_read_dimacs(const char* path, int cap_n, int64_t cap_m, int* n_out,
                        int64_t* m_out, int32_t* rowptr, int32_t* col, int32_t* color) {
  CSRGraph g;
  try {
    g = CSRGraph::fromDIMACS(path);
  } catch (const std::runtime_error&) {
    return 1;
  }
  const unsigned n = g.vertexNum;
  const int64_t m = n ? (int64_t)g.srcPtr[n] : 0;
  int rc = 0;
  if ((int64_t)n > cap_n || m > cap_m) {
    rc = 2;
  } else {
    *n_out = (int)n;
    *m_out = m;
    for (unsigned i = 0; i <= n; ++i) rowptr[i] = n ? (int32_t)g.srcPtr[i] : 0;
    for (int64_t e = 0; e < m; ++e) col[e] = (int32_t)g.dst[e];
    for (unsigned i = 0; i < n; ++i) color[i] = g.color[i];
  }
  g.cleanup();
  return rc;
}

}  // extern "C"
