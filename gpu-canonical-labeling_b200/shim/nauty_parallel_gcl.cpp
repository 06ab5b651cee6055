// nauty_parallel_gcl.cpp -- the reference's GPU entry point, Nauty_Parallel
// (src/nauty_parallel.h:9-13), on top of this library's C ABI.
//
// A maintainer drops this file into the reference's build in place of
// src/nauty_parallel.cu and links libgcl_b200.so; main.cpp, CSRGraph and the
// command-line flags stay as they are.  The contract main.cpp relies on
// (main.cpp:128-131, 151-154):
//   * n*n bytes come back, row i holding canonical vertex i's adjacency;
//   * an empty vector means failure (main prints "Canonical labeling failed."
//     and exits 1);
//   * the graph is read, not modified or freed.
// The canonical form is the reference's sequential one, bit for bit.  No CSV
// files are written (the reference writes three per call,
// nauty_parallel.cu:886-981); output_prefix is accepted and unused.
#include <cstdint>
#include <string>
#include <vector>

#include "CSRGraph.h"
#include "gcl.h"

std::vector<unsigned char> Nauty_Parallel(CSRGraph& graph, int max_aut, unsigned int* node_count,
                                          const std::string& /*output_prefix*/) {
  const int n = (int)graph.getVertexNum();
  if (n == 0) return {};  // the reference's result for an empty graph is empty too
  std::vector<unsigned char> canon((size_t)n * (size_t)n);
  int64_t nodes = 0;
  // srcPtr / dst are unsigned arrays with the bit layout of int32 CSR
  const int rc = gcl_canon_one(nullptr, reinterpret_cast<const int32_t*>(graph.getSrcPtr()),
                               reinterpret_cast<const int32_t*>(graph.getDst()),
                               graph.getColor(), n, max_aut, canon.data(), &nodes, nullptr);
  if (rc != GCL_OK) return {};
  if (node_count) *node_count = (unsigned int)nodes;
  return canon;
}
