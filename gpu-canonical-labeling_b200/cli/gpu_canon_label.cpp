// gpu_canon_label -- command-line front-end with the reference's usage
// (main.cpp:14-30, 93-203) on top of the B200 library (include/gcl.h).
//
//   gpu_canon_label <graph.txt> [--parallel|--sequential] [--max-aut=N]
//       canonical adjacency list -> file "output"
//   gpu_canon_label <g1.txt> <g2.txt> [...]
//       "Result: ISOMORPHIC" / "Result: NOT ISOMORPHIC"
//
// Both --parallel and --sequential run the GPU library, whose result is the
// reference's sequential canonical form bit for bit; --sequential also keeps
// the reference's traversal and prints its statistics.
#include <algorithm>
#include <cstdint>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../csrc/gcl_dimacs.h"
#include "../csrc/gcl_format.h"
#include "gcl.h"

namespace {

struct Graph {
  int n = 0;
  std::vector<int32_t> rowptr, col, color;
};

// CSRGraph::fromDIMACS semantics (CSRGraph.cpp:40-119) through the reader
// the file pipeline uses (csrc/gcl_dimacs.h).  Duplicate edges (which the
// reference keeps and then mis-refines), out-of-range endpoints and more than
// GCL_MAX_N vertices are rejected with a message.
Graph read_dimacs(const std::string& path) {
  gcl::DimacsGraph d;
  switch (gcl::read_dimacs_file(path.c_str(), GCL_MAX_N, &d)) {
    case gcl::kDimacsOk:
      break;
    case gcl::kDimacsOpenFailed:
      throw std::runtime_error("Failed to open DIMACS file: " + path);
    case gcl::kDimacsBadEndpoint:
      throw std::runtime_error("edge endpoint out of range in " + path);
    case gcl::kDimacsDuplicateEdge:
      throw std::runtime_error("duplicate edge in " + path + " (parallel edges are not supported)");
    default:
      throw std::runtime_error("graph too large in " + path + " (more than " +
                               std::to_string(GCL_MAX_N) + " vertices)");
  }
  Graph g;
  g.n = d.n;
  g.rowptr = std::move(d.rowptr);
  g.col = std::move(d.col);
  g.color = std::move(d.color);
  return g;
}

void print_help(const char* prog) {
  std::cout << "Usage:\n"
            << "  " << prog << " <graph.txt> [--sequential|--parallel]\n"
            << "  " << prog << " <graph1.txt> <graph2.txt> [--sequential|--parallel]\n\n"
            << "Modes:\n"
            << "  One graph file         Compute the canonical labeling of the graph.\n"
            << "                         The canonical adjacency list is written to a file.\n"
            << "  Two graph files        Compute canonical labels for both graphs and check\n"
            << "                         whether they are isomorphic.\n\n"
            << "Options:\n"
            << "  --max-aut=N            Maximum number of automorphisms stored.\n"
            << "                         Default: 10000\n"
            << "  --sequential           The reference's sequential traversal on the GPU:\n"
            << "                         same canonical form, exact statistics printed.\n"
            << "  --parallel             Use the GPU canonical labeling. Default.\n"
            << "  --group-order          Also print the order of the automorphism group.\n"
            << "  -h, --help             Print this help message.\n";
}

// The reference's adjacency-list format (main.cpp:33-70): "%3u : " prefix,
// " j" tokens, lines wrapped before column 80, ";" terminator -- written row
// by row from the packed canonical rows (gcl::format_row).
void print_adjacency_list(const std::vector<uint64_t>& rows, int n, std::ostream& out) {
  const size_t words = ((size_t)n + 63) / 64;
  std::string text;
  for (int i = 0; i < n; ++i) {
    const uint64_t* row = rows.data() + (size_t)i * words;
    const uint64_t len = gcl::format_row(row, (uint32_t)n, (uint32_t)i, nullptr);
    const size_t at = text.size();
    text.resize(at + len);
    gcl::format_row(row, (uint32_t)n, (uint32_t)i, &text[at]);
    if (text.size() >= (1u << 20)) {
      out.write(text.data(), (std::streamsize)text.size());
      text.clear();
    }
  }
  out.write(text.data(), (std::streamsize)text.size());
}

struct Options {
  unsigned max_aut = 10000;
  bool sequential = false;   // the reference's traversal: exact statistics, printed
  bool group_order = false;  // print |Aut(G)|
};

// --sequential keeps the reference's sequential traversal for every size and
// prints its two statistics lines (sequential.cpp:83-85); the default
// (--parallel) lets large graphs use the wide search, like the reference's
// GPU path.
gcl_context* context(bool sequential) {
  static gcl_context* ctx[2] = {nullptr, nullptr};
  gcl_context*& c = ctx[sequential ? 1 : 0];
  if (!c) {
    if (gcl_create(0, &c) != GCL_OK) return nullptr;
    if (sequential) gcl_set_option(c, GCL_OPT_WIDE_MIN_N, (int64_t)GCL_MAX_N + 1);
  }
  return c;
}

// The canonical form as packed rows (n rows of ceil(n/64) words); false when
// the library reports an error.
bool canonicalize(const Graph& g, const Options& o, std::vector<uint64_t>* rows) {
  std::vector<uint64_t>& out = *rows;
  out.assign((size_t)g.n * (((size_t)g.n + 63) / 64), 0);
  bool colored = std::any_of(g.color.begin(), g.color.end(), [](int c) { return c != 0; });
  int64_t nodes = 0, num_aut = 0;
  gcl_context* c = context(o.sequential);
  int rc = c ? gcl_canon_one_rows(c, g.rowptr.data(), g.col.empty() ? nullptr : g.col.data(),
                                  colored ? g.color.data() : nullptr, g.n, (int)o.max_aut,
                                  out.empty() ? nullptr : out.data(), &nodes, &num_aut)
             : GCL_ERR_CUDA;
  if (rc != GCL_OK) {
    std::cerr << "[ERROR] " << gcl_status_string(rc) << "\n";
    return false;
  }
  if (o.sequential) {
    std::cout << "Total automorphisms discovered (sequential): " << num_aut << std::endl;
    std::cout << "Total search tree nodes created (sequential): " << nodes << std::endl;
  }
  if (o.group_order) {
    double lg = 0;
    std::vector<char> digits(1 << 20);
    int checked = 0;
    int rg = gcl_group_order(c, g.rowptr.data(), g.col.empty() ? nullptr : g.col.data(),
                             colored ? g.color.data() : nullptr, g.n, &lg, digits.data(),
                             (int)digits.size(), nullptr, &checked);
    if (rg != GCL_OK)
      std::cerr << "[ERROR] group order: " << gcl_status_string(rg) << "\n";
    else
      std::cout << "Automorphism group order: " << digits.data()
                << (checked == 0 ? " (unchecked: Schreier-Sims budget exceeded)" : "")
                << std::endl;
  }
  return true;
}

}  // namespace

int main(int argc, char* argv[]) {
  Options opt;
  unsigned& max_aut = opt.max_aut;
  std::vector<std::string> files;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "-h" || a == "--help") {
      print_help(argv[0]);
      return 0;
    } else if (a.rfind("--max-aut=", 0) == 0) {
      try {
        max_aut = (unsigned)std::stoul(a.substr(10));
      } catch (const std::exception& e) {
        std::cerr << "[ERROR] " << e.what() << "\n";
        return 1;
      }
    } else if (a == "--parallel") {
      opt.sequential = false;
    } else if (a == "--sequential") {
      opt.sequential = true;
    } else if (a == "--group-order") {
      opt.group_order = true;
    } else if (!a.empty() && a[0] == '-') {
      std::cerr << "[ERROR] Unknown option: " << a << "\n";
      return 1;
    } else {
      files.push_back(a);
    }
  }
  if (files.size() != 1 && files.size() != 2) {
    std::cerr << "[ERROR] Invalid arguments.\n";
    print_help(argv[0]);
    return 1;
  }
  if (max_aut == 0) {
    std::cerr << "[ERROR] --max-aut must be positive\n";
    return 1;
  }
  try {
    if (files.size() == 1) {
      const Graph g = read_dimacs(files[0]);
      std::vector<uint64_t> canon;
      if (!canonicalize(g, opt, &canon)) {
        std::cerr << "[ERROR] Canonical labeling failed.\n";
        return 1;
      }
      std::ofstream out("output");
      if (!out.is_open()) {
        std::cerr << "[ERROR] Could not open output file: output\n";
        return 1;
      }
      print_adjacency_list(canon, g.n, out);
      return 0;
    }
    const Graph g1 = read_dimacs(files[0]);
    const Graph g2 = read_dimacs(files[1]);
    std::cout << "\nGraph 1: " << files[0] << "\n";
    std::cout << "Computing canonical form...\n";
    std::vector<uint64_t> c1, c2;
    const bool ok1 = canonicalize(g1, opt, &c1);
    std::cout << "\nGraph 2: " << files[1] << "\n";
    std::cout << "Computing canonical form...\n";
    const bool ok2 = canonicalize(g2, opt, &c2);
    if (!ok1 || !ok2) {
      std::cerr << "[ERROR] Canonical labeling failed.\n";
      return 1;
    }
    // equal upper triangles (main.cpp:73-90) of symmetric matrices with a
    // zero diagonal: equal rows; unequal sizes are not isomorphic
    const bool same = g1.n == g2.n && c1 == c2;
    std::cout << "\nResult: " << (same ? "ISOMORPHIC" : "NOT ISOMORPHIC") << "\n";
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "[ERROR] " << e.what() << "\n";
    return 1;
  }
}
