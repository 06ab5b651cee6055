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
#include <iomanip>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "gcl.h"

namespace {

struct Graph {
  int n = 0;
  std::vector<int32_t> rowptr, col, color;
};

// CSRGraph::fromDIMACS semantics (CSRGraph.cpp:40-119): 'c' and empty lines
// skipped, 'p' sets the vertex count, 'n v c' sets a colour (1-based, vertex 0
// and out-of-range ignored), 'e u v' is 1-based with self loops dropped and
// both directions stored, rows sorted.  Duplicate edges (which the reference
// keeps and then mis-refines) and out-of-range endpoints are rejected.
Graph read_dimacs(const std::string& path) {
  std::ifstream in(path);
  if (!in.is_open()) throw std::runtime_error("Failed to open DIMACS file: " + path);
  unsigned n = 0;
  std::vector<std::pair<unsigned, unsigned>> edges;
  std::vector<std::pair<unsigned, int>> colors;
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == 'c') continue;
    std::istringstream iss(line);
    char type = 0;
    iss >> type;
    if (type == 'p') {
      std::string tmp;
      unsigned m = 0;
      iss >> tmp >> n >> m;
    } else if (type == 'n') {
      unsigned vid = 0;
      int c = 0;
      iss >> vid >> c;
      if (vid == 0) continue;
      colors.emplace_back(vid - 1, c);
    } else if (type == 'e') {
      unsigned u = 0, v = 0;
      iss >> u >> v;
      if (u == v) continue;
      if (u == 0 || v == 0 || u > n || v > n)
        throw std::runtime_error("edge endpoint out of range in " + path);
      edges.emplace_back(u - 1, v - 1);
      edges.emplace_back(v - 1, u - 1);
    }
  }
  std::sort(edges.begin(), edges.end());
  for (size_t i = 1; i < edges.size(); ++i)
    if (edges[i] == edges[i - 1])
      throw std::runtime_error("duplicate edge in " + path + " (parallel edges are not supported)");
  Graph g;
  g.n = (int)n;
  g.rowptr.assign(n + 1, 0);
  g.col.resize(edges.size());
  g.color.assign(n, 0);
  for (auto& kv : colors)
    if (kv.first < n) g.color[kv.first] = kv.second;
  for (auto& e : edges) g.rowptr[e.first + 1]++;
  for (unsigned i = 0; i < n; ++i) g.rowptr[i + 1] += g.rowptr[i];
  for (size_t i = 0; i < edges.size(); ++i) g.col[i] = (int32_t)edges[i].second;
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
// " j" tokens, lines wrapped before column 80, ";" terminator.
void print_adjacency_list(const std::vector<unsigned char>& A, int n, std::ostream& out) {
  const int max_width = 80;
  for (int i = 0; i < n; ++i) {
    std::ostringstream ps;
    ps << std::setw(3) << i << " : ";
    const std::string prefix = ps.str();
    out << prefix;
    int width = (int)prefix.size();
    bool first = true;
    for (int j = 0; j < n; ++j) {
      if (!A[(size_t)i * n + j]) continue;
      const std::string tok = " " + std::to_string(j);
      if (!first && width + (int)tok.size() + 1 > max_width) {
        out << "\n    ";
        width = 4;
      }
      out << tok;
      width += (int)tok.size();
      first = false;
    }
    out << ";\n";
  }
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

std::vector<unsigned char> canonicalize(const Graph& g, const Options& o) {
  std::vector<unsigned char> out((size_t)g.n * g.n);
  bool colored = std::any_of(g.color.begin(), g.color.end(), [](int c) { return c != 0; });
  int64_t nodes = 0, num_aut = 0;
  gcl_context* c = context(o.sequential);
  int rc = c ? gcl_canon_one(c, g.rowptr.data(), g.col.empty() ? nullptr : g.col.data(),
                             colored ? g.color.data() : nullptr, g.n, (int)o.max_aut,
                             out.empty() ? nullptr : out.data(), &nodes, &num_aut)
             : GCL_ERR_CUDA;
  if (rc != GCL_OK) {
    std::cerr << "[ERROR] " << gcl_status_string(rc) << "\n";
    return {};
  }
  if (o.sequential) {
    std::cout << "Total automorphisms discovered (sequential): " << num_aut << std::endl;
    std::cout << "Total search tree nodes created (sequential): " << nodes << std::endl;
  }
  if (o.group_order) {
    double lg = 0;
    std::vector<char> digits(1 << 20);
    int rg = gcl_group_order(c, g.rowptr.data(), g.col.empty() ? nullptr : g.col.data(),
                             colored ? g.color.data() : nullptr, g.n, &lg, digits.data(),
                             (int)digits.size(), nullptr);
    if (rg != GCL_OK)
      std::cerr << "[ERROR] group order: " << gcl_status_string(rg) << "\n";
    else
      std::cout << "Automorphism group order: " << digits.data() << std::endl;
  }
  return out;
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
      const std::vector<unsigned char> canon = canonicalize(g, opt);
      if (canon.empty() && g.n > 0) {
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
    const std::vector<unsigned char> c1 = canonicalize(g1, opt);
    std::cout << "\nGraph 2: " << files[1] << "\n";
    std::cout << "Computing canonical form...\n";
    const std::vector<unsigned char> c2 = canonicalize(g2, opt);
    if ((c1.empty() && g1.n > 0) || (c2.empty() && g2.n > 0)) {
      std::cerr << "[ERROR] Canonical labeling failed.\n";
      return 1;
    }
    bool same = g1.n == g2.n;
    for (int i = 0; same && i < g1.n; ++i)
      for (int j = i + 1; j < g1.n; ++j)
        if ((c1[(size_t)i * g1.n + j] != 0) != (c2[(size_t)i * g1.n + j] != 0)) {
          same = false;
          break;
        }
    std::cout << "\nResult: " << (same ? "ISOMORPHIC" : "NOT ISOMORPHIC") << "\n";
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "[ERROR] " << e.what() << "\n";
    return 1;
  }
}
