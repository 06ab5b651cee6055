"""The DIMACS reader shared by the file pipeline and the CLI
(csrc/gcl_dimacs.h) against the reference's own reader,
CSRGraph::fromDIMACS (src/CSRGraph.cpp:40-119, compiled from its sources
into oracle/_ref), on well-formed and oddly formatted files, and its
rejections where the reference is undefined.  CPU only: the header is
compiled into a small dump program here."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gpu-canonical-labeling_b200", "csrc")

DUMP = r'''
#include <cstdio>
#include "gcl_dimacs.h"
int main(int argc, char** argv) {
  for (int a = 1; a < argc; ++a) {
    gcl::DimacsGraph g;
    const int rc = gcl::read_dimacs_file(argv[a], 65536, &g);
    std::printf("%d %d %zu %d\n", rc, rc ? 0 : g.n, rc ? (size_t)0 : g.col.size(), rc ? 0 : (int)g.colored);
    if (rc) continue;
    for (int x : g.rowptr) std::printf("%d ", x);
    std::printf("\n");
    for (int x : g.col) std::printf("%d ", x);
    std::printf("\n");
    for (int x : g.color) std::printf("%d ", x);
    std::printf("\n");
  }
  return 0;
}
'''


@pytest.fixture(scope="module")
def dump(tmp_path_factory):
    d = tmp_path_factory.mktemp("dimacs")
    src = d / "dump.cpp"
    src.write_text(DUMP)
    exe = d / "dump"
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-Wall", "-Werror", "-I", CSRC, "-o", str(exe),
                    str(src)], check=True)

    def run(paths):
        out = subprocess.run([str(exe), *map(str, paths)], check=True, capture_output=True,
                             text=True).stdout.split("\n")
        res, i = [], 0
        for _ in paths:
            rc, n, m, colored = map(int, out[i].split())
            i += 1
            if rc:
                res.append((rc, None))
                continue
            rp, cl, co = (np.array(out[i + k].split(), dtype=np.int64) for k in range(3))
            i += 3
            res.append((0, (n, rp, cl, co, bool(colored))))
        return res
    return run


def _same_as_reference(oracle_mod, path, got):
    ref = oracle_mod.ref_read_dimacs(str(path))
    n, rp, cl, co, colored = got
    rn, rrp, rcl, rco = ref
    assert n == rn, path
    assert np.array_equal(rp, rrp) and np.array_equal(cl, rcl) and np.array_equal(co, rco), path
    assert colored == bool((rco != 0).any())


@pytest.mark.skipif(not __import__("oracle").available("reference"),
                    reason="reference build (oracle/_ref) not present")
def test_reader_matches_reference_on_generated_files(G, oracle_mod, dump, tmp_path):
    rng = np.random.default_rng(15)
    graphs = G.small_batch(120, seed=8)
    graphs += [G.erdos_renyi(int(rng.integers(1, 300)), 0.05, rng) for _ in range(20)]
    graphs += [G.from_edges(40, G.erdos_renyi(40, 0.2, rng).edges(), rng.integers(-3, 4, 40))]
    graphs += [G.from_edges(0, []), G.from_edges(1, []), G.from_edges(5, [])]
    paths = []
    for i, g in enumerate(graphs):
        p = tmp_path / f"g{i}.txt"
        G.write_dimacs(g, str(p))
        paths.append(p)
    for p, g, (rc, got) in zip(paths, graphs, dump(paths)):
        assert rc == 0, p
        _same_as_reference(oracle_mod, p, got)
        h = G.read_dimacs(str(p))  # the Python reader agrees too
        assert got[0] == h.n and np.array_equal(got[1], h.rowptr) and np.array_equal(got[2], h.col)


ODD_FILES = {
    "crlf": "p edge 4 3\r\ne 1 2\r\ne 2 3\r\ne 3 4\r\n",
    "no_final_newline": "p edge 3 2\ne 1 2\ne 2 3",
    "comments_blank_lines": "c hello\n\np edge 4 2\nc mid\n\ne 1 4\n\ne 2 3\nc end\n",
    "indented_and_tabs": "  p edge 5 3\n\te 1 2\n   e\t2   5\n  c indented comment\n e 3 4\n",
    "unknown_types": "p edge 4 2\nx 1 2\nq\ne 1 3\nz 9 9 9\ne 2 4\n",
    "self_loops": "p edge 3 3\ne 1 1\ne 1 2\ne 3 3\n",
    "colours": "p edge 4 2\nn 1 5\nn 2 -7\nn 0 3\nn 9 1\nn 3 +2\ne 1 2\ne 3 4\n",
    "colour_overwritten": "p edge 3 1\nn 2 4\nn 2 9\ne 1 3\n",
    "colour_overflow": "p edge 3 1\nn 1 99999999999\nn 2 -99999999999\ne 1 2\n",
    "colour_not_a_number": "p edge 3 1\nn 3 x\ne 2 3\n",
    "trailing_garbage": "p edge 4 2 extra words\ne 1 2 junk\ne 3 4x\n",
    "leading_zeros_and_plus": "p edge 5 2\ne 001 +2\ne 04 0005\n",
    "p_without_m": "p edge 3\ne 1 3\n",
    "p_grows": "p edge 2 1\ne 1 2\np edge 5 2\ne 4 5\n",
    "empty": "",
    "only_comments": "c nothing\nc here\n",
    "p_only": "p edge 6 0\n",
    "no_p_no_edges": "n 1 3\n",
}


@pytest.mark.skipif(not __import__("oracle").available("reference"),
                    reason="reference build (oracle/_ref) not present")
def test_reader_matches_reference_on_odd_formatting(G, oracle_mod, dump, tmp_path):
    paths = []
    for name, text in ODD_FILES.items():
        p = tmp_path / f"{name}.txt"
        p.write_bytes(text.encode())
        paths.append(p)
    for p, (rc, got) in zip(paths, dump(paths)):
        assert rc == 0, p.name
        _same_as_reference(oracle_mod, p, got)
        h = G.read_dimacs(str(p))  # the Python reader follows the same rules
        assert h.n == got[0] and np.array_equal(h.rowptr, got[1]), p.name
        assert np.array_equal(h.col, got[2]) and np.array_equal(h.colors(), got[3]), p.name


def test_reader_rejects_what_the_reference_leaves_undefined(G, dump, tmp_path):
    cases = {
        "duplicate": ("p edge 3 2\ne 1 2\ne 2 1\n", 3),
        "duplicate_same_way": ("p edge 3 2\ne 1 2\ne 1 2\n", 3),
        "endpoint_zero": ("p edge 3 1\ne 0 2\n", 2),
        "endpoint_above_n": ("p edge 3 1\ne 1 4\n", 2),
        "edge_before_p": ("e 1 2\np edge 3 1\n", 2),
        "p_shrinks": ("p edge 5 1\ne 4 5\np edge 3 0\n", 2),
        "one_endpoint": ("p edge 3 1\ne 3\n", 2),
        "negative_endpoint": ("p edge 3 1\ne -1 2\n", 2),
        "too_many_vertices": ("p edge 70000 0\n", 4),
    }
    paths = []
    for name, (text, _) in cases.items():
        p = tmp_path / f"{name}.txt"
        p.write_text(text)
        paths.append(p)
    paths.append(tmp_path / "missing.txt")
    want = [rc for _, rc in cases.values()] + [1]
    got = [rc for rc, _ in dump(paths)]
    assert got == want
    for (text, rc) in cases.values():  # the Python reader raises where the C++ one rejects
        if rc in (2, 3):
            with pytest.raises(ValueError):
                G.parse_dimacs(text)


def test_reader_line_rules_where_the_reference_reads_uninitialised_values(dump, tmp_path):
    # 'n v' without a colour: the reference's colour variable is never
    # written; here the line colours v with 0 (a failed extraction stores nothing)
    p = tmp_path / "n_without_colour.txt"
    p.write_text("p edge 3 1\nn 2 7\nn 2\nn 3 4\ne 1 2\n")
    (rc, (n, rp, cl, co, colored)), = dump([p])
    assert rc == 0 and n == 3 and co.tolist() == [0, 0, 4] and colored
