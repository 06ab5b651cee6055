"""The reference's adjacency-list text from bit-packed canonical rows
(csrc/gcl_format.h, shared by the device formatter) against a restatement of
print_canonical_adjacency_list (main.cpp:33-70) over the n x n matrix.  CPU
only: the header is compiled here with g++."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from test_cli import reference_listing

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gpu-canonical-labeling_b200", "csrc")

SHIM = r'''
#include <cstdint>
#include "gcl_format.h"
extern "C" uint64_t format_graph(const uint64_t* rows, uint32_t n, char* out) {
  const uint32_t words = (n + 63) / 64;
  uint64_t at = 0;
  for (uint32_t i = 0; i < n; ++i)
    at += gcl::format_row(rows + (uint64_t)i * words, n, i, out ? out + at : nullptr);
  return at;
}
'''


@pytest.fixture(scope="module")
def fmt(tmp_path_factory):
    d = tmp_path_factory.mktemp("fmt")
    (d / "f.cpp").write_text(SHIM)
    so = d / "libfmt.so"
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-Wall", "-Werror", "-shared", "-fPIC", "-I", CSRC,
                    "-o", str(so), str(d / "f.cpp")], check=True)
    lib = ctypes.CDLL(str(so))
    lib.format_graph.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]
    lib.format_graph.restype = ctypes.c_uint64

    def run(mat):
        n = mat.shape[0]
        w = (n + 63) // 64
        padded = np.zeros((n, w * 64), np.uint8)
        padded[:, :n] = mat
        rows = np.packbits(padded, axis=1, bitorder="little").view(np.uint64).copy()
        size = lib.format_graph(rows.ctypes.data, n, None)
        buf = ctypes.create_string_buffer(int(size) + 1)
        assert lib.format_graph(rows.ctypes.data, n, buf) == size
        return buf.raw[:size].decode()
    return run


def test_rows_format_like_the_reference(G, oracle_mod, fmt):
    rng = np.random.default_rng(50)
    graphs = [G.from_edges(1, []), G.from_edges(7, []), G.torus(5), G.random_regular(200, 3, rng)]
    graphs += [G.from_edges(40, [(i, j) for i in range(40) for j in range(i + 1, 40)])]
    graphs += [G.erdos_renyi(150, 0.5, rng), G.tree_plus_edges(300, rng)]
    graphs += list(G.small_batch(30, seed=51))
    for g in graphs:
        mat = oracle_mod.canon(g)[0]
        assert fmt(mat) == reference_listing(mat), g.n


def test_wide_rows_and_long_lines(fmt):
    # 1,100 vertices: prefixes wider than %3u, five-character tokens, wrapped
    # lines, a full row, an empty row, and a row ending at the last word's edge
    rng = np.random.default_rng(52)
    n = 1100
    a = (rng.random((n, n)) < 0.05).astype(np.uint8)
    a = np.triu(a, 1)
    a = a | a.T
    a[0, 1:] = a[1:, 0] = 1
    a[5, :] = a[:, 5] = 0
    np.fill_diagonal(a, 0)
    assert fmt(a) == reference_listing(a)
