"""The CLI's host logic without a GPU: the `output` text written from packed
rows and the isomorphism verdict, with the library's entry points that the
CLI calls answered by a stand-in built here over the oracle (LD_PRELOAD, so
the CLI binary itself is the one the build made).  The stand-in is test
infrastructure: it checks the CLI's formatting and comparison code, not the
library, whose results the GPU tests pin."""
import os
import subprocess

import numpy as np
import pytest

from test_cli import CLI, reference_listing

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle")

STANDIN = r'''
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "canon_oracle.h"
typedef struct gcl_context gcl_context;
static int dummy;
int gcl_create(int device, gcl_context** out) { (void)device; *out = (gcl_context*)&dummy; return 0; }
int gcl_set_option(gcl_context* c, int o, int64_t v) { (void)c; (void)o; (void)v; return 0; }
const char* gcl_status_string(int s) { (void)s; return "stand-in error"; }
int gcl_group_order(gcl_context* c, const int32_t* rp, const int32_t* col, const int32_t* color,
                    int n, double* lg, char* digits, int cap, int64_t* gens, int* checked) {
  (void)c; (void)rp; (void)col; (void)color; (void)n; (void)lg; (void)digits; (void)cap;
  (void)gens; (void)checked;
  return -7;
}
int gcl_canon_one_rows(gcl_context* c, const int32_t* rp, const int32_t* col,
                       const int32_t* color, int n, int max_aut, uint64_t* rows,
                       int64_t* nodes, int64_t* naut) {
  (void)c;
  if (n == 0) { if (nodes) *nodes = 1; if (naut) *naut = 0; return 0; }
  uint8_t* m = (uint8_t*)malloc((size_t)n * n);
  gcl_oracle_stats st;
  memset(&st, 0, sizeof st);
  int rc = gcl_oracle_canon(n, rp, col, color, (unsigned)max_aut, m, NULL, &st);
  if (rc == 0) {
    const int words = (n + 63) / 64;
    memset(rows, 0, (size_t)n * words * 8);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        if (m[(size_t)i * n + j]) rows[(size_t)i * words + j / 64] |= 1ull << (j % 64);
  }
  free(m);
  return rc == 0 ? 0 : -7;
}
'''


@pytest.fixture(scope="module")
def standin(tmp_path_factory, oracle_mod):
    if not os.path.exists(CLI):
        pytest.skip("CLI not built")
    d = tmp_path_factory.mktemp("standin")
    (d / "standin.c").write_text(STANDIN)
    so = d / "libstandin.so"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-O2", "-shared", "-fPIC", "-I", ORACLE, "-o", str(so),
                    str(d / "standin.c"), os.path.join(ORACLE, "canon_oracle.c")], check=True)
    return str(so)


def _run(standin, args, cwd):
    env = dict(os.environ, LD_PRELOAD=standin)
    return subprocess.run([CLI, *args], cwd=cwd, env=env, capture_output=True, text=True,
                          timeout=120)


def test_output_text_from_packed_rows(G, oracle_mod, standin, tmp_path):
    rng = np.random.default_rng(12)
    graphs = [G.erdos_renyi(40, 0.3, rng), G.torus(9), G.random_regular(130, 3, rng),
              G.from_edges(70, [(i, j) for i in range(70) for j in range(i + 1, 70)
                                if (i * 7 + j) % 3 == 0]),  # rows longer than 80 columns
              G.from_edges(1, []), G.from_edges(3, [])]
    for k, g in enumerate(graphs):
        p = tmp_path / f"g{k}.txt"
        G.write_dimacs(g, str(p))
        r = _run(standin, [str(p)], tmp_path)
        assert r.returncode == 0, r.stderr
        want = reference_listing(oracle_mod.canon(g)[0])
        assert (tmp_path / "output").read_text() == want, g.n


def test_isomorphism_verdicts(G, standin, tmp_path):
    rng = np.random.default_rng(13)
    er = G.erdos_renyi(100, 0.06, rng)
    G.write_dimacs(er, str(tmp_path / "a.txt"))
    G.write_dimacs(G.random_relabel(er, rng), str(tmp_path / "b.txt"))
    G.write_dimacs(G.move_one_edge(er, rng), str(tmp_path / "c.txt"))
    G.write_dimacs(G.from_edges(99, er.edges()[er.edges().max(axis=1) < 99]),
                   str(tmp_path / "d.txt"))
    out = lambda a, b: _run(standin, [a, b], tmp_path).stdout  # noqa: E731
    assert "Result: ISOMORPHIC" in out("a.txt", "b.txt")
    assert "Result: NOT ISOMORPHIC" in out("a.txt", "c.txt")
    assert "Result: NOT ISOMORPHIC" in out("a.txt", "d.txt")  # unequal vertex counts
