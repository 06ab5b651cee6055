"""Host checks of a batched call (csrc/gcl_batch_check.h, shared by
gcl_canon_batch and gcl_canon_batch_mapped), compiled with g++ and run on
arenas built by the package's packer and on broken copies of them.  No GPU:
these checks run before anything reaches the device."""
import ctypes
import importlib
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gpu-canonical-labeling_b200", "csrc")

SHIM = r'''
#include "gcl_batch_check.h"
extern "C" int check(int count, const int64_t* voff, const int64_t* eoff, const int32_t* rowptr,
                     const int32_t* col, const int64_t* ooff, const int64_t* roff,
                     long long* shape) {
  gcl::BatchShape B;
  const int rc = gcl::check_batch(count, voff, eoff, rowptr, col, ooff, roff, &B);
  shape[0] = B.max_n; shape[1] = B.max_m2; shape[2] = (long long)B.nv;
  shape[3] = (long long)B.ne; shape[4] = (long long)B.nrp;
  shape[5] = (long long)B.dense_bytes; shape[6] = (long long)B.rows_words;
  return rc;
}
'''

OK, ARG, BAD_INPUT, TOO_LARGE = 0, -1, -4, -5


@pytest.fixture(scope="module")
def check(tmp_path_factory):
    d = tmp_path_factory.mktemp("bchk")
    (d / "shim.cpp").write_text(SHIM)
    so = d / "libbchk.so"
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-I", CSRC, "-o", str(so),
                    str(d / "shim.cpp")], check=True)
    lib = ctypes.CDLL(str(so))
    P = ctypes.c_void_p
    lib.check.argtypes = [ctypes.c_int, P, P, P, P, P, P, P]

    def run(count, voff, eoff, rowptr, col, ooff=None, roff=None):
        arrs = [None if a is None else np.ascontiguousarray(a) for a in
                (voff, eoff, rowptr, col, ooff, roff)]
        shape = np.zeros(7, np.int64)
        ptr = lambda a: None if a is None else a.ctypes.data  # noqa: E731
        rc = lib.check(count, *[ptr(a) for a in arrs], shape.ctypes.data)
        return rc, shape
    return run


@pytest.fixture(scope="module")
def arena():
    G = importlib.import_module("gpu-canonical-labeling_b200.graphs")
    api = importlib.import_module("gpu-canonical-labeling_b200.api")
    rng = np.random.default_rng(3)
    graphs = G.small_batch(12, seed=3) + [G.random_regular(80, 3, rng), G.from_edges(0, []),
                                          G.from_edges(1, [])]
    a = G.pack(graphs)
    return a, a.out_offsets(), api.rows_offsets(a), graphs


def test_packed_arena_passes_with_its_shape(check, arena):
    a, ooff, roff, graphs = arena
    rc, shape = check(a.count, a.voff, a.eoff, a.rowptr, a.col, ooff, roff)
    assert rc == OK
    ns = [g.n for g in graphs]
    assert shape[0] == max(ns)
    assert shape[1] == max(g.rowptr[-1] for g in graphs if g.n > 64)
    assert (shape[2], shape[3]) == (sum(ns), int(a.eoff[-1]))
    assert shape[4] == sum(ns) + len(graphs)
    assert (shape[5], shape[6]) == (int(ooff[-1]), int(roff[-1]))
    assert check(0, a.voff, a.eoff, a.rowptr, a.col)[0] == OK
    assert check(-1, a.voff, a.eoff, a.rowptr, a.col)[0] == ARG


def test_broken_arenas_are_rejected(check, arena):
    a, ooff, roff, _ = arena

    def with_(name, i, v):
        arrs = {"voff": a.voff.copy(), "eoff": a.eoff.copy(), "rowptr": a.rowptr.copy(),
                "ooff": ooff.copy(), "roff": roff.copy()}
        arrs[name][i] += v
        return check(a.count, arrs["voff"], arrs["eoff"], arrs["rowptr"], a.col, arrs["ooff"],
                     arrs["roff"])[0]
    assert with_("voff", 0, 1) == ARG          # offsets start at 0
    assert with_("eoff", 0, 1) == ARG
    assert with_("ooff", 0, -5) == ARG         # output offsets start at 0 too
    assert with_("roff", 0, 3) == ARG
    assert with_("ooff", 3, 1) == ARG          # a block of the wrong size
    assert with_("roff", 5, -1) == ARG
    assert with_("rowptr", int(a.voff[2]) + 2, 1) == BAD_INPUT  # local rowptr not from 0
    assert with_("eoff", 4, 1) == BAD_INPUT    # CSR size disagrees with the local rowptr
    # a descending vertex offset is a negative vertex count
    v = a.voff.copy()
    v[3] = v[2] - 1
    assert check(a.count, v, a.eoff, a.rowptr, a.col, None, None)[0] in (ARG, BAD_INPUT)
    # no col with edges in the batch
    assert check(a.count, a.voff, a.eoff, a.rowptr, None, None, None)[0] == ARG


def test_too_large_graph(check):
    n = 65537
    voff = np.array([0, n], np.int64)
    eoff = np.array([0, 0], np.int64)
    rowptr = np.zeros(n + 1, np.int32)
    assert check(1, voff, eoff, rowptr, None)[0] == TOO_LARGE
