"""Schreier-Sims with a known base (gcl::group_order_with_base) against the
general completion (gcl::group_order), on the automorphisms the CPU model
of the wide search stores, with the model's first path as the base.  For a
graph the first path's individualized vertices are a base of Aut(G): an
automorphism that fixes them fixes the first leaf's discrete partition.
CPU only: the host file csrc/gcl_group.cu is compiled here with g++."""
import ctypes
import math
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gpu-canonical-labeling_b200", "csrc")

SHIM = r'''
#include <cstring>
#include <string>
#include "gcl_group.h"
extern "C" int order_generic(unsigned n, const unsigned short* a, unsigned long long count,
                             unsigned long long cap, char* out, int out_cap) {
  double lg; std::string d; unsigned long long bl;
  if (!gcl::group_order(n, a, count, n, cap, &lg, &d, (uint64_t*)&bl)) return 1;
  if ((int)d.size() + 1 > out_cap) return 3;
  std::memcpy(out, d.c_str(), d.size() + 1);
  return 0;
}
extern "C" int order_orbits(unsigned n, const unsigned short* a, unsigned long long count,
                            const unsigned* base, unsigned nbase, char* out, int out_cap) {
  double lg; std::string d;
  if (!gcl::group_order_base_orbits(n, a, count, n, base, nbase, &lg, &d)) return 1;
  if ((int)d.size() + 1 > out_cap) return 3;
  std::memcpy(out, d.c_str(), d.size() + 1);
  return 0;
}
extern "C" int order_search(unsigned n, const unsigned short* a, unsigned long long count,
                            const unsigned* base, unsigned nbase, unsigned long long cap,
                            int* checked, char* out, int out_cap) {
  double lg; std::string d;
  const int rc = gcl::group_order_of_search(n, a, count, n, base, nbase, cap, &lg, &d, checked);
  if (rc) return rc;
  if ((int)d.size() + 1 > out_cap) return 3;
  std::memcpy(out, d.c_str(), d.size() + 1);
  return 0;
}
extern "C" int order_base(unsigned n, const unsigned short* a, unsigned long long count,
                          const unsigned* base, unsigned nbase, unsigned long long cap,
                          char* out, int out_cap) {
  double lg; std::string d; unsigned long long bl;
  const int rc = gcl::group_order_with_base(n, a, count, n, base, nbase, cap, &lg, &d,
                                            (uint64_t*)&bl);
  if (rc) return rc;
  if ((int)d.size() + 1 > out_cap) return 3;
  std::memcpy(out, d.c_str(), d.size() + 1);
  return 0;
}
'''


@pytest.fixture(scope="module")
def grp(tmp_path_factory):
    d = tmp_path_factory.mktemp("grp")
    (d / "shim.cpp").write_text(SHIM)
    so = d / "libgrp.so"
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-I", CSRC, "-o", str(so),
                    str(d / "shim.cpp"), "-x", "c++", os.path.join(CSRC, "gcl_group.cu")],
                   check=True)
    lib = ctypes.CDLL(str(so))
    P = ctypes.c_void_p
    lib.order_generic.argtypes = [ctypes.c_uint, P, ctypes.c_ulonglong, ctypes.c_ulonglong,
                                  ctypes.c_char_p, ctypes.c_int]
    lib.order_base.argtypes = [ctypes.c_uint, P, ctypes.c_ulonglong, P, ctypes.c_uint,
                               ctypes.c_ulonglong, ctypes.c_char_p, ctypes.c_int]
    lib.order_search.argtypes = [ctypes.c_uint, P, ctypes.c_ulonglong, P, ctypes.c_uint,
                                 ctypes.c_ulonglong, P, ctypes.c_char_p, ctypes.c_int]
    lib.order_orbits.argtypes = [ctypes.c_uint, P, ctypes.c_ulonglong, P, ctypes.c_uint,
                                 ctypes.c_char_p, ctypes.c_int]

    def generic(perms, cap=0):
        p = np.ascontiguousarray(perms, dtype=np.uint16)
        buf = ctypes.create_string_buffer(1 << 16)
        rc = lib.order_generic(p.shape[1], p.ctypes.data if p.size else None, p.shape[0], cap,
                               buf, len(buf))
        return rc, (int(buf.value.decode()) if rc == 0 else None)

    def based(perms, base, cap=0):
        p = np.ascontiguousarray(perms, dtype=np.uint16)
        b = np.ascontiguousarray(base, dtype=np.uint32)
        buf = ctypes.create_string_buffer(1 << 16)
        rc = lib.order_base(p.shape[1], p.ctypes.data if p.size else None, p.shape[0],
                            b.ctypes.data if b.size else None, b.size, cap, buf, len(buf))
        return rc, (int(buf.value.decode()) if rc == 0 else None)
    def orbits(perms, base):
        p = np.ascontiguousarray(perms, dtype=np.uint16)
        b = np.ascontiguousarray(base, dtype=np.uint32)
        buf = ctypes.create_string_buffer(1 << 16)
        rc = lib.order_orbits(p.shape[1], p.ctypes.data if p.size else None, p.shape[0],
                              b.ctypes.data if b.size else None, b.size, buf, len(buf))
        return rc, (int(buf.value.decode()) if rc == 0 else None)
    def search(perms, base, cap):
        p = np.ascontiguousarray(perms, dtype=np.uint16)
        b = np.ascontiguousarray(base, dtype=np.uint32)
        buf = ctypes.create_string_buffer(1 << 16)
        checked = ctypes.c_int(-1)
        rc = lib.order_search(p.shape[1], p.ctypes.data if p.size else None, p.shape[0],
                              b.ctypes.data if b.size else None, b.size, cap,
                              ctypes.byref(checked), buf, len(buf))
        return rc, (int(buf.value.decode()) if rc == 0 else None), checked.value
    based.orbits = orbits
    based.search = search
    return generic, based


def _model(wm, g, workers=16, seed=0):
    fs = []
    _, _, naut, _, store = wm.wide_model(g, workers, seed, cap=100000, auts=True, first_seq=fs)
    assert naut < 100000
    return store, fs


@pytest.fixture(scope="module")
def wm(oracle_mod):
    if not os.path.exists(oracle_mod.WIDE_SO):
        subprocess.run(["make", "-s", "-C", os.path.dirname(oracle_mod.WIDE_SO)], check=True)
    return oracle_mod


def test_known_base_matches_general_completion(G, wm, grp):
    generic, based = grp
    rng = np.random.default_rng(8)
    pet = G.from_edges(10, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 0), (0, 5), (1, 6), (2, 7),
                            (3, 8), (4, 9), (5, 7), (7, 9), (9, 6), (6, 8), (8, 5)])
    cube = lambda d: G.from_edges(1 << d, [(a, a ^ (1 << b)) for a in range(1 << d)
                                           for b in range(d) if a < a ^ (1 << b)])
    graphs = [G.torus(k) for k in (3, 5, 8, 16)] + [cube(d) for d in (3, 5, 7)]
    graphs += [G.disjoint_union(pet, 4), G.disjoint_union(G.torus(3), 3), G.from_edges(12, [])]
    graphs += [G.cfi_graph(b, rng, twist=bool(b % 4)) for b in (4, 8, 12)]
    graphs += [G.random_regular(n, 3, rng) for n in (12, 40)]
    graphs += [G.from_edges(60, G.recursive_tree(60, rng)), G.tree_plus_edges(90, rng)]
    graphs += list(G.small_batch(40, seed=77))
    for i, g in enumerate(graphs):
        store, fs = _model(wm, g, seed=i)
        rc1, a = generic(store)
        rc2, b = based(store, fs)
        rc3, c = based.orbits(store, fs)
        assert rc1 == 0 and rc2 == 0 and rc3 == 0, (i, rc1, rc2, rc3)
        assert a == b == c, (i, g.n, a, b, c)


def test_base_orbit_product_on_every_schedule(G, wm, grp):
    # the stored automorphisms of any schedule (gate on or off, work handed
    # over or not) are a strong generating set for the first path: the product
    # of its basic orbits equals the Schreier-Sims order
    generic, based = grp
    rng = np.random.default_rng(19)
    graphs = [G.torus(4, 6), G.cfi_graph(6, rng), G.disjoint_union(G.random_regular(8, 3, rng), 3)]
    graphs += [G.from_edges(10, [])] + list(G.small_batch(20, seed=19))
    for i, g in enumerate(graphs):
        for workers, seed, gate, donate in ((1, 0, True, False), (5, 3, False, False),
                                            (9, 7, True, True), (4, 2, False, True)):
            fs = []
            _, _, naut, _, store = wm.wide_model(g, workers, seed, cap=100000, auts=True,
                                                 first_seq=fs, gate=gate, donate=donate)
            rc, a = generic(store)
            rc2, c = based.orbits(store, fs)
            assert rc == 0 and rc2 == 0 and a == c, (i, workers, seed, gate, donate, a, c)


def test_base_orbit_product_for_a_large_symmetric_group(G, wm, grp):
    # S_120 (the empty graph): instant from the basic orbits
    import math
    _, based = grp
    store, fs = _model(wm, G.from_edges(120, []))
    rc, c = based.orbits(store, fs)
    assert rc == 0 and c == math.factorial(120)


def test_known_base_finishes_where_representatives_do_not_fit(grp):
    # torus 100 x 100 (10,000 points, order 80,000): explicit coset
    # representatives exceed their budget, so the general completion walks
    # Schreier vectors of ~100 generators on every point; with the base
    # (a vertex, a neighbour, a vertex off their line) only base images move
    generic, based = grp
    k = 100
    n = k * k
    idx = np.arange(n)
    x, y = idx // k, idx % k
    gens = np.array([((x + 1) % k) * k + y, x * k + (y + 1) % k, y * k + (-x) % k,
                     x * k + (-y) % k])
    rc, order = based(gens, [0, 1, k + 2])
    assert rc == 0 and order == 8 * n
    rc, _ = generic(gens, cap=int(2e9))
    assert rc == 1  # the general completion runs out of its work budget


def test_points_that_are_no_base_are_reported_when_met(grp):
    # the caller vouches for the base; an element seen to fix every base
    # point without being the identity (here an input generator) is reported
    _, based = grp
    n = 7
    cyc = [(i + 1) % n for i in range(n)]
    swap = [1, 0] + list(range(2, n))
    fix01 = [0, 1, 3, 2] + list(range(4, n))
    rc, _ = based(np.array([cyc, swap, fix01]), [0, 1])  # S_7 needs 6 base points
    assert rc == 2
    rc, order = based(np.array([cyc, swap, fix01]), list(range(6)))
    assert rc == 0 and order == math.factorial(7)


CHECK_CAP = 400_000_000  # the library's check budget (kGroupCheckCap in csrc/gcl_capi.cu)


def test_search_order_is_checked_where_schreier_sims_finishes(G, wm, grp):
    # gcl::group_order_of_search: the basic-orbit product, with the
    # Schreier-Sims completion agreeing wherever it finishes in its budget
    generic, based = grp
    rng = np.random.default_rng(31)
    graphs = [G.torus(k) for k in (4, 7, 12)] + [G.cfi_graph(8, rng), G.from_edges(9, [])]
    graphs += [G.disjoint_union(G.random_regular(10, 3, rng), 4), G.tree_plus_edges(80, rng)]
    graphs += list(G.small_batch(30, seed=31))
    for i, g in enumerate(graphs):
        store, fs = _model(wm, g, seed=i)
        rc, order, checked = based.search(store, fs, CHECK_CAP)
        rc1, want = generic(store)
        assert rc == 0 and rc1 == 0 and order == want and checked == 1, (i, g.n, order, want)
        # no check asked for: the same order, unchecked
        assert based.search(store, fs, 0) == (0, want, 0)


def test_search_order_of_a_large_symmetric_group_is_immediate(G, wm, grp):
    # S_300 (the empty graph): both completions run out of their check budget
    # (about a second) and the basic-orbit product stands; before, the general
    # and the known-base completion ran for tens of seconds first
    import time
    _, based = grp
    store, fs = _model(wm, G.from_edges(300, []))
    t = time.time()
    rc, order, checked = based.search(store, fs, CHECK_CAP)
    assert rc == 0 and order == math.factorial(300) and checked == 0
    assert time.time() - t < 10


def test_search_order_disagreement_returns_the_completion(grp):
    # a planted mistake: generators of S_4 that are no strong generating set
    # for the base (0, 1, 2) -- the basic-orbit product gives 4, Schreier-Sims
    # 24, and the completion's order is returned, flagged
    _, based = grp
    cyc = [1, 2, 3, 0]
    swap = [1, 0, 2, 3]
    assert based.search(np.array([cyc, swap]), [0, 1, 2], CHECK_CAP) == (0, 24, -1)
    # unchecked, the product alone is wrong here
    assert based.search(np.array([cyc, swap]), [0, 1, 2], 0) == (0, 4, 0)
