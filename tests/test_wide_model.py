"""CPU model of the many-worker search (oracle/wide_model.c) against the
sequential oracle.

The GPU's wide search (csrc/canon_wide.cuh) changes two rules of the
reference's traversal (src/sequential.cpp:396-624): a leaf equivalent to a
best leaf found outside the current work item steps back one level instead
of jumping to the common ancestor, and a node that is worse than a newly
adopted best is pruned.  These tests run the same rules on the CPU under
many interleavings of the workers and check that every schedule yields the
sequential canonical matrix, and that the sequential result is the maximum
over all leaves of the unpruned tree -- the property that makes the result
independent of the order in which the leaves are met.
"""
import os

import numpy as np
import pytest


@pytest.fixture(scope="module")
def wm(oracle_mod):
    if not os.path.exists(oracle_mod.WIDE_SO):
        import subprocess
        subprocess.run(["make", "-s", "-C", os.path.dirname(oracle_mod.WIDE_SO)], check=True)
    return oracle_mod


def _cases(G):
    rng = np.random.default_rng(4242)
    out = [G.torus(4), G.torus(3, 5), G.torus(6)]
    out.append(G.disjoint_union(G.torus(3), 3))
    out.append(G.disjoint_union(G.from_edges(5, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 0)]), 4))
    for n in (12, 20, 32):
        out.append(G.random_regular(n, 3, rng))
    for n in (24, 40):
        out.append(G.from_edges(n, G.recursive_tree(n, rng)))
    for n in (16, 30):
        g = G.erdos_renyi(n, 0.2, rng)
        out.append(G.from_edges(n, g.edges(), rng.integers(0, 2, n)))
    out.append(G.random_relabel(G.torus(5), rng))
    return out


def test_wide_model_matches_sequential(G, wm):
    for g in _cases(G):
        ref = wm.canon(g)[0]
        for workers in (1, 2, 3, 8):
            for seed in (0, 1, 2, 3):
                mat, nodes, _, _ = wm.wide_model(g, workers, seed)
                assert np.array_equal(mat, ref), (g.n, workers, seed)
                assert nodes >= 1


def test_wide_model_cfi_exercises_changed_rules(G, wm):
    # CFI graphs keep deep trees with many inequivalent leaves, so workers
    # meet bests found in other items, adopt newer bests and prune under them
    rng = np.random.default_rng(11)
    events = np.zeros(3, dtype=np.int64)
    for i in range(24):
        g = G.cfi_graph(int(rng.integers(4, 9)) * 2, rng, twist=bool(i % 2))
        ref = wm.canon(g)[0]
        for workers in (2, 3, 5, 8):
            for seed in range(5):
                mat, _, _, ev = wm.wide_model(g, workers, seed)
                assert np.array_equal(mat, ref), (i, g.n, workers, seed)
                events += ev
    assert (events > 0).all(), events


def test_wide_model_relabel_invariant(G, wm):
    rng = np.random.default_rng(9)
    for g in (G.torus(4, 6), G.random_regular(26, 3, rng)):
        a = wm.wide_model(g, 4, 7)[0]
        b = wm.wide_model(G.random_relabel(g, rng), 5, 11)[0]
        assert np.array_equal(a, b)


def test_wide_model_small_batch(G, wm):
    # the graphs of the batched workload (10-64 vertices), a slice of them
    for i, g in enumerate(G.small_batch(120, seed=3000)):
        ref = wm.canon(g)[0]
        mat = wm.wide_model(g, 1 + i % 6, i)[0]
        assert np.array_equal(mat, ref), i


def test_sequential_is_maximum_leaf(G, wm):
    rng = np.random.default_rng(31)
    graphs = [G.torus(3), G.torus(3, 4), G.disjoint_union(G.torus(3), 2)]
    graphs += [G.random_regular(n, 3, rng) for n in (8, 10, 12)]
    graphs += [G.erdos_renyi(n, 0.3, rng) for n in (7, 9, 11)]
    graphs += [G.cfi_graph(4, rng, twist=t) for t in (False, True)]
    checked = 0
    for g in graphs:
        full = wm.exhaustive(g, max_leaves=300000)
        if full is None:
            continue
        assert np.array_equal(full, wm.canon(g)[0]), g.n
        checked += 1
    assert checked >= 8
