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
independent of the order in which the leaves are met.  The automorphisms the
model stores are also fed to the library's host Schreier-Sims: under every
schedule they generate the whole automorphism group, which is what
gcl_group_order relies on.
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


@pytest.mark.parametrize("gate", [True, False])
def test_wide_model_matches_sequential(G, wm, gate):
    # with the level gate (the GPU's order) and without it: the rules alone
    # carry the result
    for g in _cases(G):
        ref = wm.canon(g)[0]
        for workers in (1, 2, 3, 8):
            for seed in (0, 1, 2, 3):
                mat, nodes, _, _ = wm.wide_model(g, workers, seed, gate=gate)
                assert np.array_equal(mat, ref), (g.n, workers, seed)
                assert nodes >= 1


@pytest.mark.parametrize("gate", [True, False])
def test_wide_model_cfi_exercises_changed_rules(G, wm, gate):
    # CFI graphs keep deep trees with many inequivalent leaves, so workers
    # meet bests found in other items, adopt newer bests and prune under them
    rng = np.random.default_rng(11)
    events = np.zeros(3, dtype=np.int64)
    for i in range(24):
        g = G.cfi_graph(int(rng.integers(4, 9)) * 2, rng, twist=bool(i % 2))
        ref = wm.canon(g)[0]
        for workers in (2, 3, 5, 8):
            for seed in range(5):
                mat, _, _, ev = wm.wide_model(g, workers, seed, gate=gate)
                assert np.array_equal(mat, ref), (i, g.n, workers, seed)
                events += ev
    assert (events > 0).all(), events


def test_wide_model_gate_serialises_trees(G, wm):
    # On trees each level holds about one item, so the level gate runs the
    # items one after another (rounds ~ nodes); without it the items run
    # together and the rounds fall to about the first path's depth.
    rng = np.random.default_rng(2)
    g = G.from_edges(300, G.recursive_tree(300, rng))
    ref = wm.canon(g)
    r_gate, r_free = [], []
    m1, nodes_gate, _, _ = wm.wide_model(g, 64, 0, gate=True, rounds=r_gate)
    m2, nodes_free, _, _ = wm.wide_model(g, 64, 0, gate=False, rounds=r_free)
    assert np.array_equal(m1, ref[0]) and np.array_equal(m2, ref[0])
    depth = r_gate[1]
    assert r_gate[0] > 0.5 * nodes_gate
    assert r_free[0] <= depth + 2 and nodes_free <= 1.5 * ref[3]


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


def _brute_order(g):
    import itertools
    n = g.n
    e = {tuple(x) for x in g.edges().tolist()}
    e |= {(b, a) for a, b in e}
    col = g.color if g.color is not None else np.zeros(n, int)
    return sum(1 for p in itertools.permutations(range(n))
               if all(col[p[v]] == col[v] for v in range(n)) and all((p[a], p[b]) in e for a, b in e))


def test_wide_model_automorphisms_generate_the_group(G, wm, pkg):
    # gcl_group_order rests on this: the automorphisms a wide search stores
    # generate Aut(G), whatever the schedule.  The model's store goes through
    # the library's host Schreier-Sims (gcl_perm_group_order, no GPU needed).
    import math
    rng = np.random.default_rng(21)
    cases = [(G.torus(k), 8 * k * k) for k in (5, 6, 7)]  # (C4 x C4 is Q4: 384)
    cases += [(G.from_edges(n, [(i, (i + 1) % n) for i in range(n)]), 2 * n) for n in (5, 12)]
    cases += [(G.from_edges(n, [(i, j) for i in range(n) for j in range(i + 1, n)]),
               math.factorial(n)) for n in (4, 7)]
    cases += [(G.from_edges(9, [(0, i) for i in range(1, 9)]), math.factorial(8))]
    cases += [(G.from_edges(100, []), math.factorial(100))]  # S_100: a long base
    cube = [(a, a ^ (1 << b)) for a in range(16) for b in range(4) if a < a ^ (1 << b)]
    cases += [(G.from_edges(16, cube), 384)]
    c5 = G.from_edges(5, [(i, (i + 1) % 5) for i in range(5)])
    cases += [(G.disjoint_union(c5, k), 10 ** k * math.factorial(k)) for k in (2, 3)]
    for _ in range(25):
        n = int(rng.integers(2, 8))
        g = G.erdos_renyi(n, float(rng.uniform(0.15, 0.7)), rng)
        if rng.random() < 0.4:
            g = G.from_edges(n, g.edges(), rng.integers(0, 2, n))
        cases.append((g, _brute_order(g)))
    for i, (g, want) in enumerate(cases):
        for workers, seed in ((1, 0), (3, i + 1), (8, 2 * i + 5)):
            _, _, naut, _, store = wm.wide_model(g, workers, seed, cap=20000, auts=True)
            assert naut < 20000
            assert pkg.perm_group_order(store.astype(np.uint16)) == want, (i, g.n, workers)


def test_wide_model_group_order_schedule_independent_on_cfi(G, wm, pkg):
    rng = np.random.default_rng(77)
    for i in range(8):
        g = G.cfi_graph(int(rng.integers(3, 7)) * 2, rng, twist=bool(i % 2))
        h = G.random_relabel(g, rng)
        orders = set()
        for x, workers, seed in ((g, 1, 0), (g, 4, 3 + i), (h, 7, 11 + i)):
            _, _, naut, _, store = wm.wide_model(x, workers, seed, cap=20000, auts=True)
            assert naut < 20000
            orders.add(pkg.perm_group_order(store.astype(np.uint16)))
        assert len(orders) == 1, (i, orders)


@pytest.mark.parametrize("gate", [True, False])
def test_wide_model_donation_matches_sequential(G, wm, gate):
    # busy workers hand untried children to idle ones (work sharing below the
    # first path's siblings); every schedule still gives the sequential form
    rng = np.random.default_rng(33)
    graphs = [G.disjoint_union(G.random_regular(10, 3, rng), k) for k in (2, 3, 4)]
    graphs += [G.cfi_graph(b, rng, twist=bool(b % 4)) for b in (6, 8, 12)]
    graphs += [G.tree_plus_edges(n, rng) for n in (60, 150)] + [G.torus(6)]
    for g in graphs:
        ref = wm.canon(g)[0]
        for workers in (2, 5, 16):
            for seed in (0, 1, 2):
                mat = wm.wide_model(g, workers, seed, gate=gate, donate=True)[0]
                assert np.array_equal(mat, ref), (g.n, workers, seed)


def test_wide_model_donation_splits_unions(G, wm):
    # unions of identical components: a few items hold most of the tree;
    # handing over children after a level's first child is done spreads them
    rng = np.random.default_rng(3)
    g = G.disjoint_union(G.random_regular(32, 3, rng), 5)
    ref = wm.canon(g)[0]
    r0, r1 = [], []
    m0, nodes0, _, _ = wm.wide_model(g, 592, 0, cap=100000, gate=False, rounds=r0)
    m1, nodes1, _, _ = wm.wide_model(g, 592, 0, cap=100000, gate=False, donate=True, rounds=r1)
    assert np.array_equal(m0, ref) and np.array_equal(m1, ref)
    assert r1[0] * 3 < r0[0] and nodes1 < nodes0


def test_wide_model_replayed_parents_match(G, wm):
    # the GPU's receiver rebuilds a handed-over parent from the first leaf:
    # back to the level shared with the first path, then the remaining
    # vertices individualized -- the codes must be the giver's, and the
    # canonical form the sequential one
    rng = np.random.default_rng(34)
    graphs = [G.disjoint_union(G.random_regular(10, 3, rng), k) for k in (2, 3, 4)]
    graphs += [G.disjoint_union(G.random_regular(32, 3, rng), 5)]
    graphs += [G.cfi_graph(b, rng) for b in (6, 10)] + [G.tree_plus_edges(150, rng)]
    for g in graphs:
        ref = wm.canon(g)[0]
        for workers, seed, gate in ((3, 1, True), (16, 2, False), (64, 0, False)):
            r = []
            mat, _, _, ev = wm.wide_model(g, workers, seed, gate=gate, donate=2, rounds=r)
            assert np.array_equal(mat, ref), (g.n, workers, seed, gate)
            assert ev[3] == 0, (g.n, workers, seed)
    # the unions hand work over, so parents are rebuilt
    r0, r1 = [], []
    g = graphs[3]
    wm.wide_model(g, 64, 0, gate=False, rounds=r0)
    wm.wide_model(g, 64, 0, gate=False, donate=2, rounds=r1)
    assert r1[0] < r0[0]


def test_wide_model_automatic_gate(G, wm):
    # gate 2 (the GPU's automatic rule): off for a tree (about one item per
    # level), on for a torus (many items per level) -- same rounds as the
    # explicit settings it picks
    rng = np.random.default_rng(2)
    tree = G.from_edges(300, G.recursive_tree(300, rng))
    torus = G.torus(10)
    for g, picks in ((tree, 0), (torus, 1)):
        r_auto, r_pick = [], []
        m1 = wm.wide_model(g, 64, 0, gate=2, rounds=r_auto)[0]
        m2 = wm.wide_model(g, 64, 0, gate=picks, rounds=r_pick)[0]
        assert np.array_equal(m1, m2) and r_auto[0] == r_pick[0], (g.n, picks)


def test_wide_model_probe_matches_sequential_and_prunes_tori(G, wm):
    # The probe (GCL_OPT_WIDE_PROBE): under the gate each level's first item
    # runs alone before the rest of the level (at most 2D rounds), so the
    # automorphisms it finds prune its siblings.  Every schedule still gives
    # the sequential form; on tori one sibling per level covers the whole
    # cell, and the nodes fall to the sequential count.
    rng = np.random.default_rng(77)
    cases = _cases(G) + [G.cfi_graph(12, rng), G.disjoint_union(G.random_regular(16, 3, rng), 4)]
    for g in cases:
        ref = wm.canon(g)[0]
        for workers, seed in ((1, 0), (3, 1), (8, 2), (64, 0), (64, 3)):
            mat = wm.wide_model(g, workers, seed, gate=True, probe=True)[0]
            assert np.array_equal(mat, ref), (g.n, workers, seed)
    for k in (16, 32):
        g = G.torus(k)
        seq_nodes = wm.canon(g)[3]
        _, nodes_plain, _, _ = wm.wide_model(g, 592, 0, gate=True)
        _, nodes_probe, _, _ = wm.wide_model(g, 592, 0, gate=True, probe=True)
        assert nodes_probe == seq_nodes < nodes_plain, (k, nodes_probe, seq_nodes, nodes_plain)
