"""Graph model, DIMACS parsing (CSRGraph::fromDIMACS semantics) and arenas."""
import numpy as np
import pytest


def test_dimacs_semantics(G):
    txt = "c comment\n\np edge 5 99\nn 2 7\nn 0 3\nn 9 1\ne 1 2\ne 3 3\ne 5 1\ne 2 4\n"
    g = G.parse_dimacs(txt)
    assert g.n == 5
    assert g.rowptr.tolist() == [0, 2, 4, 4, 5, 6]
    assert g.col.tolist() == [1, 4, 0, 3, 1, 0]
    assert g.color.tolist() == [0, 7, 0, 0, 0]
    h = G.parse_dimacs(G.to_dimacs(g))
    assert np.array_equal(h.rowptr, g.rowptr) and np.array_equal(h.col, g.col)
    assert np.array_equal(h.color, g.color)


def test_duplicate_edges_rejected(G):
    with pytest.raises(ValueError):
        G.parse_dimacs("p edge 3 2\ne 1 2\ne 2 1\n")


def test_arena_roundtrip(G):
    gs = G.small_batch(30, seed=2)
    a = G.pack(gs)
    assert a.count == 30
    for i, g in enumerate(gs):
        h = a.graph(i)
        assert h.n == g.n and np.array_equal(h.rowptr, g.rowptr) and np.array_equal(h.col, g.col)
    assert a.out_offsets()[-1] == sum(g.n * g.n for g in gs)


def test_generators(G):
    rng = np.random.default_rng(0)
    r = G.random_regular(64, 3, rng)
    assert (np.diff(r.rowptr) == 3).all()
    t = G.torus(5)
    assert t.n == 25 and (np.diff(t.rowptr) == 4).all()
    u = G.disjoint_union(r, 3)
    assert u.n == 192 and u.m == 3 * r.m
    for g in G.small_batch(100, seed=1):
        assert 10 <= g.n <= 64
        assert np.diff(g.rowptr).max() <= 4
        assert g.m >= g.n - 1


def _is_tree(n, edges):
    if len(edges) != n - 1:
        return False
    parent = list(range(n))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for a, b in edges:
        ra, rb = find(a), find(b)
        if ra == rb:
            return False
        parent[ra] = rb
    return True


def test_large_trees_keep_degree_bound(G):
    rng = np.random.default_rng(17)
    for n in (129, 500, 3000):
        t = G.recursive_tree(n, rng)
        assert _is_tree(n, t)
        g = G.tree_plus_edges(n, rng)
        deg = np.diff(g.rowptr)
        assert deg.max() <= 4 and n - 1 <= g.col.size // 2 <= n + 5


def test_serving_workload_mix(G):
    W = G.serving_workload(3000, rate=1000.0, seed=3, n_max=4096)
    ns = np.array([max(W.graphs[a].n, W.graphs[b].n) for a, b in zip(W.g1, W.g2)])
    assert abs((ns <= 128).mean() - 0.90) < 0.03
    assert abs(((ns > 128) & (ns <= 2048)).mean() - 0.09) < 0.03
    assert 0 < (ns > 2048).mean() < 0.03 and ns.max() <= 4096
    assert abs(W.kind.mean() - 0.30) < 0.04
    assert (np.diff(W.arrival) >= 0).all() and W.arrival[0] == 0
    assert abs(len(W.kind) / W.arrival[-1] - 1000.0) < 100.0
    iso = np.nonzero(W.kind == 1)[0]
    assert all(W.graphs[W.g1[i]].n == W.graphs[W.g2[i]].n for i in iso)


def test_cfi_graphs_cubic_and_twist_distinguished(G, oracle_mod):
    # every vertex of a CFI graph over a cubic base has degree 3; the twisted
    # and untwisted graphs over the same connected base are not isomorphic
    # (colour refinement cannot tell them apart; the individualization search
    # does), and a relabeling of either is
    import numpy as np
    for b in (4, 6, 8):
        seed = 100 + b
        g0 = G.cfi_graph(b, np.random.default_rng(seed), twist=False)
        g1 = G.cfi_graph(b, np.random.default_rng(seed), twist=True)
        assert g0.n == g1.n == 10 * b
        assert set(np.diff(g0.rowptr).tolist()) == {3} == set(np.diff(g1.rowptr).tolist())
        c0, c1 = oracle_mod.canon(g0)[0], oracle_mod.canon(g1)[0]
        base = G.random_regular(b, 3, np.random.default_rng(seed))
        if _connected(base):
            assert not np.array_equal(c0, c1)
        h = G.random_relabel(g1, np.random.default_rng(seed + 1))
        assert np.array_equal(oracle_mod.canon(h)[0], c1)


def _connected(g):
    seen, stack = {0}, [0]
    while stack:
        u = stack.pop()
        for v in g.col[g.rowptr[u]:g.rowptr[u + 1]]:
            if int(v) not in seen:
                seen.add(int(v))
                stack.append(int(v))
    return len(seen) == g.n
