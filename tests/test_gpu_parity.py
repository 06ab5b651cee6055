"""CUDA path vs the oracle, through the C ABI.  Integer work: bit-exact.

Compared per graph: canonical matrix, best-leaf labeling, number of stored
automorphisms and number of search-tree nodes (the last two pin the search
order, not only the result)."""
import hashlib

import numpy as np
import pytest

from conftest import golden_graph

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(pkg):
    # sequential traversal for every size: statistics comparable with the oracle
    return pkg.Context(0, wide_min_n=pkg.api.GCL_MAX_N + 1)


def _check_batch(pkg, G, oracle_mod, graphs, ctx, max_aut=10000):
    res = pkg.canon_batch(graphs, max_aut=max_aut, ctx=ctx)
    arena = res.arena
    out, ooff, na, nd = oracle_mod.canon_batch(arena, max_aut=max_aut)
    assert (res.status == 0).all()
    assert np.array_equal(res.dense[: ooff[-1]], out[: ooff[-1]])
    assert np.array_equal(res.stats[:, 0], na)
    assert np.array_equal(res.stats[:, 1], nd)
    return res


def test_golden_batch(pkg, G, golden, ctx):
    by_aut = {}
    for rec in golden:
        by_aut.setdefault(rec["max_aut"], []).append(rec)
    for max_aut, recs in by_aut.items():
        graphs = [golden_graph(G, r) for r in recs]
        res = pkg.canon_batch(graphs, max_aut=max_aut, ctx=ctx)
        assert (res.status == 0).all()
        for i, r in enumerate(recs):
            m = res.matrix(i)
            assert hashlib.sha256(m.tobytes()).hexdigest() == r["matrix_sha256"], r["name"]
            assert res.labeling(i).tolist() == r["label"], r["name"]
            assert res.stats[i].tolist() == [r["num_aut"], r["nodes"]], r["name"]


def test_small_batch_vs_oracle(pkg, G, oracle_mod, ctx):
    _check_batch(pkg, G, oracle_mod, G.small_batch(3000, seed=3000), ctx)


def test_dense_random_vs_oracle(pkg, G, oracle_mod, ctx):
    rng = np.random.default_rng(42)
    graphs = []
    for i in range(600):
        n = int(rng.integers(1, 65))
        g = G.erdos_renyi(n, float(rng.uniform(0.0, 0.9)), rng)
        col = rng.integers(-2, 3, n) if i % 3 == 0 else None
        graphs.append(G.from_edges(n, g.edges(), col))
    _check_batch(pkg, G, oracle_mod, graphs, ctx)


def test_symmetric_and_small_max_aut(pkg, G, oracle_mod, ctx):
    rng = np.random.default_rng(3)
    graphs = [G.torus(k) for k in (3, 4, 5, 6, 7, 8)]
    graphs += [G.from_edges(n, []) for n in (1, 2, 17, 32, 33, 64)]
    graphs += [G.from_edges(n, [(i, j) for i in range(n) for j in range(i + 1, n)])
               for n in (2, 9, 32, 33, 64)]
    graphs += [G.disjoint_union(G.random_regular(8, 3, rng), k) for k in (2, 4, 8)]
    graphs += [G.from_edges(64, [(i, (i + 1) % 64) for i in range(64)])]
    for max_aut in (1, 2, 3, 7, 300, 10000):
        _check_batch(pkg, G, oracle_mod, graphs, ctx, max_aut=max_aut)


def test_relabel_invariance_and_iso(pkg, G, ctx):
    rng = np.random.default_rng(9)
    gs = G.small_batch(200, seed=55)
    hs = [G.random_relabel(g, rng) for g in gs]
    a = pkg.canon_batch(gs, ctx=ctx)
    b = pkg.canon_batch(hs, ctx=ctx)
    assert np.array_equal(a.dense, b.dense)
    assert pkg.is_isomorphic(gs[0], hs[0], ctx=ctx)
    moved = G.move_one_edge(gs[1], rng)
    assert not pkg.is_isomorphic(gs[1], moved, ctx=ctx)
    small = next(g for g in gs if g.n < 64)
    assert not pkg.is_isomorphic(small, G.from_edges(small.n + 1, small.edges()), ctx=ctx)


def test_canon_one_matches_oracle(pkg, G, oracle_mod, ctx):
    for g in G.small_batch(20, seed=8) + [G.from_edges(0, []), G.from_edges(1, [])]:
        r = pkg.canon(g, ctx=ctx)
        mat, _, na, nd = oracle_mod.canon(g)
        assert np.array_equal(r.matrix, mat)
        assert (r.num_aut, r.nodes) == (na, nd)
        assert pkg.Nauty_Parallel(g) == mat.tobytes()


def test_bad_input_rejected(pkg, G, ctx):
    g = G.from_edges(4, [(0, 1), (1, 2)])
    bad = G.Graph(4, np.array([0, 1, 2, 2, 2], np.int32), np.array([1, 0], np.int32) * 0 + 1)
    with pytest.raises(pkg.GclError):
        pkg.canon(bad, ctx=ctx)  # one-directional / self loop edges
    asym = G.Graph(3, np.array([0, 1, 1, 1], np.int32), np.array([1], np.int32))
    with pytest.raises(pkg.GclError):
        pkg.canon(asym, ctx=ctx)
    # the context is still usable afterwards
    assert pkg.canon(g, ctx=ctx).matrix.shape == (4, 4)


# ---- graphs above 64 vertices (the sparse warp kernel) --------------------

def test_large_random_vs_oracle(pkg, G, oracle_mod, ctx):
    rng = np.random.default_rng(77)
    graphs = []
    for i in range(60):
        n = int(rng.integers(65, 260))
        fam = i % 5
        if fam == 0:
            g = G.erdos_renyi(n, float(rng.uniform(0.01, 0.08)), rng)
        elif fam == 1:
            g = G.random_regular(n + (n % 2), 3, rng)
        elif fam == 2:
            g = G.from_edges(n, G.erdos_renyi(n, 0.05, rng).edges(), rng.integers(0, 3, n))
        elif fam == 3:
            g = G.tree_plus_edges(n, rng)
        else:
            g = G.erdos_renyi(n, float(rng.uniform(0.2, 0.5)), rng)
        graphs.append(g)
    _check_batch(pkg, G, oracle_mod, graphs, ctx)


def test_large_symmetric_vs_oracle(pkg, G, oracle_mod, ctx):
    rng = np.random.default_rng(5)
    graphs = [G.torus(k) for k in (9, 10, 12, 16)] + [G.torus(7, 11)]
    graphs += [G.disjoint_union(G.random_regular(16, 3, rng), k) for k in (5, 8)]
    graphs += [G.disjoint_union(G.random_regular(64, 4, rng), 2)]
    graphs += [G.from_edges(n, []) for n in (65, 100)]
    graphs += [G.from_edges(70, [(i, j) for i in range(70) for j in range(i + 1, 70)])]
    graphs += [G.from_edges(200, [(0, i) for i in range(1, 200)])]
    graphs += [G.from_edges(128, [(i, (i + 1) % 128) for i in range(128)])]
    for max_aut in (10000, 3, 1):
        _check_batch(pkg, G, oracle_mod, graphs, ctx, max_aut=max_aut)


def test_mixed_small_and_large(pkg, G, oracle_mod, ctx):
    rng = np.random.default_rng(12)
    graphs = G.small_batch(300, seed=4) + [G.erdos_renyi(int(rng.integers(65, 200)), 0.04, rng)
                                          for _ in range(30)]
    order = rng.permutation(len(graphs))
    _check_batch(pkg, G, oracle_mod, [graphs[i] for i in order], ctx)


def test_er256_triple_iso(pkg, G, oracle_mod, ctx):
    # plain single-graph workload: G(256, 0.05), a relabeling, one edge moved
    rng = np.random.default_rng(1000)
    er = G.erdos_renyi(256, 0.05, rng)
    rel = G.random_relabel(er, rng)
    moved = G.move_one_edge(er, rng)
    for g in (er, rel, moved):
        r = pkg.canon(g, ctx=ctx)
        mat, _, na, nd = oracle_mod.canon(g)
        assert np.array_equal(r.matrix, mat) and (r.num_aut, r.nodes) == (na, nd)
    assert pkg.is_isomorphic(er, rel, ctx=ctx)
    assert not pkg.is_isomorphic(er, moved, ctx=ctx)


def test_uncoloured_single_large(pkg, G, oracle_mod, ctx):
    # one graph per call with no colour array at all (color == NULL)
    rng = np.random.default_rng(21)
    for g in (G.torus(9), G.random_regular(100, 3, rng), G.erdos_renyi(120, 0.05, rng)):
        r = pkg.canon(g, ctx=ctx)
        mat, _, na, nd = oracle_mod.canon(g)
        assert np.array_equal(r.matrix, mat) and (r.num_aut, r.nodes) == (na, nd)


def test_packed_rows_match_dense(pkg, G, ctx):
    rng = np.random.default_rng(8)
    graphs = G.small_batch(200, seed=71) + [G.erdos_renyi(int(rng.integers(65, 300)), 0.03, rng)
                                           for _ in range(10)] + [G.torus(12), G.from_edges(64, [])]
    res = pkg.canon_batch(graphs, ctx=ctx, rows=True)
    for g in range(res.arena.count):
        n = res.arena.graph(g).n
        assert np.array_equal(pkg.api.unpack_rows(res.packed(g), n), res.matrix(g))
