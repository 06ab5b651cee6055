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
    return pkg.Context(0)


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
