"""The CPU oracle (oracle/canon_oracle.c) against the reference's golden
vectors, and against the reference itself where it was compiled here."""
import hashlib

import numpy as np
import pytest

from conftest import golden_graph


def test_port_matches_golden(G, golden, oracle_mod):
    assert len(golden) > 150
    for rec in golden:
        g = golden_graph(G, rec)
        mat, lab, na, nodes = oracle_mod.canon(g, max_aut=rec["max_aut"], kind="port")
        assert lab.tolist() == rec["label"], rec["name"]
        assert hashlib.sha256(mat.tobytes()).hexdigest() == rec["matrix_sha256"], rec["name"]
        assert (na, nodes) == (rec["num_aut"], rec["nodes"]), rec["name"]


def test_golden_matrix_is_label_permutation(G, golden, oracle_mod):
    # canonical matrix == input relabelled by the best leaf (certificate validity)
    for rec in golden[:60]:
        g = golden_graph(G, rec)
        mat, lab, _, _ = oracle_mod.canon(g, max_aut=rec["max_aut"])
        a = g.adjacency()
        assert np.array_equal(mat, a[np.ix_(lab, lab)]), rec["name"]


@pytest.mark.skipif(not __import__("oracle").available("reference"),
                    reason="reference build (oracle/_ref) not present")
def test_port_matches_reference_fresh_seeds(G, oracle_mod):
    rng = np.random.default_rng(777)
    graphs = G.small_batch(300, seed=91)
    for i in range(40):
        n = int(rng.integers(1, 70))
        g = G.erdos_renyi(n, float(rng.uniform(0.02, 0.6)), rng)
        col = rng.integers(0, 3, n) if i % 2 else None
        graphs.append(G.from_edges(n, g.edges(), col))
    # deep trees with many inequivalent leaves, and strongly regular / cube families
    graphs += [G.cfi_graph(b, rng, twist=bool(b % 4)) for b in (4, 6, 8, 10, 12)]
    from test_gpu_hard_families import _families
    graphs += _families(G)
    for g in graphs:
        a = oracle_mod.canon(g, kind="port")
        b = oracle_mod.canon(g, kind="reference")
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        assert a[2:] == b[2:]


def test_relabel_invariance(G, oracle_mod):
    rng = np.random.default_rng(5)
    for g in G.small_batch(50, seed=17):
        h = G.random_relabel(g, rng)
        assert np.array_equal(oracle_mod.canon(g)[0], oracle_mod.canon(h)[0])


@pytest.mark.skipif(not __import__("oracle").available("reference"),
                    reason="reference build (oracle/_ref) not present")
def test_port_matches_reference_across_families_and_rings(G, oracle_mod):
    # labels, matrices and both counters, with max_aut small enough for the
    # reference's automorphism ring to wrap (num_aut % max_aut)
    from test_gpu_hard_families import _cube, _rook
    rng = np.random.default_rng(2026)
    for i in range(900):
        f = i % 9
        if f == 0:
            n = int(rng.integers(1, 90))
            g = G.erdos_renyi(n, float(rng.uniform(0, .6)), rng)
        elif f == 1:
            n = int(rng.integers(4, 60))
            g = G.from_edges(n, G.erdos_renyi(n, float(rng.uniform(0.05, .5)), rng).edges(),
                             rng.integers(0, 4, n))
        elif f == 2:
            g = G.tree_plus_edges(int(rng.integers(5, 120)), rng)
        elif f == 3:
            g = G.random_regular(int(rng.integers(3, 30)) * 2, int(rng.choice([3, 4])), rng)
        elif f == 4:
            g = G.torus(int(rng.integers(3, 9)), int(rng.integers(3, 9)))
        elif f == 5:
            g = G.disjoint_union(G.random_regular(int(rng.integers(3, 7)) * 2, 3, rng),
                                 int(rng.integers(2, 4)))
        elif f == 6:
            g = G.cfi_graph(int(rng.integers(2, 6)) * 2, rng, bool(rng.integers(2)))
        elif f == 7:
            g = _rook(G, int(rng.integers(2, 6)), int(rng.integers(2, 6)))
        else:
            g = G.random_relabel(_cube(G, int(rng.integers(2, 6))), rng)
        ma = int(rng.choice([1, 2, 3, 7, 10000]))
        a = oracle_mod.canon(g, max_aut=ma, kind="port")
        b = oracle_mod.canon(g, max_aut=ma, kind="reference")
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (i, g.n, ma)
        assert a[2:] == b[2:], (i, g.n, ma)
