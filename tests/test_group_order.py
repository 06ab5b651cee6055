"""Automorphism group order.

The reference never computes |Aut(G)| (it prints a traversal-dependent count
of stored automorphisms), so these orders are pinned by mathematics: the
host Schreier-Sims part against groups of known order and a brute-force
closure (CPU, no GPU), and the whole entry point (GPU) against textbook
automorphism groups and brute force over all permutations for n <= 8."""
import itertools
import math

import numpy as np
import pytest


def _closure_order(gens, n):
    """Order of <gens> by breadth-first closure (small groups only)."""
    ident = tuple(range(n))
    seen = {ident}
    frontier = [ident]
    while frontier:
        nxt = []
        for p in frontier:
            for g in gens:
                q = tuple(g[p[i]] for i in range(n))
                if q not in seen:
                    seen.add(q)
                    nxt.append(q)
        frontier = nxt
    return len(seen)


def test_perm_group_order_known_groups(pkg):
    n = 7
    cyc = [(i + 1) % n for i in range(n)]
    swap = [1, 0] + list(range(2, n))
    assert pkg.perm_group_order([cyc, swap]) == math.factorial(n)  # S_7
    assert pkg.perm_group_order([cyc]) == n  # C_7
    refl = [(-i) % n for i in range(n)]
    assert pkg.perm_group_order([cyc, refl]) == 2 * n  # D_7
    assert pkg.perm_group_order(np.zeros((0, 5), np.uint16)) == 1
    # a direct product of 40 transpositions: 2^40 (big integer)
    m = 80
    gens = []
    for k in range(40):
        p = list(range(m))
        p[2 * k], p[2 * k + 1] = p[2 * k + 1], p[2 * k]
        gens.append(p)
    assert pkg.perm_group_order(gens) == 2 ** 40
    # S_30 from a transposition and a 30-cycle
    m = 30
    assert pkg.perm_group_order([[(i + 1) % m for i in range(m)],
                                 [1, 0] + list(range(2, m))]) == math.factorial(30)


def test_perm_group_order_random_vs_closure(pkg):
    rng = np.random.default_rng(9)
    for _ in range(40):
        n = int(rng.integers(2, 8))
        gens = [list(rng.permutation(n)) for _ in range(int(rng.integers(1, 4)))]
        assert pkg.perm_group_order(gens) == _closure_order([tuple(g) for g in gens], n)


def test_perm_group_order_rejects_non_permutations(pkg):
    with pytest.raises(pkg.GclError):
        pkg.perm_group_order([[0, 0, 1]])


def _brute_aut(g):
    n = g.n
    e = {tuple(x) for x in g.edges().tolist()}
    e |= {(b, a) for a, b in e}
    col = g.color if g.color is not None else np.zeros(n, int)
    cnt = 0
    for p in itertools.permutations(range(n)):
        if any(col[p[v]] != col[v] for v in range(n)):
            continue
        if all((p[a], p[b]) in e for a, b in e):
            cnt += 1
    return cnt


@pytest.mark.gpu
def test_group_order_known_graphs(pkg, G):
    ctx = pkg.Context(0)
    cases = [(G.torus(k), 8 * k * k) for k in (5, 6, 8)]
    cases += [(G.from_edges(n, [(i, (i + 1) % n) for i in range(n)]), 2 * n) for n in (5, 12, 40)]
    cases += [(G.from_edges(n, [(i, j) for i in range(n) for j in range(i + 1, n)]), math.factorial(n))
              for n in (3, 8, 20)]
    cases += [(G.from_edges(n, []), math.factorial(n)) for n in (1, 2, 10, 33)]
    cases += [(G.from_edges(10, [(0, i) for i in range(1, 10)]), math.factorial(9))]
    cases += [(G.from_edges(10, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 0), (0, 5), (1, 6), (2, 7),
                                 (3, 8), (4, 9), (5, 7), (7, 9), (9, 6), (6, 8), (8, 5)]), 120)]
    cube = [(a, a ^ (1 << b)) for a in range(8) for b in range(3) if a < a ^ (1 << b)]
    cases += [(G.from_edges(8, cube), 48)]
    cases += [(G.from_edges(12, [(i, i + 1) for i in range(11)]), 2)]
    rng = np.random.default_rng(4)
    comp = G.random_regular(10, 3, rng)
    a1 = pkg.group_order(comp, ctx=ctx)
    for k in (2, 3, 4):  # k identical components: a1^k * k!
        cases.append((G.disjoint_union(comp, k), a1 ** k * math.factorial(k)))
    for g, want in cases:
        # small groups: a Schreier-Sims completion finishes and confirms
        assert pkg.group_order(g, ctx=ctx, return_checked=True) == (want, 1), (g.n, want)


@pytest.mark.gpu
def test_group_order_brute_force_small(pkg, G):
    ctx = pkg.Context(0)
    rng = np.random.default_rng(12)
    for _ in range(40):
        n = int(rng.integers(1, 8))
        g = G.erdos_renyi(n, float(rng.uniform(0.1, 0.7)), rng)
        if rng.random() < 0.4:
            g = G.from_edges(n, g.edges(), rng.integers(0, 2, n))
        assert pkg.group_order(g, ctx=ctx) == _brute_aut(g)
    for g in G.small_batch(30, seed=5):  # trees: relabeling leaves the order alone
        assert pkg.group_order(g, ctx=ctx) == pkg.group_order(G.random_relabel(g, rng), ctx=ctx)


def test_perm_group_order_large_orbits_and_many_generators(pkg):
    # cases the completion must finish quickly: a vertex-transitive group of
    # 4096 points (torus 64x64: translations, a rotation, a reflection) and
    # 30 disjoint 5-cycles with their dihedral symmetries and the swaps of
    # components as separate generators
    import time
    k = 64
    n = k * k
    idx = np.arange(n)
    x, y = idx // k, idx % k
    gens = [((x + 1) % k) * k + y, x * k + (y + 1) % k, y * k + (-x) % k, x * k + (-y) % k]
    t = time.time()
    assert pkg.perm_group_order(np.array(gens)) == 8 * n
    gens = []
    c = 30
    for comp in range(c):
        for g in ([1, 2, 3, 4, 0], [0, 4, 3, 2, 1]):
            p = np.arange(5 * c)
            p[5 * comp:5 * comp + 5] = 5 * comp + np.array(g)
            gens.append(p)
    for comp in range(c - 1):
        p = np.arange(5 * c)
        p[5 * comp:5 * comp + 5], p[5 * comp + 5:5 * comp + 10] = (np.arange(5 * comp + 5, 5 * comp + 10),
                                                                    np.arange(5 * comp, 5 * comp + 5))
        gens.append(p)
    assert pkg.perm_group_order(np.array(gens)) == 10 ** c * math.factorial(c)
    assert time.time() - t < 20
