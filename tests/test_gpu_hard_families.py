"""Graph families with deep, wide search trees through every GPU path, bit
for bit against the oracle: Cai-Fuerer-Immerman graphs (refinement leaves
them almost undivided), Paley graphs, rook's graphs, hypercubes and
strongly symmetric unions.  The oracle itself is checked on the CFI graphs
against the reference's own sequential code (tests/test_oracle.py)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


def _paley(G, q):
    sq = {(x * x) % q for x in range(1, q)}
    return G.from_edges(q, [(i, j) for i in range(q) for j in range(i + 1, q) if (j - i) % q in sq])


def _rook(G, a, b):
    n = a * b
    return G.from_edges(n, [(i, j) for i in range(n) for j in range(i + 1, n)
                            if (i // b == j // b) != (i % b == j % b)])


def _cube(G, d):
    n = 1 << d
    return G.from_edges(n, [(a, a ^ (1 << k)) for a in range(n) for k in range(d) if a < a ^ (1 << k)])


def _families(G):
    rng = np.random.default_rng(61)
    out = [G.cfi_graph(b, rng, twist=bool(i % 2)) for i, b in enumerate((4, 6, 8, 10, 12, 16, 20))]
    out += [_paley(G, q) for q in (13, 17, 29, 37, 61)]
    out += [_rook(G, a, b) for a, b in ((3, 5), (4, 4), (6, 7), (8, 8))]
    out += [_cube(G, d) for d in (4, 5, 6, 7)]
    out += [G.disjoint_union(_paley(G, 13), 3), G.disjoint_union(G.cfi_graph(4, rng), 2)]
    return out


def test_hard_families_batched_vs_oracle(pkg, G, oracle_mod):
    # the sequential kernels (w64 for n <= 64, the sparse kernel above)
    graphs = _families(G)
    ctx = pkg.Context(0, wide_min_n=pkg.api.GCL_MAX_N + 1)
    res = pkg.canon_batch(graphs, ctx=ctx)
    assert (res.status == 0).all()
    for k, g in enumerate(graphs):
        mat, lab, na, nodes = oracle_mod.canon(g)
        assert np.array_equal(res.matrix(k), mat), k
        assert np.array_equal(res.labeling(k), lab), k
        assert tuple(res.stats[k]) == (na, nodes), k


@pytest.mark.parametrize("gate", [1, 0, 2])
def test_hard_families_wide_vs_oracle(pkg, G, oracle_mod, gate):
    ctx = pkg.Context(0, wide_min_n=1)
    ctx.set_option(pkg.api.GCL_OPT_WIDE_GATE, gate)
    for k, g in enumerate(_families(G)):
        assert np.array_equal(pkg.canon(g, ctx=ctx).matrix, oracle_mod.canon(g)[0]), k


def test_cfi_pairs_iso_verdicts(pkg, G):
    # twisted and untwisted CFI graphs over one connected cubic base: the
    # classic pairs colour refinement cannot separate
    ctx = pkg.Context(0)
    for b in (6, 10, 16):
        seed = 300 + b
        g0 = G.cfi_graph(b, np.random.default_rng(seed), twist=False)
        g1 = G.cfi_graph(b, np.random.default_rng(seed), twist=True)
        h = G.random_relabel(g1, np.random.default_rng(seed + 1))
        assert pkg.is_isomorphic(g1, h, ctx=ctx)
        base = G.random_regular(b, 3, np.random.default_rng(seed))
        from test_graphs import _connected
        if _connected(base):
            assert not pkg.is_isomorphic(g0, g1, ctx=ctx)
