"""The wide search's opt-in counters (GCL_OPT_COUNTERS, gcl_wide_counters):
the counted items kernel gives the same canonical form as the plain one,
and its counters agree with the search's own statistics -- every stored
automorphism came from a leaf equal to the first or the best leaf, the
nodes are the search's minus the first path's, every handed-over subtree
was taken."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


def _graphs(G):
    rng = np.random.default_rng(88)
    return [G.random_regular(200, 3, rng), G.torus(12), G.tree_plus_edges(300, rng),
            G.disjoint_union(G.random_regular(16, 3, rng), 4)]


@pytest.mark.parametrize("share", [0, 1])
def test_counters_match_the_search(pkg, G, oracle_mod, share):
    api = pkg.api
    plain = pkg.Context(0, wide_min_n=1)
    counted = pkg.Context(0, wide_min_n=1)
    for ctx in (plain, counted):
        ctx.set_option(api.GCL_OPT_WIDE_SHARE, share)
    counted.set_option(api.GCL_OPT_COUNTERS, 1)
    with pytest.raises(pkg.GclError):
        plain.wide_counters()  # no counted search on this context
    for g in _graphs(G):
        want = oracle_mod.canon(g)[0]
        a = pkg.canon(g, ctx=plain)
        b = pkg.canon(g, ctx=counted)
        assert np.array_equal(a.matrix, want) and np.array_equal(b.matrix, want)
        c = counted.wide_counters()
        assert list(c) == list(api.WIDE_COUNTERS)
        assert all(v >= 0 for v in c.values()), c
        assert c["auts_first"] + c["auts_best"] == b.num_aut, c
        assert 0 < b.nodes - c["nodes"] <= g.n, (b.nodes, c)  # the first path's nodes
        assert c["items"] >= 1 and c["leaves"] >= 1, c
        assert c["gifts_taken"] == c["gifts_given"], c
        if not share:
            assert c["gifts_given"] == 0 and c["gift_wait_cycles"] == 0, c
        parts = ("refine_cycles", "orbit_cycles", "gate_cycles", "gift_wait_cycles",
                 "leaf_cycles")
        assert sum(c[p] for p in parts) <= c["warp_cycles"], c
    # counting off again: the next search is not counted
    counted.set_option(api.GCL_OPT_COUNTERS, 0)
    pkg.canon(_graphs(G)[0], ctx=counted)
    with pytest.raises(pkg.GclError):
        counted.wide_counters()


def test_counters_option_values(pkg):
    lib = pkg.api.load_library()
    ctx = pkg.Context(0)
    for bad in (-1, 2):
        assert lib.gcl_set_option(ctx.handle, pkg.api.GCL_OPT_COUNTERS, bad) == -1
