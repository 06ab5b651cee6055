"""gcl_canon_batch in two halves (GCL_OPT_BATCH_SPLIT = 1, for batches of
at least 4,096 graphs of up to 64 vertices): the second half runs
on a companion context with its own stream and workspace, over the same
arena seen from its first graph.  Every output -- dense matrices, packed
rows, labelings, both counters, statuses -- must equal the one-piece call's
and the oracle's (integer work: bit-exact), for uncoloured and coloured
graphs, empty graphs, an odd count (unequal halves) and a small ring
(max_aut 2, the full-ring rerun in both halves)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(G, count, seed, colored=False):
    gs = G.small_batch(count - 3, seed=seed)
    gs += [G.from_edges(0, []), G.from_edges(1, []), G.torus(8)]
    if colored:
        rng = np.random.default_rng(seed)
        gs = [G.from_edges(g.n, g.edges(), rng.integers(0, 3, g.n)) for g in gs]
    rng = np.random.default_rng(seed + 1)
    order = rng.permutation(len(gs))
    return [gs[i] for i in order]


@pytest.mark.parametrize("count,colored,max_aut", [(6001, False, 10000), (4096, True, 10000),
                                                    (5000, False, 2)])
def test_halves_equal_one_piece_and_oracle(pkg, G, oracle_mod, count, colored, max_aut):
    graphs = _batch(G, count, seed=900 + count, colored=colored)
    arena = G.pack(graphs)
    ctx = pkg.Context(0)
    ctx.set_option(pkg.api.GCL_OPT_BATCH_SPLIT, 1)
    split = pkg.canon_batch(arena, max_aut=max_aut, ctx=ctx, dense=True, rows=True)
    again = pkg.canon_batch(arena, max_aut=max_aut, ctx=ctx, dense=True, rows=True)
    ctx.set_option(pkg.api.GCL_OPT_BATCH_SPLIT, 0)
    whole = pkg.canon_batch(arena, max_aut=max_aut, ctx=ctx, dense=True, rows=True)
    ctx.close()
    for r in (split, again):
        assert (r.status == 0).all()
        assert np.array_equal(r.dense, whole.dense)
        assert np.array_equal(r.rows, whole.rows)
        assert np.array_equal(r.label, whole.label)
        assert np.array_equal(r.stats, whole.stats)
    out, ooff, na, nd = oracle_mod.canon_batch(arena, max_aut=max_aut)
    assert np.array_equal(split.dense[: ooff[-1]], out[: ooff[-1]])
    assert np.array_equal(split.stats[:, 0], na) and np.array_equal(split.stats[:, 1], nd)


def test_split_option_values(pkg):
    ctx = pkg.Context(0)
    for v in (0, 1):
        ctx.set_option(pkg.api.GCL_OPT_BATCH_SPLIT, v)
    with pytest.raises(pkg.api.GclError):
        ctx.set_option(pkg.api.GCL_OPT_BATCH_SPLIT, 2)
    ctx.close()
