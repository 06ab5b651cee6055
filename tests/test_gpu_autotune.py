"""Autotuning of the batched path's launch shapes (gcl_autotune): the choice
moves only the launch shape, so results stay bit-exact -- canonical rows,
labelings and statistics equal those of an untuned context."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_keeps_results(pkg, G):
    rng = np.random.default_rng(31)
    graphs = G.small_batch(300, seed=31)
    graphs += [G.tree_plus_edges(int(rng.integers(65, 250)), rng) for _ in range(20)]
    graphs += [G.erdos_renyi(int(rng.integers(260, 900)), 0.01, rng) for _ in range(6)]
    graphs += [G.random_regular(130, 3, rng), G.torus(12)]
    plain = pkg.Context(0, wide_min_n=pkg.api.GCL_MAX_N + 1)
    ref = pkg.canon_batch(graphs, ctx=plain, dense=False, rows=True)
    tuned = pkg.Context(0, wide_min_n=pkg.api.GCL_MAX_N + 1)
    t = tuned.autotune(graphs, repeats=1)
    assert t["w64_blocks_per_sm"] >= 1 and t["w64_ms"] > 0
    assert t["sp_ms"][0] > 0 and t["sp_ms"][1] > 0  # buckets n <= 256 and <= 1024 timed
    assert t["sp_stage"][0] in (0, 1) and t["sp_stage"][3] == -1  # no graph above 4096
    res = pkg.canon_batch(graphs, ctx=tuned, dense=False, rows=True)
    assert np.array_equal(res.rows, ref.rows)
    assert np.array_equal(res.label, ref.label)
    assert np.array_equal(res.stats, ref.stats)
    # a saved choice applies to another context
    other = pkg.Context(0, wide_min_n=pkg.api.GCL_MAX_N + 1)
    other.set_tuning(t)
    assert np.array_equal(pkg.canon_batch(graphs, ctx=other, dense=False, rows=True).rows,
                          ref.rows)
