"""The serving loop with big_wide = 1: requests of 257-2048 vertices go
through the wide search with the automatic level gate instead of the batched
sequential search.  Canonical forms must equal those of each graph canonized
alone (the wide search's labeling is one of the equivalent best leaves, so
the labelings are checked by applying them); the timing of a burst of trees
is printed beside the default configuration's."""
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


def _drain(srv, n_expected, timeout_polls=60000):
    got = {}
    for _ in range(timeout_polls):
        for r, rows, lab in srv.poll(timeout_ms=10):
            got[r.id] = (r, rows, lab)
        if len(got) >= n_expected:
            break
    assert len(got) == n_expected
    return got


def _burst(pkg, graphs, **cfg):
    srv = pkg.Server(0, **cfg)
    t = time.perf_counter()
    for i, g in enumerate(graphs):
        srv.submit_canon(i, g)
    got = _drain(srv, len(graphs))
    dt = time.perf_counter() - t
    st = srv.stats()
    srv.close()
    return got, dt, st


def test_big_wide_forms_equal_alone(pkg, G):
    rng = np.random.default_rng(90)
    graphs = [G.tree_plus_edges(int(rng.integers(257, 2048)), rng) for _ in range(24)]
    graphs += [G.random_regular(400, 3, rng), G.torus(20), G.cfi_graph(30, rng)]
    graphs += G.small_batch(100, seed=90)
    ctx = pkg.Context(0)
    ref = [pkg.canon_batch([g], ctx=ctx, dense=False, rows=True).packed(0).copy() for g in graphs]
    got, dt_wide, st = _burst(pkg, graphs, big_wide=1)
    for i, g in enumerate(graphs):
        r, rows, lab = got[i]
        assert r.status == 0
        assert np.array_equal(rows, ref[i]), i
        assert sorted(lab.tolist()) == list(range(g.n))
        a = g.adjacency()
        assert np.array_equal(pkg.api.unpack_rows(rows, g.n), a[np.ix_(lab, lab)]), i
    _, dt_seq, _ = _burst(pkg, graphs)
    print(f"burst of {len(graphs)} requests: big_wide {dt_wide * 1e3:.0f} ms, "
          f"default {dt_seq * 1e3:.0f} ms; wide-searched graphs {st['large_graphs']}")
