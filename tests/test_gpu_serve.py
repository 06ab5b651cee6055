"""The serving loop (gcl_serve_*): every result is the one the batched entry
point gives for the same graph alone, whatever else shares its batch or its
time on the GPU.  Canonical forms and labelings are integers: bit-exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _alone(pkg, G, graphs, ctx):
    """Packed rows and labeling of each graph canonized on its own."""
    out = []
    for g in graphs:
        r = pkg.canon_batch([g], ctx=ctx, dense=False, rows=True)
        assert (r.status == 0).all()
        out.append((r.packed(0).copy(), r.labeling(0).copy()))
    return out


def _drain(srv, n_expected, timeout_polls=6000):
    got = {}
    for _ in range(timeout_polls):
        for r, rows, lab in srv.poll(timeout_ms=10):
            got[r.id] = (r, rows, lab)
        if len(got) >= n_expected:
            break
    assert len(got) == n_expected
    return got


def test_serve_results_equal_alone(pkg, G):
    ctx = pkg.Context(0)
    rng = np.random.default_rng(404)
    graphs = G.small_batch(300, seed=404)
    graphs += [G.tree_plus_edges(int(rng.integers(65, 600)), rng) for _ in range(25)]
    graphs += [G.torus(9), G.random_regular(200, 3, rng), G.from_edges(1, []),
               G.from_edges(40, [])]
    n = len(graphs)
    ref = _alone(pkg, G, graphs, ctx)
    srv = pkg.Server(0, lanes=2, mid_lanes=2, large_lanes=1, max_batch=64)
    # burst: everything queued at once, so batches form while others run
    order = rng.permutation(n)
    for i in order:
        srv.submit_canon(int(i), graphs[i])
    got = _drain(srv, n)
    for i in range(n):
        r, rows, lab = got[i]
        assert r.status == 0
        assert np.array_equal(rows, ref[i][0]), i
        assert np.array_equal(lab, ref[i][1]), i
        assert r.latency_s > 0
    st = srv.stats()
    assert st["completed"] == n and st["batches"] >= 2
    srv.close()


def test_serve_iso_and_classes(pkg, G, oracle_mod):
    rng = np.random.default_rng(77)
    srv = pkg.Server(0, lanes=2, mid_lanes=1, large_lanes=1)
    base = G.small_batch(60, seed=77) + [G.tree_plus_edges(150, rng), G.torus(10)]
    pairs = []
    for g in base:
        pairs.append((g, G.random_relabel(g, rng)))
        pairs.append((g, G.move_one_edge(g, rng)))
    for i, (a, b) in enumerate(pairs):
        srv.submit_iso(i, a, b)
    got = _drain(srv, len(pairs))
    for i, (a, b) in enumerate(pairs):
        r = got[i][0]
        assert r.status == 0
        ma, mb = oracle_mod.canon(a)[0], oracle_mod.canon(b)[0]
        truth = a.n == b.n and np.array_equal(ma, mb)
        assert r.verdict == int(truth), i
    # relabelings fall in the class of the original; repeats are reported
    g = base[3]
    srv.submit_canon(1000, g)
    first = _drain(srv, 1)[1000][0]
    srv.submit_canon(1001, G.random_relabel(g, rng))
    again = _drain(srv, 1)[1001][0]
    assert again.class_id == first.class_id and again.class_id >= 0
    assert again.repeat == 1 and again.canon_hash == first.canon_hash
    # an identical input is answered from the memo, with the same form
    srv.submit_canon(1002, g)
    memo = _drain(srv, 1)[1002]
    assert memo[0].repeat == 2 and memo[0].batch == 0
    srv.close()


def test_serve_large_lane_matches_wide(pkg, G):
    rng = np.random.default_rng(9)
    big = [G.random_regular(2100, 3, rng), G.torus(46)]
    small = G.small_batch(50, seed=9)
    wctx = pkg.Context(0)  # default: the wide search for n > 64
    srv = pkg.Server(0, lanes=1, mid_lanes=1, large_lanes=1)
    for i, g in enumerate(big + small):
        srv.submit_canon(i, g)
    got = _drain(srv, len(big) + len(small))
    for i, g in enumerate(big):
        r, rows, lab = got[i]
        assert r.status == 0 and r.batch == 1
        mat = pkg.api.unpack_rows(rows, g.n)
        assert np.array_equal(mat, pkg.canon(g, ctx=wctx).matrix)
        e = g.edges()
        adj = np.zeros((g.n, g.n), np.uint8)
        adj[e[:, 0], e[:, 1]] = 1
        adj[e[:, 1], e[:, 0]] = 1
        assert np.array_equal(adj[np.ix_(lab, lab)], mat)
    assert srv.stats()["large_graphs"] == 2
    srv.close()


def test_serve_open_loop_replay(pkg, G):
    W = G.serving_workload(1500, rate=2000.0, seed=11, n_max=2600)
    arena = G.pack(W.graphs)
    srv = pkg.Server(0)
    res = srv.replay(arena, W.kind, W.g1, W.g2, W.arrival, timeout_s=300)
    bad = [(i, r.status, W.graphs[W.g1[i]].n, int(W.kind[i])) for i, r in enumerate(res)
           if r.status != 0]
    assert not bad, bad[:10]
    lat = np.array([r.latency_s for r in res])
    assert (lat > 0).all()
    ctx = pkg.Context(0)
    # canonization requests vs the batched entry point alone: equal canonical
    # hashes exactly when the lone canonical forms are equal
    idx = [i for i in range(len(res)) if W.kind[i] == 0 and W.graphs[W.g1[i]].n <= 2048][:300]
    ref = pkg.canon_batch([W.graphs[W.g1[i]] for i in idx], ctx=ctx, dense=False, rows=True)
    by_hash = {}
    for k, i in enumerate(idx):
        key = (W.graphs[W.g1[i]].n, ref.packed(k).tobytes())
        by_hash.setdefault(res[i].canon_hash, set()).add(key)
    assert all(len(v) == 1 for v in by_hash.values())
    assert len(by_hash) == len({k for v in by_hash.values() for k in v})
    st = srv.stats()
    assert st["completed"] >= len(res)
    srv.close()
