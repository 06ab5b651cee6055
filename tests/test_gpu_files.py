"""gcl_canon_files: DIMACS files parsed on host threads while the GPU works.
Every file's result equals that of the batched entry point on the graph
parsed by the Python reader (same fromDIMACS semantics); unreadable or
malformed files come back as bad input without stopping the others."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_canon_files_match_batch(pkg, G, tmp_path):
    rng = np.random.default_rng(6)
    graphs = G.small_batch(150, seed=6)
    graphs += [G.tree_plus_edges(int(rng.integers(65, 400)), rng) for _ in range(10)]
    n = 12
    graphs.append(G.from_edges(n, G.erdos_renyi(n, 0.3, rng).edges(), rng.integers(0, 3, n)))
    paths = []
    for i, g in enumerate(graphs):
        p = tmp_path / f"g{i}.txt"
        G.write_dimacs(g, str(p))
        paths.append(str(p))
    bad = tmp_path / "bad.txt"
    bad.write_text("p edge 3 2\ne 1 2\ne 2 1\n")  # the same edge twice
    missing = str(tmp_path / "missing.txt")
    paths_all = paths[:50] + [str(bad)] + paths[50:] + [missing]
    ctx = pkg.Context(0, wide_min_n=pkg.api.GCL_MAX_N + 1)
    res = pkg.api.canon_files(paths_all, ctx=ctx, chunk=37, threads=4)
    parsed = [G.read_dimacs(p) for p in paths]
    ref = pkg.canon_batch(parsed, ctx=ctx, dense=False, rows=True)
    assert res[50].status == 3 and res[-1].status == 3  # GCL_GRAPH_BAD_INPUT
    good = [r for i, r in enumerate(res) if i not in (50, len(res) - 1)]
    assert len(good) == len(parsed)
    for k, r in enumerate(good):
        assert r.status == 0 and r.n == parsed[k].n
        assert np.array_equal(r.rows, ref.packed(k)), k
        assert np.array_equal(r.label, ref.labeling(k)), k
        assert (r.num_aut, r.nodes) == tuple(ref.stats[k])
