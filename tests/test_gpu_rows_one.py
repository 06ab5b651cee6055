"""gcl_canon_one_rows (the CLI's path): the packed form of gcl_canon_one's
matrix, through the wide search (n >= 65 by default) and the sequential
path, with the sequential path's statistics unchanged."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


@pytest.mark.parametrize("wide", [True, False])
def test_rows_equal_the_dense_form(pkg, G, oracle_mod, wide):
    api = pkg.api
    rng = np.random.default_rng(71)
    ctx = pkg.Context(0, wide_min_n=None if wide else api.GCL_MAX_N + 1)
    graphs = [G.erdos_renyi(30, 0.2, rng), G.torus(9), G.random_regular(200, 3, rng),
              G.tree_plus_edges(150, rng), G.from_edges(1, []), G.from_edges(70, [])]
    for g in graphs:
        d = pkg.canon(g, ctx=ctx)
        rows, nodes, naut = api.canon_rows(g, ctx=ctx)
        assert np.array_equal(api.unpack_rows(rows, g.n), d.matrix), g.n
        assert np.array_equal(d.matrix, oracle_mod.canon(g)[0]), g.n
        if not wide:
            assert (nodes, naut) == (d.nodes, d.num_aut)
