"""Bounded searches: a graph whose search outlasts its time budget
(GCL_GRAPH_BUDGET_S, read at each call) ends with GCL_ERR_TIMEOUT (its
status GCL_GRAPH_TIMEOUT), no result, and the context stays usable -- the same graph
with a normal budget then gives the oracle's form.  No fault is involved:
the search loop reads the global timer and returns."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


@pytest.fixture
def tiny_budget():
    old = os.environ.get("GCL_GRAPH_BUDGET_S")

    def set_budget(s):
        os.environ["GCL_GRAPH_BUDGET_S"] = str(s)
    yield set_budget
    if old is None:
        os.environ.pop("GCL_GRAPH_BUDGET_S", None)
    else:
        os.environ["GCL_GRAPH_BUDGET_S"] = old


@pytest.mark.parametrize("wide", [False, True])
def test_budget_runs_out_and_context_recovers(pkg, G, oracle_mod, tiny_budget, wide):
    rng = np.random.default_rng(21)
    hard = G.disjoint_union(G.random_regular(32, 3, rng), 6)  # ~76 k nodes sequentially
    ctx = pkg.Context(0, wide_min_n=1 if wide else pkg.api.GCL_MAX_N + 1)
    tiny_budget(0.0005)
    with pytest.raises(pkg.GclError) as e:
        pkg.canon(hard, ctx=ctx)
    assert e.value.rc == -6  # GCL_ERR_TIMEOUT
    if not wide:
        # the batch reports the first failing graph's error
        with pytest.raises(pkg.GclError) as e:
            pkg.canon_batch([G.torus(3), hard], ctx=ctx)
        assert e.value.rc == -6
    tiny_budget(60)
    assert np.array_equal(pkg.canon(G.torus(5), ctx=ctx).matrix, oracle_mod.canon(G.torus(5))[0])
    assert np.array_equal(pkg.canon(hard, ctx=ctx).matrix, oracle_mod.canon(hard)[0])
