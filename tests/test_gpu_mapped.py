"""Batches in mapped host memory (gcl_host_alloc, gcl_canon_batch_mapped):
the same results as gcl_canon_batch, the warp kernel reading the arena and
writing the results in place over the bus; batches with larger graphs go
through device copies; arrays outside the context's mapped buffers, whole,
are refused before any device work."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


def _same(a, b):
    assert np.array_equal(a.dense, b.dense)
    assert np.array_equal(a.label, b.label)
    assert np.array_equal(a.stats, b.stats)
    assert np.array_equal(a.status, b.status)
    assert (a.rows is None) == (b.rows is None)
    if a.rows is not None:
        assert np.array_equal(a.rows, b.rows)


@pytest.mark.parametrize("mixed", [False, True])
def test_mapped_batch_equals_copied_batch(pkg, G, oracle_mod, mixed):
    api = pkg.api
    rng = np.random.default_rng(61)
    graphs = G.small_batch(500, seed=61)
    if mixed:
        graphs += [G.random_regular(100, 3, rng), G.tree_plus_edges(200, rng)]
    ctx = pkg.Context(0)
    want = api.canon_batch(graphs, ctx=ctx, rows=True)
    got = api.canon_batch_mapped(graphs, ctx=ctx, rows=True)
    _same(got, want)
    for i in range(0, len(graphs), 50):
        assert np.array_equal(got.matrix(i), oracle_mod.canon(graphs[i])[0])
    # colours and an edgeless graph through the mapped path
    col = [G.from_edges(g.n, g.edges(), rng.integers(0, 3, g.n)) for g in graphs[:40]]
    col += [G.from_edges(5, [])]
    _same(api.canon_batch_mapped(col, ctx=ctx, rows=True), api.canon_batch(col, ctx=ctx, rows=True))


def test_arrays_outside_mapped_buffers_are_refused(pkg, G):
    api = pkg.api
    ctx = pkg.Context(0)
    lib = ctx.lib
    a = G.pack(G.small_batch(20, seed=62))
    P = lambda x: None if x is None else x.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    status = ctx.host_array((a.count,), np.int32)
    # plain numpy arrays (pageable memory): refused
    rc = lib.gcl_canon_batch_mapped(ctx.handle, a.count, P(a.voff), P(a.eoff), P(a.rowptr),
                                    P(a.col), None, 10000, None, None, None, None, None, None,
                                    P(status))
    assert rc == -1
    # mapped arrays, but the edge array one entry short of its extent
    mv, me, mr = (ctx.host_array(x.shape, x.dtype) for x in (a.voff, a.eoff, a.rowptr))
    mv[...], me[...], mr[...] = a.voff, a.eoff, a.rowptr
    short = ctx.host_array((a.col.size - 1,), np.int32)
    short[...] = a.col[:-1]
    rc = lib.gcl_canon_batch_mapped(ctx.handle, a.count, P(mv), P(me), P(mr), P(short), None,
                                    10000, None, None, None, None, None, None, P(status))
    assert rc == -1
    # and whole: accepted
    full = ctx.host_array(a.col.shape, np.int32)
    full[...] = a.col
    rc = lib.gcl_canon_batch_mapped(ctx.handle, a.count, P(mv), P(me), P(mr), P(full), None,
                                    10000, None, None, None, None, None, None, P(status))
    assert rc == 0 and not status.any()
    # freeing: known buffers once, unknown pointers refused
    ctx.host_free(short)
    with pytest.raises(pkg.GclError):
        ctx.host_free(short)
    with pytest.raises(pkg.GclError):
        ctx.host_free(a.voff)
