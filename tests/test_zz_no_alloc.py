"""gcl_canon_batch_noalloc -- the allocation-free batched entry point.

It exists for callers that cannot call cudaMalloc where they canonize (a
framework that owns all device memory through its own allocator, a plugin in
a process that forbids device allocations after start-up, a latency-critical
path where allocate/free would synchronize the device).  The tests own every
device buffer themselves, call the entry point through the C ABI twice in a
row and check both results against the existing batched entry point: the
results are integer, so the tolerance is bit-exact.  This file sorts last so
that a run stopping at the first failure has already run every other test.

The entry point's one outcome of its own, GCL_GRAPH_AUT_OVERFLOW (a graph
that stores more than 128 automorphisms with max_aut > 128), has no test
input: the oracle stored at most 63 automorphisms (n - 1) on every one of
117,709 random graphs of at most 64 vertices tried (complete multipartite
graphs, unions of identical components and their complements, sparse random
graphs, tori, cycle unions), and at most 11 on CFI graphs of 40 and 60
vertices.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GCL_ERR_TOO_LARGE = -5
GRAPH_TOO_LARGE = 2


def _graphs(G):
    rng = np.random.default_rng(321)
    gs = G.small_batch(800, seed=321)
    gs += [G.torus(8), G.torus(4, 7), G.from_edges(40, []), G.from_edges(1, []),
           G.from_edges(33, [(i, j) for i in range(33) for j in range(i + 1, 33)]),
           G.disjoint_union(G.random_regular(8, 3, rng), 4)]
    for _ in range(40):
        n = int(rng.integers(2, 65))
        gs.append(G.from_edges(n, G.erdos_renyi(n, 0.3, rng).edges(), rng.integers(0, 3, n)))
    return gs


class _Call:
    """Device buffers owned by the test and the C-ABI call over them."""

    def __init__(self, pkg, arena, max_aut):
        import torch

        self.torch = torch
        self.dev = torch.device("cuda", 0)
        torch.cuda.set_device(self.dev)
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(self.dev, dtype=dt)  # noqa: E731
        self.arena, self.max_aut = arena, max_aut
        self.ooff = arena.out_offsets()
        self.d_voff, self.d_eoff = t(arena.voff, torch.int64), t(arena.eoff, torch.int64)
        self.d_rp = t(arena.rowptr, torch.int32)
        self.d_col = t(arena.col if arena.col.size else np.zeros(1, np.int32), torch.int32)
        self.d_color = t(arena.color, torch.int32)
        self.d_ooff = t(self.ooff, torch.int64)
        self.d_dense = torch.empty(max(int(self.ooff[-1]), 1), dtype=torch.uint8, device=self.dev)
        self.d_label = torch.empty(max(int(arena.voff[-1]), 1), dtype=torch.int32, device=self.dev)
        self.d_stats = torch.empty((arena.count, 2), dtype=torch.int64, device=self.dev)
        self.d_status = torch.empty(arena.count, dtype=torch.int32, device=self.dev)
        self.lib = pkg.api.load_library()
        self.stream = torch.cuda.current_stream(self.dev)

    def poison(self):
        for buf in (self.d_dense, self.d_label, self.d_stats, self.d_status):
            buf.fill_(-1 if buf.dtype != self.torch.uint8 else 0xAB)

    def __call__(self, max_n, color=True, dense=True, label=True, stats=True):
        P = ctypes.c_void_p
        ptr = lambda b, on: P(b.data_ptr()) if on else None  # noqa: E731
        return self.lib.gcl_canon_batch_noalloc(
            P(self.stream.cuda_stream), self.arena.count, P(self.d_voff.data_ptr()),
            P(self.d_eoff.data_ptr()), P(self.d_rp.data_ptr()), P(self.d_col.data_ptr()),
            ptr(self.d_color, color), self.max_aut, max_n, ptr(self.d_dense, dense),
            ptr(self.d_ooff, dense), ptr(self.d_label, label), ptr(self.d_stats, stats),
            P(self.d_status.data_ptr()))

    def results(self):
        self.torch.cuda.synchronize()
        return (self.d_status.cpu().numpy(), self.d_dense.cpu().numpy(),
                self.d_label.cpu().numpy(), self.d_stats.cpu().numpy())


@pytest.mark.parametrize("max_aut", [10000, 2])
def test_noalloc_matches_batched_entry_point(pkg, G, max_aut):
    graphs = _graphs(G)
    arena = G.pack(graphs)
    expected = pkg.canon_batch(arena, max_aut=max_aut)  # the existing entry point
    assert (expected.status == 0).all()
    call = _Call(pkg, arena, max_aut)
    nv = int(arena.voff[-1])
    for _ in range(2):  # the scratch keeps the first call's contents for the second
        call.poison()
        assert call(int(arena.sizes().max())) == 0
        status, dense, label, stats = call.results()
        assert (status == 0).all()
        assert np.array_equal(dense[: call.ooff[-1]], expected.dense[: call.ooff[-1]])
        assert np.array_equal(label[:nv], expected.label[:nv])
        assert np.array_equal(stats, expected.stats)

    # sizes beyond the entry point's maximum are refused before any launch
    assert call(65) == GCL_ERR_TOO_LARGE


def test_noalloc_optional_outputs_absent(pkg, G):
    """Uncoloured graphs without the colour array, and the optional outputs
    (dense matrices, labelings, statistics) left out one at a time: the
    status and the outputs still given equal the batched entry point's."""
    graphs = G.small_batch(300, seed=77) + [G.torus(6), G.from_edges(20, [])]
    arena = G.pack(graphs)
    expected = pkg.canon_batch(arena, max_aut=10000)
    assert (expected.status == 0).all()
    call = _Call(pkg, arena, 10000)
    nv, nd = int(arena.voff[-1]), int(call.ooff[-1])
    for omit in ("dense", "label", "stats", "color"):
        for _ in range(2):
            call.poison()
            kw = {omit: False}
            assert call(int(arena.sizes().max()), **kw) == 0
            status, dense, label, stats = call.results()
            assert (status == 0).all(), omit
            if omit != "dense":
                assert np.array_equal(dense[:nd], expected.dense[:nd]), omit
            else:
                assert (dense[:nd] == 0xAB).all()  # nothing written
            if omit != "label":
                assert np.array_equal(label[:nv], expected.label[:nv]), omit
            if omit != "stats":
                assert np.array_equal(stats, expected.stats), omit
            else:
                assert (stats == -1).all()


def test_noalloc_graph_above_64_vertices_in_batch(pkg, G):
    """A batch whose declared max_n is 64 but which holds graphs of more than
    64 vertices: exactly those graphs report GCL_GRAPH_TOO_LARGE and the
    rest equal the batched entry point's results."""
    rng = np.random.default_rng(9)
    small = G.small_batch(200, seed=99)
    big = [G.from_edges(70, G.erdos_renyi(70, 0.1, rng).edges()), G.torus(9)]
    graphs = small[:50] + [big[0]] + small[50:150] + [big[1]] + small[150:]
    arena = G.pack(graphs)
    expected = pkg.canon_batch(arena, max_aut=10000)
    assert (expected.status == 0).all()
    call = _Call(pkg, arena, 10000)
    too_big = arena.sizes() > 64
    assert too_big.sum() == 2
    for _ in range(2):
        call.poison()
        assert call(64) == 0
        status, dense, label, stats = call.results()
        assert (status[too_big] == GRAPH_TOO_LARGE).all()
        assert (status[~too_big] == 0).all()
        for g in np.flatnonzero(~too_big):
            a, b = int(call.ooff[g]), int(call.ooff[g + 1])
            assert np.array_equal(dense[a:b], expected.dense[a:b]), g
            va, vb = int(arena.voff[g]), int(arena.voff[g + 1])
            assert np.array_equal(label[va:vb], expected.label[va:vb]), g
            assert np.array_equal(stats[g], expected.stats[g]), g
