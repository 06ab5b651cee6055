"""gcl_canon_batch_noalloc -- the allocation-free batched entry point.

It exists for callers that cannot call cudaMalloc where they canonize (a
framework that owns all device memory through its own allocator, a plugin in
a process that forbids device allocations after start-up, a latency-critical
path where allocate/free would synchronize the device).  The test owns every
device buffer itself, calls the entry point through the C ABI twice in a row
and checks both results against the existing batched entry point: the
results are integer, so the tolerance is bit-exact.  This file sorts last so
that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GCL_ERR_TOO_LARGE = -5


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


@pytest.mark.parametrize("max_aut", [10000, 2])
def test_noalloc_matches_batched_entry_point(pkg, G, max_aut):
    import torch

    graphs = _graphs(G)
    arena = G.pack(graphs)
    expected = pkg.canon_batch(arena, max_aut=max_aut)  # the existing entry point
    assert (expected.status == 0).all()

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dtype=dt)  # noqa: E731
    ooff = arena.out_offsets()
    d_voff, d_eoff = t(arena.voff, torch.int64), t(arena.eoff, torch.int64)
    d_rp, d_col, d_color = (t(arena.rowptr, torch.int32), t(arena.col, torch.int32),
                            t(arena.color, torch.int32))
    d_ooff = t(ooff, torch.int64)
    d_dense = torch.empty(int(ooff[-1]), dtype=torch.uint8, device=dev)
    d_label = torch.empty(int(arena.voff[-1]), dtype=torch.int32, device=dev)
    d_stats = torch.empty((arena.count, 2), dtype=torch.int64, device=dev)
    d_status = torch.empty(arena.count, dtype=torch.int32, device=dev)
    lib = pkg.api.load_library()
    P = ctypes.c_void_p
    stream = torch.cuda.current_stream(dev)

    def call(max_n):
        return lib.gcl_canon_batch_noalloc(
            P(stream.cuda_stream), arena.count, P(d_voff.data_ptr()), P(d_eoff.data_ptr()),
            P(d_rp.data_ptr()), P(d_col.data_ptr()), P(d_color.data_ptr()), max_aut, max_n,
            P(d_dense.data_ptr()), P(d_ooff.data_ptr()), P(d_label.data_ptr()),
            P(d_stats.data_ptr()), P(d_status.data_ptr()))

    for _ in range(2):  # the scratch keeps the first call's contents for the second
        for buf in (d_dense, d_label, d_stats, d_status):
            buf.fill_(-1 if buf.dtype != torch.uint8 else 0xAB)
        assert call(int(arena.sizes().max())) == 0
        torch.cuda.synchronize()
        assert (d_status.cpu().numpy() == 0).all()
        assert np.array_equal(d_dense.cpu().numpy(), expected.dense[: ooff[-1]])
        assert np.array_equal(d_label.cpu().numpy(), expected.label[: arena.voff[-1]])
        assert np.array_equal(d_stats.cpu().numpy(), expected.stats)

    # sizes beyond the entry point's maximum are refused before any launch
    assert call(65) == GCL_ERR_TOO_LARGE
