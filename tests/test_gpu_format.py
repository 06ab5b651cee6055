"""gcl_format_adjacency_device_async: the reference's `output` text written
on the device from packed canonical rows, for a whole batch, against a
restatement of print_canonical_adjacency_list over the oracle's matrices.
The row format itself is checked on the CPU (tests/test_format.py)."""
import ctypes

import numpy as np
import pytest

from test_cli import reference_listing

torch = pytest.importorskip("torch")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


def test_device_text_equals_reference_listing(pkg, G, oracle_mod):
    rng = np.random.default_rng(70)
    graphs = list(G.small_batch(200, seed=70))
    graphs += [G.random_regular(500, 3, rng), G.erdos_renyi(300, 0.3, rng), G.torus(12),
               G.from_edges(1, []), G.from_edges(1100, G.recursive_tree(1100, rng))]
    ctx = pkg.Context(0)
    res = pkg.canon_batch(graphs, ctx=ctx, dense=False, rows=True)
    assert (res.status == 0).all()
    dev = torch.device("cuda", 0)
    P = ctypes.c_void_p
    d_voff = torch.from_numpy(np.ascontiguousarray(res.arena.voff)).to(dev)
    d_roff = torch.from_numpy(np.ascontiguousarray(res.roff)).to(dev)
    d_rows = torch.from_numpy(res.rows.view(np.int64).copy()).to(dev)
    d_toff = torch.zeros(len(graphs) + 1, dtype=torch.int64, device=dev)
    lib = pkg.api.load_library()
    rc = lib.gcl_format_adjacency_device_async(ctx.handle, len(graphs), P(d_voff.data_ptr()),
                                               P(d_rows.data_ptr()), P(d_roff.data_ptr()),
                                               P(d_toff.data_ptr()), None)
    assert rc == 0
    ctx.sync()
    toff = d_toff.cpu().numpy()
    text = torch.zeros(int(toff[-1]), dtype=torch.uint8, device=dev)
    rc = lib.gcl_format_adjacency_device_async(ctx.handle, len(graphs), P(d_voff.data_ptr()),
                                               P(d_rows.data_ptr()), P(d_roff.data_ptr()),
                                               P(d_toff.data_ptr()), P(text.data_ptr()))
    assert rc == 0
    ctx.sync()
    out = text.cpu().numpy().tobytes()
    for k, g in enumerate(graphs):
        want = reference_listing(oracle_mod.canon(g)[0])
        assert out[toff[k]:toff[k + 1]].decode() == want, k
