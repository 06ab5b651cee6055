"""The wide search with its level gate off (GCL_OPT_WIDE_GATE = 0), the
automatic gate, work sharing and the level probe, vs the oracle.  Without
the gate every first-path sibling starts at once and tests its vertex in its
warp's own union-find; the CPU model of the search (tests/test_wide_model.py)
shows the same canonical form under every schedule with or without the
gate."""
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


@pytest.fixture(scope="module")
def free_ctx(pkg):
    c = pkg.Context(0, wide_min_n=1)
    c.set_option(pkg.api.GCL_OPT_WIDE_GATE, 0)
    return c


def test_gate_off_small_and_symmetric_vs_oracle(pkg, G, oracle_mod, free_ctx):
    rng = np.random.default_rng(2024)
    graphs = [G.torus(k) for k in (3, 4, 5, 6, 8, 10)]
    graphs += [G.disjoint_union(G.random_regular(10, 3, rng), k) for k in (2, 3, 4)]
    graphs += G.small_batch(120, seed=99)
    graphs += [G.tree_plus_edges(int(rng.integers(10, 64)), rng) for _ in range(40)]
    graphs += [G.cfi_graph(b, rng, twist=bool(b % 4)) for b in (4, 6, 8, 10, 12)]
    for g in graphs:
        mat = oracle_mod.canon(g)[0]
        for _ in range(2):
            assert np.array_equal(pkg.canon(g, ctx=free_ctx).matrix, mat)


def test_gate_off_trees_vs_oracle_and_timing(pkg, G, oracle_mod, free_ctx):
    rng = np.random.default_rng(7)
    gated = pkg.Context(0, wide_min_n=1)
    for n in (300, 1000, 2048):
        g = G.from_edges(n, G.recursive_tree(n, rng))
        mat = oracle_mod.canon(g)[0]
        t = time.perf_counter()
        a = pkg.canon(g, ctx=free_ctx).matrix
        t_free = time.perf_counter() - t
        t = time.perf_counter()
        b = pkg.canon(g, ctx=gated).matrix
        t_gate = time.perf_counter() - t
        assert np.array_equal(a, mat) and np.array_equal(b, mat)
        print(f"tree n={n}: gate off {t_free * 1e3:.1f} ms, gate on {t_gate * 1e3:.1f} ms")


@pytest.mark.parametrize("max_aut", [1, 3])
def test_gate_off_small_store(pkg, G, oracle_mod, free_ctx, max_aut):
    rng = np.random.default_rng(5)
    for g in (G.torus(8), G.disjoint_union(G.random_regular(10, 3, rng), 4),
              G.tree_plus_edges(400, rng)):
        mat = oracle_mod.canon(g, max_aut=max_aut)[0]
        assert np.array_equal(pkg.canon(g, max_aut=max_aut, ctx=free_ctx).matrix, mat)


def test_gate_auto_vs_oracle(pkg, G, oracle_mod):
    # 2: off on trees (about one item per level), on for tori and regular graphs
    ctx = pkg.Context(0, wide_min_n=1)
    ctx.set_option(pkg.api.GCL_OPT_WIDE_GATE, 2)
    rng = np.random.default_rng(12)
    graphs = [G.from_edges(n, G.recursive_tree(n, rng)) for n in (100, 700)]
    graphs += [G.torus(12), G.random_regular(300, 3, rng), G.cfi_graph(10, rng)]
    for g in graphs:
        assert np.array_equal(pkg.canon(g, ctx=ctx).matrix, oracle_mod.canon(g)[0])


def _wide_direct(pkg, ctx, g):
    """The wide search through the device entry point, which has no
    fallback: (status, n x n matrix)."""
    import ctypes
    dev = torch.device("cuda", 0)
    P = ctypes.c_void_p
    lib = pkg.api.load_library()
    n = g.n
    rp = torch.from_numpy(np.ascontiguousarray(g.rowptr, np.int32)).to(dev)
    cl = torch.from_numpy(np.ascontiguousarray(g.col if g.col.size else np.zeros(1), np.int32)).to(dev)
    co = None if g.color is None else torch.from_numpy(np.ascontiguousarray(g.color, np.int32)).to(dev)
    dense = torch.zeros(max(n * n, 1), dtype=torch.uint8, device=dev)
    status = torch.full((1,), -1, dtype=torch.int32, device=dev)
    rc = lib.gcl_canon_wide_device_async(ctx.handle, P(rp.data_ptr()), P(cl.data_ptr()),
                                         None if co is None else P(co.data_ptr()), n,
                                         int(g.col.size), 10000, P(dense.data_ptr()), None, None,
                                         None, P(status.data_ptr()))
    assert rc == 0
    ctx.sync()
    return int(status.item()), dense[:n * n].cpu().numpy().reshape(n, n)


@pytest.mark.parametrize("share", [0, 1])
@pytest.mark.parametrize("gate", [1, 0, 2])
def test_gate_and_sharing_no_fallback(pkg, G, oracle_mod, gate, share):
    # through the device entry point: a search that failed (a hand-over, the
    # own-union-find orbit test) would show as a status here instead of being
    # covered by the host's sequential fallback
    rng = np.random.default_rng(45)
    ctx = pkg.Context(0, wide_min_n=1)
    ctx.set_option(pkg.api.GCL_OPT_WIDE_GATE, gate)
    ctx.set_option(pkg.api.GCL_OPT_WIDE_SHARE, share)
    comp = G.random_regular(24, 3, rng)
    for g in [G.disjoint_union(comp, k) for k in (2, 3, 4, 5)] + [G.cfi_graph(10, rng),
                                                                   G.tree_plus_edges(300, rng)]:
        st, mat = _wide_direct(pkg, ctx, g)
        assert st == 0, (g.n, st)
        assert np.array_equal(mat, oracle_mod.canon(g)[0]), g.n


@pytest.mark.parametrize("gate", [1, 0])
def test_work_sharing_vs_oracle(pkg, G, oracle_mod, gate):
    # GCL_OPT_WIDE_SHARE: busy warps hand subtrees to idle ones; unions of
    # identical components keep most of their tree in a few siblings
    import time
    rng = np.random.default_rng(44)
    ctx = pkg.Context(0, wide_min_n=1)
    ctx.set_option(pkg.api.GCL_OPT_WIDE_GATE, gate)
    ctx.set_option(pkg.api.GCL_OPT_WIDE_SHARE, 1)
    plain = pkg.Context(0, wide_min_n=1)
    plain.set_option(pkg.api.GCL_OPT_WIDE_GATE, gate)
    comp = G.random_regular(32, 3, rng)
    graphs = [G.disjoint_union(comp, k) for k in (2, 3, 4, 5)]
    graphs += [G.cfi_graph(b, rng) for b in (8, 16)] + [G.torus(10), G.tree_plus_edges(400, rng)]
    graphs += G.small_batch(40, seed=44)
    for g in graphs:
        want = oracle_mod.canon(g)[0]
        t = time.perf_counter()
        a = pkg.canon(g, ctx=ctx).matrix
        t_share = time.perf_counter() - t
        t = time.perf_counter()
        b = pkg.canon(g, ctx=plain).matrix
        t_plain = time.perf_counter() - t
        assert np.array_equal(a, want) and np.array_equal(b, want), g.n
        if g.n >= 96:
            print(f"n={g.n}: sharing {t_share * 1e3:.1f} ms, without {t_plain * 1e3:.1f} ms")


@pytest.mark.parametrize("probe", [0, 1])
def test_probe_vs_oracle(pkg, G, oracle_mod, probe):
    # GCL_OPT_WIDE_PROBE: under the gate a level's first item runs before the
    # rest of the level; same canonical form either way, and on tori the
    # probe's automorphisms prune the other siblings (far fewer nodes)
    ctx = pkg.Context(0, wide_min_n=1)
    ctx.set_option(pkg.api.GCL_OPT_WIDE_PROBE, probe)
    rng = np.random.default_rng(3131)
    graphs = [G.torus(k) for k in (4, 6, 8, 12, 16)]
    graphs += [G.disjoint_union(G.random_regular(10, 3, rng), k) for k in (2, 3, 4)]
    graphs += [G.cfi_graph(b, rng, twist=bool(b % 4)) for b in (6, 10, 14)]
    graphs += [G.random_regular(200, 3, rng), G.tree_plus_edges(300, rng)]
    graphs += G.small_batch(60, seed=3131)
    for g in graphs:
        mat = oracle_mod.canon(g)[0]
        for _ in range(2):
            assert np.array_equal(pkg.canon(g, ctx=ctx).matrix, mat), g.n
    nodes = pkg.canon(G.torus(16), ctx=ctx).nodes
    seq_nodes = oracle_mod.canon(G.torus(16))[3]
    if probe:
        assert nodes <= 3 * seq_nodes, (nodes, seq_nodes)
    ctx.close()


def test_option_values_checked(pkg):
    ctx = pkg.Context(0)
    for opt, bad in ((pkg.api.GCL_OPT_WIDE_GATE, 3), (pkg.api.GCL_OPT_WIDE_GATE, -1),
                     (pkg.api.GCL_OPT_WIDE_SHARE, 2), (pkg.api.GCL_OPT_WIDE_PROBE, 2),
                     (pkg.api.GCL_OPT_WIDE_PROBE, -1)):
        with pytest.raises(pkg.GclError) as e:
            ctx.set_option(opt, bad)
        assert e.value.rc == -1
    for opt, good in ((pkg.api.GCL_OPT_WIDE_GATE, 0), (pkg.api.GCL_OPT_WIDE_GATE, 2),
                      (pkg.api.GCL_OPT_WIDE_SHARE, 1), (pkg.api.GCL_OPT_WIDE_SHARE, 0)):
        ctx.set_option(opt, good)
