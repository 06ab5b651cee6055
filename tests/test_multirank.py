"""The multi-rank path on CPU: two gloo ranks on 127.0.0.1.

Graphs are independent, so a batch shards by graph with no collective on the
data path: each rank canonizes its own size-balanced range (here with the CPU
oracle standing in for its GPU) and the results are gathered at the end; the
job's time is the slowest rank's (bench.py's max_over_ranks / job_rate)."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, root, out):
    import importlib
    import sys

    import torch.distributed as dist

    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import bench
        import oracle
        G = importlib.import_module("gpu-canonical-labeling_b200.graphs")
        graphs = G.small_batch(120, seed=42)
        lo, hi = G.shard_ranges([g.n for g in graphs], world)[rank]
        mine = {i: oracle.canon(graphs[i])[0].tobytes() for i in range(lo, hi)}
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        # the slowest rank sets the job time
        slowest = bench.max_over_ranks(1.0 + rank, world)
        rate = bench.job_rate(len(graphs) // world, world, 3, slowest)
        if rank == 0:
            merged = {}
            for part in gathered:
                merged.update(part)
            out.put((sorted(merged), [merged[i] for i in sorted(merged)], slowest, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_gather(G):
    import multiprocessing as mp

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, root, q)) for r in range(2)]
    for p in procs:
        p.start()
    keys, mats, slowest, rate = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    import oracle

    graphs = G.small_batch(120, seed=42)
    assert keys == list(range(len(graphs)))
    for i, m in zip(keys, mats):
        assert m == oracle.canon(graphs[i])[0].tobytes()
    assert slowest == 2.0
    assert rate == pytest.approx(2 * 60 * 3 / 2.0)


def test_shard_ranges_cover_and_balance(G):
    rng = np.random.default_rng(3)
    sizes = rng.integers(10, 4096, 500)
    for world in (1, 2, 3, 8):
        rs = G.shard_ranges(sizes, world)
        assert rs[0][0] == 0 and rs[-1][1] == len(sizes)
        assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
        cost = [float((sizes[a:b].astype(float) ** 2).sum()) for a, b in rs]
        assert max(cost) - min(cost) <= 2 * (float(sizes.max()) ** 2 + 1)
