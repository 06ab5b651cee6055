"""bench.py on the CPU: the reference arm's JSON line, the rank rule of the
reference arm under a multi-process launch, and the roofline accounting
(algorithmic bytes per graph, the committed ncu traffic figure)."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                          env=e, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_contract_line():
    r = _bench(["--impl", "reference", "--steps", "1", "--warmup", "1"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 1
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["unit"] == d["unit"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
    assert d["cpu_baseline"]["cores"] >= 1 and d["cpu_baseline"]["value"] == d["value"]
    assert "workload" in d["config"]


def test_reference_arm_other_ranks_exit_quietly():
    r = _bench(["--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1"],
               env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_algorithmic_bytes_formula(G, oracle_mod):
    sys.path.insert(0, ROOT)
    import bench
    graphs = G.small_batch(200, seed=3000)
    arena = G.pack(graphs)
    nodes = np.array([oracle_mod.canon(g)[3] for g in graphs], dtype=np.int64)
    want = 0
    for g, k in zip(graphs, nodes):
        csr = 4 * (g.n + 1) + 8 * g.m
        want += csr + g.n * g.n + int(k) * (csr + 32 * g.n)
    assert bench.algorithmic_bytes(arena, nodes) == want
    per_graph = want / len(graphs)
    assert 5_000 < per_graph < 30_000  # about 11.5 KB per graph on this workload


def test_roofline_traffic_comes_from_the_committed_profile():
    sys.path.insert(0, ROOT)
    import bench
    t = bench.read_traffic()
    assert t is not None and t > 0
