"""gpu_canon_label: the reference's command-line behaviour (main.cpp:93-203)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "gpu-canonical-labeling_b200", "bin", "gpu_canon_label")


def reference_listing(A: np.ndarray) -> str:
    """print_canonical_adjacency_list (main.cpp:33-70) restated for the check."""
    n = A.shape[0]
    out = []
    for i in range(n):
        prefix = f"{i:3d} : "
        s, width, first = prefix, len(prefix), True
        for j in range(n):
            if not A[i, j]:
                continue
            tok = f" {j}"
            if not first and width + len(tok) + 1 > 80:
                s += "\n    "
                width = 4
            s += tok
            width += len(tok)
            first = False
        out.append(s + ";\n")
    return "".join(out)


def run(args, cwd):
    return subprocess.run([CLI, *args], cwd=cwd, capture_output=True, text=True, timeout=300)


@pytest.fixture(scope="module", autouse=True)
def built():
    if not os.path.exists(CLI):
        pytest.skip("CLI not built (python gpu-canonical-labeling_b200/build.py)")


def test_usage_and_bad_arguments(tmp_path):
    r = run(["-h"], tmp_path)
    assert r.returncode == 0 and "Usage:" in r.stdout and "--max-aut=N" in r.stdout
    r = run(["--bogus", "x.txt"], tmp_path)
    assert r.returncode == 1 and "Unknown option: --bogus" in r.stderr
    r = run([], tmp_path)
    assert r.returncode == 1 and "Invalid arguments" in r.stderr
    r = run(["a", "b", "c"], tmp_path)
    assert r.returncode == 1
    r = run([str(tmp_path / "missing.txt")], tmp_path)
    assert r.returncode == 1 and "Failed to open DIMACS file" in r.stderr


def test_duplicate_edge_rejected(tmp_path):
    (tmp_path / "d.txt").write_text("p edge 3 2\ne 1 2\ne 2 1\n")
    r = run(["d.txt"], tmp_path)
    assert r.returncode == 1 and "duplicate edge" in r.stderr


@pytest.mark.gpu
def test_single_graph_output_file(G, oracle_mod, tmp_path):
    rng = np.random.default_rng(3)
    for k, g in enumerate([G.erdos_renyi(256, 0.05, rng), G.torus(6)] + G.small_batch(5, seed=2)):
        p = tmp_path / f"g{k}.txt"
        G.write_dimacs(g, str(p))
        r = run([p.name, "--max-aut=10000"], tmp_path)
        assert r.returncode == 0, r.stderr
        mat, _, _, _ = oracle_mod.canon(g)
        assert (tmp_path / "output").read_text() == reference_listing(mat)


@pytest.mark.gpu
def test_two_graph_verdicts(G, tmp_path):
    rng = np.random.default_rng(1000)
    er = G.erdos_renyi(256, 0.05, rng)
    G.write_dimacs(er, str(tmp_path / "a.txt"))
    G.write_dimacs(G.random_relabel(er, rng), str(tmp_path / "b.txt"))
    G.write_dimacs(G.move_one_edge(er, rng), str(tmp_path / "c.txt"))
    r = run(["a.txt", "b.txt"], tmp_path)
    assert r.returncode == 0 and "Result: ISOMORPHIC" in r.stdout
    r = run(["a.txt", "c.txt", "--sequential"], tmp_path)
    assert r.returncode == 0 and "Result: NOT ISOMORPHIC" in r.stdout


@pytest.mark.gpu
def test_sequential_statistics_and_group_order(G, oracle_mod, tmp_path):
    # --sequential prints the reference's two statistics lines with its exact
    # counts (sequential.cpp:83-85); --group-order prints |Aut(G)|
    rng = np.random.default_rng(8)
    for k, (g, order) in enumerate([(G.torus(6), 8 * 36), (G.erdos_renyi(120, 0.05, rng), None)]):
        p = tmp_path / f"s{k}.txt"
        G.write_dimacs(g, str(p))
        r = run([p.name, "--sequential", "--group-order"], tmp_path)
        assert r.returncode == 0, r.stderr
        mat, _, na, nd = oracle_mod.canon(g)
        assert f"Total automorphisms discovered (sequential): {na}\n" in r.stdout
        assert f"Total search tree nodes created (sequential): {nd}\n" in r.stdout
        assert (tmp_path / "output").read_text() == reference_listing(mat)
        line = [x for x in r.stdout.splitlines() if x.startswith("Automorphism group order: ")]
        assert len(line) == 1
        if order is not None:
            assert int(line[0].split(": ")[1]) == order
