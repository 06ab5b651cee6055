"""The drop-in: the reference's own main.cpp and sources, unchanged, linked
with Nauty_Parallel from shim/nauty_parallel_gcl.cpp over libgcl_b200.so
(built by `make -C oracle dropin`, as a maintainer would build it).

On the CPU the binary's --sequential path is the reference's own code, and
its default --parallel path must reach this library (which, with no GPU,
fails the way the reference's main reports a failed labeling).  The staged
GPU test checks that --parallel writes the same `output` as --sequential."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "gpu_canon_label_dropin")

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def dropin(oracle_mod):
    if not os.path.exists(BIN):
        if not oracle_mod.available("reference"):
            pytest.skip("the reference's sources were not available to build the oracles")
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "dropin"], check=True)
    return BIN


def _run(args, cwd):
    return subprocess.run([BIN, *args], cwd=cwd, capture_output=True, text=True, timeout=300)


def test_dropin_help_and_sequential_path(G, oracle_mod, dropin, tmp_path):
    from test_cli import reference_listing
    r = _run(["-h"], tmp_path)
    assert r.returncode == 0 and "Usage:" in r.stdout
    rng = np.random.default_rng(3)
    for i, g in enumerate([G.torus(4), G.tree_plus_edges(30, rng), G.random_regular(20, 3, rng)]):
        p = tmp_path / f"g{i}.txt"
        G.write_dimacs(g, str(p))
        r = _run([p.name, "--sequential"], tmp_path)
        assert r.returncode == 0, r.stderr
        assert (tmp_path / "output").read_text() == reference_listing(oracle_mod.canon(g)[0])


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the failure path without a GPU")
def test_dropin_parallel_path_reaches_the_library(G, dropin, tmp_path):
    p = tmp_path / "c5.txt"
    G.write_dimacs(G.from_edges(5, [(i, (i + 1) % 5) for i in range(5)]), str(p))
    r = _run([p.name], tmp_path)
    assert r.returncode == 1 and "Canonical labeling failed" in r.stderr


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")
def test_dropin_parallel_equals_sequential_on_gpu(G, dropin, tmp_path):
    rng = np.random.default_rng(4)
    graphs = [G.torus(6), G.tree_plus_edges(200, rng), G.random_regular(300, 3, rng),
              G.from_edges(40, G.erdos_renyi(40, 0.2, rng).edges(), rng.integers(0, 3, 40))]
    for i, g in enumerate(graphs):
        p = tmp_path / f"g{i}.txt"
        G.write_dimacs(g, str(p))
        assert _run([p.name, "--sequential"], tmp_path).returncode == 0
        seq = (tmp_path / "output").read_text()
        assert _run([p.name, "--parallel"], tmp_path).returncode == 0
        assert (tmp_path / "output").read_text() == seq
    a, b = tmp_path / "g0.txt", tmp_path / "h0.txt"
    G.write_dimacs(G.random_relabel(graphs[0], rng), str(b))
    r = _run([a.name, b.name], tmp_path)
    assert r.returncode == 0 and "Result: ISOMORPHIC" in r.stdout
