"""The config-scale fixture (tests/golden/golden_large.json) on the CPU: every
recipe rebuilds the graph it was made from (same edge-list hash), and the C
restatement of the oracle gives the reference's canonical form, labeling and
counters on the records it finishes quickly -- so the GPU tests that use the
fixture compare against values the restatement and the reference share."""
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden_large as GL  # noqa: E402


@pytest.fixture(scope="module")
def records():
    with open(os.path.join(HERE, "golden", "golden_large.json")) as f:
        return json.load(f)["records"]


def test_fixture_covers_the_configurations(records):
    names = {r["name"] for r in records}
    for want in ("reg3_1024", "reg3_4096", "torus_32x32", "torus_64x64", "tree_2048",
                 "union_reg4_64_x6", "er_20000"):
        assert want in names
    assert sum(r["name"].startswith("mixed_") for r in records) > 1000
    assert any(r["n"] > 4096 for r in records)


def test_recipes_rebuild_the_graphs(records):
    for r in records:
        g = GL.build(r["recipe"])
        assert g.n == r["n"] and len(g.col) // 2 == r["m"], r["name"]
        assert GL.edges_sha256(g) == r["edges_sha256"], r["name"]


def test_restatement_matches_the_reference_fixture(records, oracle_mod):
    # the quick records (a few hundred graphs of every family that has them)
    quick = [r for r in records if r["ref_seconds"] <= 0.02]
    assert len(quick) > 300
    for r in quick:
        g = GL.build(r["recipe"])
        mat, lab, na, nodes = oracle_mod.canon(g, max_aut=r["max_aut"], kind="port")
        got = (GL.rows_sha256(GL.pack_rows(mat)), GL.label_sha256(lab), na, nodes)
        want = (r["rows_sha256"], r["label_sha256"], r["num_aut"], r["nodes"])
        assert got == want, r["name"]


def test_pack_rows_layout():
    # bit j of word w of row i is entry (i, 64 w + j)
    rng = np.random.default_rng(5)
    n = 130
    m = (rng.random((n, n)) < 0.3).astype(np.uint8)
    rows = GL.pack_rows(m).reshape(n, 3)
    for i in range(0, n, 7):
        for j in range(n):
            assert ((int(rows[i, j // 64]) >> (j % 64)) & 1) == m[i, j]
