"""Generate tests/golden/golden.json by running the reference's own sequential
canonical labeler (src/sequential.cpp et al., compiled unchanged from the
reference sources by ``make -C oracle ref REF_SRC=<reference>/src`` into
oracle/_ref/libgcl_ref.so).

Each record holds a seeded input graph and the reference's outputs for it:
the best leaf's vertex order (``label``, position -> vertex), the SHA-256 of
the n x n canonical adjacency matrix, the number of stored automorphisms and
the number of search-tree nodes (the two counters sequential.cpp:83-85
prints).  The fixtures pin the C restatement in oracle/ and the CUDA path.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import importlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
G = importlib.import_module("gpu-canonical-labeling_b200.graphs")
import oracle as O  # noqa: E402


def cases():
    out = []
    # batched small-graph workload (first 120 graphs of the bench input)
    for i, g in enumerate(G.small_batch(120, seed=3000)):
        out.append((f"small_{i}", g, 10000))
    # Erdos-Renyi G(256, 0.05), a relabeling and a one-edge-moved copy
    rng = np.random.default_rng(1000)
    er = G.erdos_renyi(256, 0.05, rng)
    out += [("er256", er, 10000), ("er256_relabel", G.random_relabel(er, rng), 10000),
            ("er256_moved", G.move_one_edge(er, rng), 10000)]
    # symmetric graphs
    for k in (3, 4, 5, 6, 8):
        out.append((f"torus_{k}", G.torus(k), 10000))
    out.append(("torus_4x7", G.torus(4, 7), 10000))
    rng = np.random.default_rng(2000)
    r8 = G.random_regular(8, 3, rng)
    for k in (2, 3, 4):
        out.append((f"union_r8_x{k}", G.disjoint_union(r8, k), 10000))
    c5 = G.from_edges(5, [(i, (i + 1) % 5) for i in range(5)])
    out.append(("union_c5_x3", G.disjoint_union(c5, 3), 10000))
    out.append(("petersen", G.from_edges(10, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 0), (0, 5),
                                              (1, 6), (2, 7), (3, 8), (4, 9), (5, 7), (7, 9),
                                              (9, 6), (6, 8), (8, 5)]), 10000))
    out.append(("reg3_64", G.random_regular(64, 3, rng), 10000))
    out.append(("reg4_100", G.random_regular(100, 4, rng), 10000))
    out.append(("reg3_64_relabel", G.random_relabel(out[-2][1], rng), 10000))
    # edge cases
    out += [
        ("n0", G.from_edges(0, []), 10000),
        ("n1", G.from_edges(1, []), 10000),
        ("n2_edge", G.from_edges(2, [(0, 1)]), 10000),
        ("n2_empty", G.from_edges(2, []), 10000),
        ("empty10", G.from_edges(10, []), 10000),
        ("empty40", G.from_edges(40, []), 10000),
        ("K8", G.from_edges(8, [(i, j) for i in range(8) for j in range(i + 1, 8)]), 10000),
        ("K33", G.from_edges(33, [(i, j) for i in range(33) for j in range(i + 1, 33)]), 10000),
        ("star10", G.from_edges(10, [(0, i) for i in range(1, 10)]), 10000),
        ("cycle12", G.from_edges(12, [(i, (i + 1) % 12) for i in range(12)]), 10000),
        ("cycle64", G.from_edges(64, [(i, (i + 1) % 64) for i in range(64)]), 10000),
        ("path63", G.from_edges(63, [(i, i + 1) for i in range(62)]), 10000),
        ("hexcol", G.from_edges(6, [(i, (i + 1) % 6) for i in range(6)], [1, 0, 1, 0, 2, 0]), 10000),
        ("negcol", G.from_edges(5, [(0, 1), (1, 2), (2, 3), (3, 4)], [-3, 7, -3, 0, 2]), 10000),
    ]
    # max_aut small enough that the automorphism ring wraps
    for ma in (1, 2, 3, 5):
        out.append((f"torus6_maxaut{ma}", G.torus(6), ma))
        out.append((f"empty10_maxaut{ma}", G.from_edges(10, []), ma))
    # coloured random graphs
    rng = np.random.default_rng(2500)
    for i in range(24):
        n = int(rng.integers(4, 65))
        g = G.erdos_renyi(n, float(rng.uniform(0.03, 0.5)), rng)
        col = rng.integers(0, 4, n)
        out.append((f"colored_{i}", G.from_edges(n, g.edges(), col), 10000))
    # denser random graphs up to 64 vertices
    for i in range(24):
        n = int(rng.integers(2, 65))
        out.append((f"er_{i}", G.erdos_renyi(n, float(rng.uniform(0.02, 0.7)), rng), 10000))
    return out


def main():
    if not O.available("reference"):
        raise SystemExit("oracle/_ref/libgcl_ref.so missing: run make -C oracle ref "
                         "REF_SRC=<reference>/src")
    recs = []
    for name, g, max_aut in cases():
        mat, lab, na, nodes = O.canon(g, max_aut=max_aut, kind="reference")
        recs.append({
            "name": name,
            "n": g.n,
            "edges": g.edges().reshape(-1).tolist(),
            "color": None if g.color is None else g.color.tolist(),
            "max_aut": max_aut,
            "label": lab.tolist(),
            "matrix_sha256": hashlib.sha256(mat.tobytes()).hexdigest(),
            "num_aut": na,
            "nodes": nodes,
        })
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
    with open(path, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "source": "reference sequential path (oracle/_ref)",
                   "records": recs}, f, separators=(",", ":"))
    print(f"wrote {len(recs)} records to {path}")


if __name__ == "__main__":
    main()
