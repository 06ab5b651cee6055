"""Generate tests/golden/golden_large.json: the reference's own sequential
canonical labeler (oracle/_ref/libgcl_ref.so, built from the reference
sources by ``make -C oracle ref REF_SRC=<reference>/src``) run on graphs of
the search-heavy and mixed-size configurations, at their full sizes.

The graphs are too large to store as edge lists, so each record holds a
recipe (a seeded generator call of ``graphs.py``, rebuilt by ``build``) and
the SHA-256 of its sorted edge list, so a test can check that it rebuilt the
same graph.  The reference's outputs are recorded as

* ``rows_sha256`` -- SHA-256 of the canonical matrix as bit-packed rows: n
  rows of ceil(n/64) little-endian 64-bit words, bit j of word w of row i =
  entry (i, 64w + j) (the ``out_rows`` layout of include/gcl.h);
* ``label_sha256`` -- SHA-256 of the best leaf's vertex order (int32);
* ``num_aut`` / ``nodes`` -- the two counters sequential.cpp:83-85 prints;
* ``ref_seconds`` -- how long the reference took here (one core).

Cases: random 3-regular graphs of 1,024 and 4,096 vertices, tori 32x32 and
64x64, disjoint unions of 2-6 copies of a random 4-regular graph on 64
vertices (the union the configuration names has 16 copies, beyond the
reference: 8 copies take it over two minutes, and the search grows
exponentially with the copies), trees of 2,048 vertices (the serving
tail's family), Erdos-Renyi graphs of 8,000-20,000 vertices with mean degree
8, several of them relabeled, and the graphs of the 2,000-graph mixed-size
batch (n log-uniform in [64, 4096]) that the reference finishes within
MIXED_LIMIT_S seconds each.

Run from the repository root:  python tests/golden/make_golden_large.py
(about ten minutes on eight cores).
"""
from __future__ import annotations

import hashlib
import importlib
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
G = importlib.import_module("gpu-canonical-labeling_b200.graphs")

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "golden_large.json")
MIXED_SEED, MIXED_COUNT = 4000, 2000
MIXED_LIMIT_S = 5.0

_mixed = None


def mixed_graph(i: int):
    global _mixed
    if _mixed is None:
        _mixed = G.mixed_batch(MIXED_COUNT, seed=MIXED_SEED)
    return _mixed[i]


def build(recipe: dict):
    """The graph a recipe names (deterministic: seeded generators)."""
    fam = recipe["fam"]
    if fam == "mixed":
        g = mixed_graph(recipe["index"])
    else:
        rng = np.random.default_rng(recipe.get("seed", 0))
        if fam == "regular":
            g = G.random_regular(recipe["n"], recipe["d"], rng)
        elif fam == "torus":
            g = G.torus(recipe["k1"], recipe["k2"])
        elif fam == "recursive_tree":
            g = G.from_edges(recipe["n"], G.recursive_tree(recipe["n"], rng))
        elif fam == "tree_plus_edges":
            g = G.tree_plus_edges(recipe["n"], rng)
        elif fam == "union_regular":
            g = G.disjoint_union(G.random_regular(recipe["c"], recipe["d"], rng), recipe["k"])
        elif fam == "er_deg":
            n = recipe["n"]
            g = G.erdos_renyi(n, recipe["deg"] / (n - 1), rng)
        else:
            raise ValueError(fam)
    if "relabel" in recipe:
        g = G.random_relabel(g, np.random.default_rng(recipe["relabel"]))
    return g


def edges_sha256(g) -> str:
    e = np.sort(np.asarray(g.edges(), dtype=np.int64).reshape(-1, 2), axis=1)
    e = e[np.lexsort((e[:, 1], e[:, 0]))].astype(np.int32)
    return hashlib.sha256(e.tobytes()).hexdigest()


def pack_rows(mat: np.ndarray) -> np.ndarray:
    """n x n 0/1 matrix -> n rows of ceil(n/64) uint64 words (bit j of word
    w of row i = entry (i, 64w + j))."""
    n = mat.shape[0]
    w = (n + 63) // 64
    padded = np.zeros((n, 64 * w), dtype=np.uint8)
    padded[:, :n] = mat != 0
    return np.packbits(padded, axis=1, bitorder="little").view(np.uint64).reshape(-1)


def rows_sha256(rows: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(rows, dtype=np.uint64).tobytes()).hexdigest()


def label_sha256(label: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(label, dtype=np.int32).tobytes()).hexdigest()


def fixed_cases():
    out = []
    for n, seed in ((1024, 61), (4096, 63)):
        r = {"fam": "regular", "n": n, "d": 3, "seed": seed}
        out += [(f"reg3_{n}", r), (f"reg3_{n}_relabel", dict(r, relabel=seed + 1))]
    for k in (32, 64):
        r = {"fam": "torus", "k1": k, "k2": k}
        out += [(f"torus_{k}x{k}", r), (f"torus_{k}x{k}_relabel", dict(r, relabel=70 + k))]
    r = {"fam": "recursive_tree", "n": 2048, "seed": 64}
    out += [("tree_2048", r), ("tree_2048_relabel", dict(r, relabel=164))]
    out.append(("tree_plus_edges_2048", {"fam": "tree_plus_edges", "n": 2048, "seed": 65}))
    for k in (2, 3, 4, 5, 6):
        out.append((f"union_reg4_64_x{k}", {"fam": "union_regular", "c": 64, "d": 4, "k": k,
                                            "seed": 66}))
    out.append(("union_reg4_64_x4_relabel", {"fam": "union_regular", "c": 64, "d": 4, "k": 4,
                                             "seed": 66, "relabel": 166}))
    for n, seed in ((8000, 67), (12000, 68), (20000, 69)):
        out.append((f"er_{n}", {"fam": "er_deg", "n": n, "deg": 8.0, "seed": seed}))
    out.append(("er_8000_relabel", {"fam": "er_deg", "n": 8000, "deg": 8.0, "seed": 67,
                                    "relabel": 167}))
    return out


def _run(item):
    name, recipe = item
    import oracle as O  # the reference's own code, compiled unchanged (oracle/_ref)
    g = build(recipe)
    t = time.perf_counter()
    mat, lab, na, nodes = O.canon(g, max_aut=10000, kind="reference")
    dt = time.perf_counter() - t
    return {"name": name, "recipe": recipe, "n": g.n, "m": int(len(g.col) // 2),
            "edges_sha256": edges_sha256(g), "max_aut": 10000,
            "rows_sha256": rows_sha256(pack_rows(mat)), "label_sha256": label_sha256(lab),
            "num_aut": int(na), "nodes": int(nodes), "ref_seconds": round(dt, 3)}


def _time_one(i, q):
    import oracle as O
    g = mixed_graph(i)
    t = time.perf_counter()
    O.canon(g, max_aut=10000, kind="reference")
    q.put((i, time.perf_counter() - t))


def mixed_indices(limit_s: float, workers: int):
    """Indices of the mixed batch whose reference run ends within limit_s
    (each tried in a child process that is stopped at the limit)."""
    ctx = mp.get_context("fork")
    mixed_graph(0)  # generated once, inherited by the children
    q = ctx.Queue()
    pending, running, ok = list(range(MIXED_COUNT)), {}, []
    while pending or running:
        while pending and len(running) < workers:
            i = pending.pop(0)
            p = ctx.Process(target=_time_one, args=(i, q))
            p.start()
            running[i] = (p, time.perf_counter())
        time.sleep(0.02)
        while not q.empty():
            i, dt = q.get()
            ok.append(i)
        for i, (p, t0) in list(running.items()):
            if not p.is_alive():
                p.join()
                running.pop(i)
            elif time.perf_counter() - t0 > limit_s:
                p.kill()
                p.join()
                running.pop(i)
    time.sleep(0.2)
    while not q.empty():
        ok.append(q.get()[0])
    return sorted(set(ok))


def main():
    import oracle as O
    if not O.available("reference"):
        raise SystemExit("oracle/_ref/libgcl_ref.so missing: run make -C oracle ref "
                         "REF_SRC=<reference>/src")
    workers = max(1, (os.cpu_count() or 2) - 1)
    idx = mixed_indices(MIXED_LIMIT_S, workers)
    items = fixed_cases() + [(f"mixed_{i}", {"fam": "mixed", "index": i}) for i in idx]
    # the longest first, so the pool does not end on one slow graph
    with mp.get_context("fork").Pool(workers) as pool:
        recs = pool.map(_run, sorted(items, key=lambda it: -build(it[1]).n), chunksize=1)
    order = {name: k for k, (name, _) in enumerate(items)}
    recs.sort(key=lambda r: order[r["name"]])
    with open(OUT, "w") as f:
        json.dump({"generator": "tests/golden/make_golden_large.py",
                   "source": "reference sequential path (oracle/_ref)",
                   "mixed": {"seed": MIXED_SEED, "count": MIXED_COUNT, "limit_s": MIXED_LIMIT_S,
                             "finished": len(idx)},
                   "records": recs}, f, separators=(",", ":"))
    print(f"wrote {len(recs)} records to {OUT} ({len(idx)} of {MIXED_COUNT} mixed graphs)")


if __name__ == "__main__":
    main()
