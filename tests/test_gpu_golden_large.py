"""GPU parity at the configurations' full sizes, against golden hashes that
the reference's own sequential path produced (tests/golden/golden_large.json,
made by tests/golden/make_golden_large.py): random 3-regular graphs of
1,024 and 4,096 vertices, tori 32x32 and 64x64, trees of 2,048 vertices,
unions of 2-6 identical 4-regular components, Erdos-Renyi graphs of
8,000-20,000 vertices (above the 4,096-vertex tier: the sparse kernel's
large tier and the wide search's largest layouts) and the mixed-size graphs
the reference finishes within seconds.

* the wide search (one graph, many warps; gcl_canon_one_rows) must give the
  reference's canonical form on every record (its statistics and its
  labeling, one of the equivalent best leaves, are its own);
* the batched sequential search (gcl_canon_batch) must give the canonical
  form, the labeling and both counters of the reference on the records
  whose search is short enough for one warp;
* a 4-regular graph of 20,000 vertices, beyond the reference's reach, is
  checked by relabeling invariance.
"""
import json
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden_large as GL  # noqa: E402  (recipes and hashing of the fixture)

# one warp runs the batched search: keep to the records whose reference run
# (one CPU core) is short, or whose search has few nodes (the reference spends
# its time on n^2 certificates there, the GPU kernel's are O(m))
BATCH_REF_SECONDS = 1.0
BATCH_NODES = 100


@pytest.fixture(scope="module")
def records():
    with open(os.path.join(HERE, "golden", "golden_large.json")) as f:
        return json.load(f)["records"]


@pytest.fixture(scope="module")
def built(records):
    out = {}
    for rec in records:
        g = GL.build(rec["recipe"])
        assert GL.edges_sha256(g) == rec["edges_sha256"], rec["name"]
        out[rec["name"]] = g
    return out


def test_wide_search_equals_reference_at_scale(pkg, records, built):
    # every named configuration graph and every fourth mixed-size graph (the
    # whole fixture takes about three minutes)
    ctx = pkg.Context(0)
    bad = []
    for rec in records:
        if rec["name"].startswith("mixed_") and rec["recipe"]["index"] % 4:
            continue
        g = built[rec["name"]]
        rows, _, _ = pkg.api.canon_rows(g, max_aut=rec["max_aut"], ctx=ctx)
        if GL.rows_sha256(rows) != rec["rows_sha256"]:
            bad.append(rec["name"])
    ctx.close()
    assert not bad, bad


def test_batched_search_equals_reference_at_scale(pkg, records, built):
    ctx = pkg.Context(0)
    recs = [r for r in records
            if r["ref_seconds"] <= BATCH_REF_SECONDS or r["nodes"] <= BATCH_NODES]
    assert any(r["n"] > 4096 for r in recs)  # the large tier is covered
    recs.sort(key=lambda r: r["n"])
    bad = []
    for k in range(0, len(recs), 64):
        chunk = recs[k:k + 64]
        res = pkg.canon_batch([built[r["name"]] for r in chunk], ctx=ctx, dense=False,
                              rows=True)
        for i, rec in enumerate(chunk):
            got = (int(res.status[i]), GL.rows_sha256(res.packed(i)),
                   GL.label_sha256(res.labeling(i)), int(res.stats[i, 0]), int(res.stats[i, 1]))
            want = (0, rec["rows_sha256"], rec["label_sha256"], rec["num_aut"], rec["nodes"])
            if got != want:
                bad.append((rec["name"], got[0]))
    ctx.close()
    assert not bad, bad


def test_relabel_invariance_beyond_the_reference(pkg, G):
    rng = np.random.default_rng(20000)
    g = G.random_regular(20000, 4, rng)
    ctx = pkg.Context(0)
    a, _, _ = pkg.api.canon_rows(g, ctx=ctx)
    b, _, _ = pkg.api.canon_rows(G.random_relabel(g, rng), ctx=ctx)
    ctx.close()
    assert np.array_equal(a, b)
    # the rows describe a 4-regular graph (degree of each canonical vertex)
    words = a.reshape(g.n, (g.n + 63) // 64)
    assert (np.bitwise_count(words).sum(axis=1) == 4).all()


def test_batch_handoff_to_wide_search(pkg, G, records, built):
    """GCL_OPT_BATCH_HANDOFF_MS: a graph whose batch warp runs past the
    hand-off budget (a random 3-regular graph of 1,024 vertices searches
    about 4 s on one warp) is finished by the wide search, with the
    reference's canonical form; the small graphs of the batch are untouched."""
    by = {r["name"]: r for r in records}
    rec = by["reg3_1024"]
    small = G.small_batch(40, seed=71)
    graphs = small[:20] + [built["reg3_1024"]] + small[20:]
    ctx = pkg.Context(0)
    plain = pkg.canon_batch(small, ctx=ctx, dense=False, rows=True)
    ctx.set_option(pkg.api.GCL_OPT_BATCH_HANDOFF_MS, 100)
    res = pkg.canon_batch(graphs, ctx=ctx, dense=False, rows=True)
    ctx.close()
    assert (res.status == 0).all()
    assert GL.rows_sha256(res.packed(20)) == rec["rows_sha256"]
    for i in range(40):
        j = i if i < 20 else i + 1
        assert np.array_equal(res.packed(j), plain.packed(i))
        assert np.array_equal(res.stats[j], plain.stats[i])
