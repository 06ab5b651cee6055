"""Out-of-memory on the host-pointer paths, injected on the host: with
GCL_FAULT_ALLOC_AT=k the k-th device or pinned allocation of the process
reports out of memory without calling the allocator (csrc/gcl_alloc.h).  For
every k up to the number of allocations a short session makes, a child
process runs that session: context creation, a batch with warp and sparse
graphs, one graph through the wide search, the group order, an isomorphism
query and the file pipeline (or, in the second test, a server).  Each call
either gives the oracle's result or fails with GCL_ERR_NOMEM -- the wide
search may instead fall back to the sequential one -- and the same call
repeated on the same context (server) then gives the oracle's result.  No
device fault is involved."""
import json
import os
import pickle
import subprocess
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NOMEM = -3
MAX_K = 400

CHILD = r'''
import importlib, json, pickle, sys
import numpy as np
pkg = importlib.import_module("gpu-canonical-labeling_b200")
G = pkg.graphs
spec = pickle.load(open(sys.argv[1], "rb"))
mk = lambda t: G.from_edges(t[0], np.asarray(t[1], np.int64).reshape(-1, 2), t[2])
log = []

def call(name, fn, check):
    for attempt in (0, 1):
        try:
            out = fn()
        except pkg.GclError as e:
            log.append([name, attempt, int(e.rc)])
            continue
        log.append([name, attempt, 0 if check(out) else "mismatch"])
        return

def same(g_mat, want):
    return np.array_equal(np.asarray(g_mat, np.uint8) != 0, np.asarray(want) != 0)

if spec["mode"] == "context":
    ctx = []
    call("create", lambda: ctx.append(pkg.Context(0)) or True, lambda ok: ok)
    c = ctx[-1]
    batch = [mk(t) for t in spec["batch"]]
    def check_batch(r):
        return all(same(r.matrix(i), w) for i, w in enumerate(spec["batch_want"]))
    call("batch", lambda: pkg.canon_batch(batch, ctx=c), check_batch)
    wide = mk(spec["wide"])
    call("wide", lambda: pkg.canon(wide, ctx=c), lambda r: same(r.matrix, spec["wide_want"]))
    grp = mk(spec["group"])
    call("group", lambda: pkg.group_order(grp, ctx=c), lambda o: o == spec["group_want"])
    a, b = mk(spec["iso"][0]), mk(spec["iso"][1])
    call("iso", lambda: pkg.is_isomorphic(a, b, ctx=c), lambda v: v is True)
    def check_files(res):
        return all(r.status == 0 and same(pkg.api.unpack_rows(r.rows, r.n), w)
                   for r, w in zip(res, spec["files_want"]))
    call("files", lambda: pkg.api.canon_files(spec["files"], ctx=c), check_files)
else:
    srv = []
    call("serve_create", lambda: srv.append(pkg.Server(0, **spec["cfg"])) or True, lambda ok: ok)
    S = srv[-1]
    graphs = [mk(t) for t in spec["serve"]]
    pending = set(range(len(graphs)))
    for attempt in (0, 1):
        sent = []
        for i in sorted(pending):
            try:
                S.submit_canon(i, graphs[i])
                sent.append(i)
            except pkg.GclError as e:
                log.append(["serve_submit", attempt, int(e.rc)])
        got = 0
        for _ in range(3000):  # 30 s at most
            if got >= len(sent):
                break
            for r, rows, lab in S.poll(timeout_ms=10):
                got += 1
                i = int(r.id)
                if r.status == 0:
                    ok = same(pkg.api.unpack_rows(rows, graphs[i].n), spec["serve_want"][i])
                    log.append(["serve", attempt, 0 if ok else "mismatch"])
                    pending.discard(i)
                else:
                    log.append(["serve", attempt, int(r.status)])
        if not pending:
            break
    if pending:
        log.append(["serve", 2, "unfinished"])
    S.close()
print("LOG " + json.dumps(log))
'''


def _edges(g):
    return (g.n, g.edges().reshape(-1).tolist(), None if g.color is None else g.color.tolist())


def _run_child(spec_path, k, mode_timeout=120):
    env = dict(os.environ)
    env["GCL_FAULT_ALLOC_AT"] = str(k)
    p = subprocess.run([sys.executable, "-c", CHILD, spec_path], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=mode_timeout)
    assert p.returncode == 0, (k, p.stdout[-2000:], p.stderr[-2000:])
    line = [ln for ln in p.stdout.splitlines() if ln.startswith("LOG ")]
    assert line, (k, p.stdout[-2000:], p.stderr[-2000:])
    fired = f"gcl: injected allocation failure {k}" in p.stderr
    return json.loads(line[-1][4:]), fired


def _sweep(spec_path):
    """Runs sessions with k = 1, 2, ... until the k-th allocation is never
    reached (the library reports on stderr when it fails one); returns the
    names of the calls that met an injected failure and that first k.  A
    failure a call recovers from (the wide search falls back to the
    sequential one) counts as reached but is met by no call."""
    faulted = set()
    # every k up to 40, then every 4th: a session's k-th allocation is the
    # same with or without the fault until it happens, so the sessions whose
    # fault fires are exactly k <= its number of allocations
    for k in list(range(1, 41)) + list(range(44, MAX_K + 1, 4)):
        log, fired = _run_child(spec_path, k)
        hit = False
        for name, attempt, rc in log:
            assert rc != "mismatch", (k, name, attempt)
            assert rc != "unfinished", (k, name)
            if attempt == 0:
                assert rc in (0, NOMEM), (k, name, rc)
                if rc == NOMEM:
                    hit = True
                    faulted.add(name)
            else:
                assert rc == 0, (k, name, rc)  # the repeated call succeeds
        assert fired or not hit, k  # a NOMEM comes only from the injected failure
        if not fired:
            return faulted, k
    raise AssertionError(f"still faulting at k = {MAX_K}")


def test_every_allocation_failure_of_a_context_session(G, oracle_mod, tmp_path):
    rng = np.random.default_rng(404)
    batch = G.small_batch(24, seed=404) + [G.random_regular(80, 3, rng),
                                           G.tree_plus_edges(150, rng)]
    wide = G.random_regular(120, 3, rng)
    iso_a = G.erdos_renyi(90, 0.08, rng)
    files = [G.small_batch(1, seed=9)[0], G.torus(6), G.random_regular(100, 4, rng)]
    paths = []
    for i, g in enumerate(files):
        p = tmp_path / f"g{i}.txt"
        G.write_dimacs(g, str(p))
        paths.append(str(p))
    spec = {
        "mode": "context",
        "batch": [_edges(g) for g in batch],
        "batch_want": [oracle_mod.canon(g)[0] for g in batch],
        "wide": _edges(wide), "wide_want": oracle_mod.canon(wide)[0],
        "group": _edges(G.torus(5)), "group_want": 200,  # C5 x C5: 8 k^2
        "iso": [_edges(iso_a), _edges(G.random_relabel(iso_a, rng))],
        "files": paths, "files_want": [oracle_mod.canon(g)[0] for g in files],
    }
    sp = tmp_path / "spec.pkl"
    sp.write_bytes(pickle.dumps(spec))
    faulted, k_end = _sweep(str(sp))
    print(f"context session: under {k_end} allocations, faults met by {sorted(faulted)}")
    # every call of the session allocates on first use
    assert {"create", "batch", "files"} <= faulted


def test_every_allocation_failure_of_a_server(G, oracle_mod, tmp_path):
    rng = np.random.default_rng(405)
    graphs = G.small_batch(6, seed=405) + [G.random_regular(100, 3, rng),
                                           G.tree_plus_edges(300, rng)]
    spec = {
        "mode": "serve",
        "cfg": {"lanes": 1, "mid_lanes": 1, "big_lanes": 1, "large_lanes": 1},
        "serve": [_edges(g) for g in graphs],
        "serve_want": [oracle_mod.canon(g)[0] for g in graphs],
    }
    sp = tmp_path / "spec.pkl"
    sp.write_bytes(pickle.dumps(spec))
    faulted, k_end = _sweep(str(sp))
    print(f"server session: under {k_end} allocations, faults met by {sorted(faulted)}")
    assert "serve_create" in faulted
