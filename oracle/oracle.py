"""ctypes front-end for the CPU oracles -- TEST INFRASTRUCTURE ONLY.

Two oracles live here:

* ``port``      -- ``libgcl_oracle.so``: the plain-C restatement of the
                   reference's sequential labeler (canon_oracle.c).
* ``reference`` -- ``_ref/libgcl_ref.so``: the reference's own sequential
                   sources (src/sequential.cpp et al.) compiled unchanged by
                   ``make -C oracle ref``, behind ref_shim.cpp; also its
                   DIMACS reader (``ref_read_dimacs``).

and a model: ``libgcl_wide_model.so`` (wide_model.c), the many-worker search's
rules on the CPU (``wide_model``) and an unpruned maximum-leaf search
(``exhaustive``).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, and only as the oracle / the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "libgcl_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libgcl_ref.so")


class _Stats(ctypes.Structure):
    _fields_ = [("num_aut", ctypes.c_int64), ("nodes", ctypes.c_int64)]


_P = ctypes.c_void_p
_libs = {}


def _load(kind: str):
    if kind in _libs:
        return _libs[kind]
    path = PORT_SO if kind == "port" else REF_SO
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library missing: {path} (run make -C oracle"
                                f"{' ref' if kind == 'reference' else ''})")
    lib = ctypes.CDLL(path)
    if kind == "port":
        lib.gcl_oracle_canon.argtypes = [ctypes.c_int, _P, _P, _P, ctypes.c_uint, _P, _P, _P]
        lib.gcl_oracle_canon.restype = ctypes.c_int
        lib.gcl_oracle_canon_batch.argtypes = [ctypes.c_int, _P, _P, _P, _P, _P, ctypes.c_uint,
                                               _P, _P, _P, _P]
        lib.gcl_oracle_canon_batch.restype = ctypes.c_int
        lib.gcl_oracle_root_refine.argtypes = [ctypes.c_int, _P, _P, _P, _P, _P]
        lib.gcl_oracle_root_refine.restype = ctypes.c_int
    else:
        lib.gcl_ref_canon.argtypes = [ctypes.c_int, _P, _P, _P, ctypes.c_uint, _P, _P, _P]
        lib.gcl_ref_canon.restype = ctypes.c_int
        lib.gcl_ref_canon_batch.argtypes = [ctypes.c_int, _P, _P, _P, _P, _P, ctypes.c_uint,
                                            _P, _P, _P]
        lib.gcl_ref_canon_batch.restype = ctypes.c_int
        lib.gcl_ref_quiet.argtypes = [ctypes.c_int]
        lib.gcl_ref_quiet(1)
    _libs[kind] = lib
    return lib


def available(kind: str) -> bool:
    return os.path.exists(PORT_SO if kind == "port" else REF_SO)


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_P)


def canon(g, max_aut: int = 10000, kind: str = "port") -> Tuple[np.ndarray, np.ndarray, int, int]:
    """(canonical n x n uint8 matrix, best label, num_aut, nodes) for one graph."""
    lib = _load(kind)
    n = g.n
    rp = np.ascontiguousarray(g.rowptr, dtype=np.int32)
    cl = np.ascontiguousarray(g.col, dtype=np.int32)
    co = None if g.color is None else np.ascontiguousarray(g.color, dtype=np.int32)
    out = np.zeros((n, n), dtype=np.uint8)
    lab = np.zeros(n, dtype=np.int32)
    st = _Stats()
    fn = lib.gcl_oracle_canon if kind == "port" else lib.gcl_ref_canon
    rc = fn(n, _ptr(rp), _ptr(cl if cl.size else np.zeros(1, np.int32)), _ptr(co), max_aut,
            _ptr(out if out.size else np.zeros(1, np.uint8)), _ptr(lab if lab.size else
                                                                   np.zeros(1, np.int32)),
            ctypes.byref(st))
    if rc != 0:
        raise RuntimeError(f"oracle ({kind}) failed rc={rc}")
    return out, lab, int(st.num_aut), int(st.nodes)


def canon_batch(arena, max_aut: int = 10000, kind: str = "port",
                want_matrix: bool = True):
    """Run the oracle over an Arena.  Returns (out_arena or None, ooff,
    num_aut[count], nodes[count])."""
    lib = _load(kind)
    ooff = arena.out_offsets()
    out = np.zeros(max(int(ooff[-1]), 1), dtype=np.uint8) if (want_matrix or kind != "port") else None
    st = (_Stats * max(arena.count, 1))()
    col = arena.col if arena.col.size else np.zeros(1, np.int32)
    if kind == "port":
        rc = lib.gcl_oracle_canon_batch(arena.count, _ptr(arena.voff), _ptr(arena.eoff),
                                        _ptr(arena.rowptr), _ptr(col), _ptr(arena.color),
                                        max_aut, _ptr(out), _ptr(ooff), None, st)
    else:
        rc = lib.gcl_ref_canon_batch(arena.count, _ptr(arena.voff), _ptr(arena.eoff),
                                     _ptr(arena.rowptr), _ptr(col), _ptr(arena.color),
                                     max_aut, _ptr(out), _ptr(ooff), st)
    if rc != 0:
        raise RuntimeError(f"oracle batch ({kind}) failed rc={rc}")
    na = np.array([st[i].num_aut for i in range(arena.count)], dtype=np.int64)
    nd = np.array([st[i].nodes for i in range(arena.count)], dtype=np.int64)
    return out, ooff, na, nd


def root_refine(g) -> Tuple[int, np.ndarray, np.ndarray]:
    lib = _load("port")
    n = g.n
    rp = np.ascontiguousarray(g.rowptr, dtype=np.int32)
    cl = np.ascontiguousarray(g.col, dtype=np.int32)
    co = None if g.color is None else np.ascontiguousarray(g.color, dtype=np.int32)
    el = np.zeros(n, np.int32)
    cs = np.zeros(n, np.int32)
    code = lib.gcl_oracle_root_refine(n, _ptr(rp), _ptr(cl if cl.size else np.zeros(1, np.int32)),
                                      _ptr(co), _ptr(el), _ptr(cs))
    return code, el, cs


WIDE_SO = os.path.join(HERE, "libgcl_wide_model.so")


def _load_wide():
    if "wide" in _libs:
        return _libs["wide"]
    if not os.path.exists(WIDE_SO):
        raise FileNotFoundError(f"oracle library missing: {WIDE_SO} (run make -C oracle)")
    lib = ctypes.CDLL(WIDE_SO)
    lib.gcl_wide_model.argtypes = [ctypes.c_int, _P, _P, _P, ctypes.c_int, ctypes.c_uint,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, _P,
                                   ctypes.POINTER(ctypes.c_long),
                                   ctypes.POINTER(ctypes.c_int), _P, _P, _P, _P]
    lib.gcl_wide_model.restype = ctypes.c_int
    lib.gcl_exhaustive_canon.argtypes = [ctypes.c_int, _P, _P, _P, ctypes.c_long, _P,
                                         ctypes.POINTER(ctypes.c_long)]
    lib.gcl_exhaustive_canon.restype = ctypes.c_int
    _libs["wide"] = lib
    return lib


def _csr(g):
    rp = np.ascontiguousarray(g.rowptr, dtype=np.int32)
    cl = np.ascontiguousarray(g.col, dtype=np.int32)
    co = None if g.color is None else np.ascontiguousarray(g.color, dtype=np.int32)
    return rp, (cl if cl.size else np.zeros(1, np.int32)), co


def wide_model(g, workers: int, seed: int = 0, cap: int = 10000, auts: bool = False,
               gate: int = 1, rounds: Optional[list] = None,
               first_seq: Optional[list] = None, donate: int = 0, probe: bool = False):
    """CPU model of the many-worker search (wide_model.c): `workers` simulated
    workers over the first path's sibling items, stepped round-robin (seed 0)
    or in a seeded random order.  Returns (canonical matrix, nodes, automorphisms
    stored, events) where events counts [leaves equivalent to a best found
    outside their item, nodes pruned as worse than the private best, leaves
    that beat the private best but not a newer shared one]; with auts=True a
    fifth item, the stored automorphisms (naut x n, position -> image).
    gate: items start level by level as on the GPU (0 off, 2 the GPU's
    automatic choice; with probe, each level's first item runs before the
    rest of the level, GCL_OPT_WIDE_PROBE); `rounds`, when a list,
    receives the number of scheduling rounds (every worker steps once per
    round), the first leaf's level D and the number of items; `first_seq`,
    when a list, the first path's individualized vertices.  donate: busy
    workers hand their shallowest untried child to idle ones (1: with the
    parent's partition; 2: the receiver rebuilds it from the first leaf, as
    the GPU does, and events[3] counts replayed codes that differed)."""
    lib = _load_wide()
    rp, cl, co = _csr(g)
    out = np.zeros((g.n, g.n), dtype=np.uint8)
    nodes = ctypes.c_long(0)
    naut = ctypes.c_int(0)
    ev = np.zeros(4, dtype=np.int64)
    store = np.zeros((cap, max(g.n, 1)), dtype=np.uint32) if auts else None
    nr = (ctypes.c_long * 3)()
    fs = np.zeros(max(g.n, 1), dtype=np.uint32)
    rc = lib.gcl_wide_model(g.n, _ptr(rp), _ptr(cl), _ptr(co), workers, seed, cap,
                            int(gate) | (8 if probe else 0),
                            int(donate), _ptr(out), ctypes.byref(nodes), ctypes.byref(naut), _ptr(ev),
                            _ptr(store), nr, _ptr(fs))
    if rc != 0:
        raise RuntimeError(f"wide model failed rc={rc}")
    if rounds is not None:
        rounds.extend(int(x) for x in nr)
    if first_seq is not None:
        first_seq.extend(int(x) for x in fs[:max(int(nr[1]) - 1, 0)])
    if auts:
        return out, int(nodes.value), int(naut.value), ev[:3] if donate != 2 else ev, store[:naut.value, :g.n].copy()
    return out, int(nodes.value), int(naut.value), ev[:3] if donate != 2 else ev


def exhaustive(g, max_leaves: int = 200000) -> Optional[np.ndarray]:
    """The maximum leaf over the whole search tree (no pruning), or None when
    the tree has more than `max_leaves` leaves."""
    lib = _load_wide()
    rp, cl, co = _csr(g)
    out = np.zeros((g.n, g.n), dtype=np.uint8)
    leaves = ctypes.c_long(0)
    rc = lib.gcl_exhaustive_canon(g.n, _ptr(rp), _ptr(cl), _ptr(co), max_leaves, _ptr(out),
                                  ctypes.byref(leaves))
    if rc < 0:
        raise RuntimeError("exhaustive search failed")
    return None if rc else out


def ref_read_dimacs(path: str, cap_n: int = 1 << 17, cap_m: int = 1 << 24):
    """The reference's own CSRGraph::fromDIMACS on `path` (only for files on
    which it is well defined): (n, rowptr, col, color), or None when the file
    cannot be opened."""
    lib = _load("reference")
    if not hasattr(lib.gcl_ref_read_dimacs, "_typed"):
        lib.gcl_ref_read_dimacs.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int64,
                                            ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int64), _P, _P, _P]
        lib.gcl_ref_read_dimacs.restype = ctypes.c_int
        lib.gcl_ref_read_dimacs._typed = True
    n = ctypes.c_int(0)
    m = ctypes.c_int64(0)
    rp = np.zeros(cap_n + 1, np.int32)
    cl = np.zeros(max(cap_m, 1), np.int32)
    co = np.zeros(max(cap_n, 1), np.int32)
    rc = lib.gcl_ref_read_dimacs(path.encode(), cap_n, cap_m, ctypes.byref(n), ctypes.byref(m),
                                 _ptr(rp), _ptr(cl), _ptr(co))
    if rc == 1:
        return None
    if rc != 0:
        raise RuntimeError("reference reader: capacity too small")
    k = n.value
    return k, rp[:k + 1].copy(), cl[:m.value].copy(), co[:k].copy()
