"""Python binding of the C ABI (include/gcl.h) over ctypes.

Names mirror the reference's entry points: ``Nauty_Parallel`` returns the
n*n canonical adjacency bytes like src/nauty_parallel.h:9-13, ``canon`` adds
the search statistics, ``canon_batch`` is the batched arena form and
``is_isomorphic`` is the two-graph check of main.cpp:172-197.

The library is the CUDA build in this directory; there is no CPU fallback:
importing a function that needs it raises if ``libgcl_b200.so`` is missing or
no GPU is visible.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import List, Optional, Sequence, Union

import numpy as np

from .graphs import Arena, Graph, pack

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libgcl_b200.so")

GCL_OK = 0
ERRORS = {
    -1: "invalid argument",
    -2: "CUDA error",
    -3: "out of memory",
    -4: "bad input graph",
    -5: "graph too large",
    -6: "bounded device wait timed out",
    -7: "internal error",
}

# Every symbol include/gcl.h declares.
EXPORTS = [
    "gcl_status_string", "gcl_version", "gcl_create", "gcl_destroy", "gcl_stream",
    "gcl_canon_one", "gcl_canon_batch", "gcl_canon_batch_device_async", "gcl_sync", "gcl_iso",
    "gcl_canon_batch_noalloc", "gcl_set_option", "gcl_canon_wide_device_async",
    "gcl_serve_create", "gcl_serve_destroy", "gcl_serve_submit", "gcl_serve_poll",
    "gcl_serve_stats_get", "gcl_serve_replay", "gcl_group_order", "gcl_perm_group_order",
    "gcl_autotune", "gcl_set_tuning", "gcl_canon_files", "gcl_format_adjacency_device_async",
    "gcl_wide_counters", "gcl_host_alloc", "gcl_host_free", "gcl_canon_batch_mapped",
    "gcl_canon_one_rows",
]

GCL_OPT_WIDE_MIN_N = 1
GCL_OPT_WORKSPACE_BYTES = 2
GCL_OPT_WIDE_MAX_WARPS = 3
GCL_OPT_SMEM_STAGE = 4
GCL_OPT_STREAM_PRIORITY = 5
GCL_OPT_WIDE_GATE = 6
GCL_OPT_WIDE_SHARE = 7
GCL_OPT_COUNTERS = 8
GCL_OPT_WIDE_PROBE = 9
GCL_OPT_BATCH_HANDOFF_MS = 10
GCL_OPT_BATCH_SPLIT = 11

# gcl_wide_counters, in index order (include/gcl.h)
WIDE_COUNTERS = ("items", "items_pruned", "gifts_taken", "gifts_given", "nodes", "leaves",
                 "auts_first", "auts_best", "best_published", "publish_retries",
                 "refine_cycles", "orbit_cycles", "gate_cycles", "gift_wait_cycles",
                 "leaf_cycles", "warp_cycles")
GCL_MAX_N = 65536


class Tuning(ctypes.Structure):
    """Launch shapes of the batched path per size bucket (gcl_tuning)."""
    _fields_ = [("w64_blocks_per_sm", ctypes.c_int), ("sp_blocks_per_sm", ctypes.c_int * 4),
                ("sp_stage", ctypes.c_int * 4), ("w64_ms", ctypes.c_float),
                ("sp_ms", ctypes.c_float * 4)]

    def as_dict(self) -> dict:
        return {"w64_blocks_per_sm": self.w64_blocks_per_sm,
                "sp_blocks_per_sm": list(self.sp_blocks_per_sm),
                "sp_stage": list(self.sp_stage), "w64_ms": self.w64_ms,
                "sp_ms": list(self.sp_ms)}


class GclError(RuntimeError):
    def __init__(self, rc: int, what: str = ""):
        super().__init__(f"{what}: {ERRORS.get(rc, 'error')} (status {rc})")
        self.rc = rc


_P = ctypes.c_void_p
_lib = None
_FILE_CB = ctypes.CFUNCTYPE(None, _P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int,
                            ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int32),
                            ctypes.c_int64, ctypes.c_int64)


def load_library(path: str = LIB_PATH):
    """Load libgcl_b200.so and declare its signatures (no GPU needed)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with python gpu-canonical-labeling_b200/build.py")
    lib = ctypes.CDLL(path)
    lib.gcl_status_string.restype = ctypes.c_char_p
    lib.gcl_status_string.argtypes = [ctypes.c_int]
    lib.gcl_version.restype = ctypes.c_int
    lib.gcl_create.argtypes = [ctypes.c_int, ctypes.POINTER(_P)]
    lib.gcl_destroy.argtypes = [_P]
    lib.gcl_stream.argtypes = [_P]
    lib.gcl_stream.restype = _P
    lib.gcl_sync.argtypes = [_P]
    lib.gcl_canon_one.argtypes = [_P, _P, _P, _P, ctypes.c_int, ctypes.c_int, _P, _P, _P]
    lib.gcl_canon_batch.argtypes = [_P, ctypes.c_int, _P, _P, _P, _P, _P, ctypes.c_int, _P, _P,
                                    _P, _P, _P, _P, _P]
    lib.gcl_canon_batch_device_async.argtypes = [_P, ctypes.c_int, _P, _P, _P, _P, _P,
                                                 ctypes.c_int, ctypes.c_int, ctypes.c_int64, _P,
                                                 _P, _P, _P, _P, _P, _P]
    lib.gcl_iso.argtypes = [_P, _P, _P, _P, ctypes.c_int, _P, _P, _P, ctypes.c_int,
                            ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.gcl_canon_batch_noalloc.argtypes = [_P, ctypes.c_int, _P, _P, _P, _P, _P, ctypes.c_int,
                                            ctypes.c_int, _P, _P, _P, _P, _P]
    lib.gcl_set_option.argtypes = [_P, ctypes.c_int, ctypes.c_int64]
    lib.gcl_canon_files.argtypes = [_P, ctypes.c_int64, ctypes.POINTER(ctypes.c_char_p),
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int, _FILE_CB, _P]
    lib.gcl_autotune.argtypes = [_P, ctypes.c_int, _P, _P, _P, _P, _P, ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(Tuning)]
    lib.gcl_set_tuning.argtypes = [_P, ctypes.POINTER(Tuning)]
    lib.gcl_group_order.argtypes = [_P, _P, _P, _P, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                    ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int64),
                                    ctypes.POINTER(ctypes.c_int)]
    lib.gcl_perm_group_order.argtypes = [ctypes.c_int, _P, ctypes.c_int64,
                                         ctypes.POINTER(ctypes.c_double), ctypes.c_char_p,
                                         ctypes.c_int]
    lib.gcl_canon_wide_device_async.argtypes = [_P, _P, _P, _P, ctypes.c_int, ctypes.c_int64,
                                                ctypes.c_int, _P, _P, _P, _P, _P]
    lib.gcl_format_adjacency_device_async.argtypes = [_P, ctypes.c_int, _P, _P, _P, _P, _P]
    lib.gcl_wide_counters.argtypes = [_P, _P, ctypes.c_int]
    lib.gcl_canon_one_rows.argtypes = [_P, _P, _P, _P, ctypes.c_int, ctypes.c_int, _P, _P, _P]
    lib.gcl_host_alloc.argtypes = [_P, ctypes.c_size_t, ctypes.POINTER(_P)]
    lib.gcl_host_free.argtypes = [_P, _P]
    lib.gcl_canon_batch_mapped.argtypes = [_P, ctypes.c_int, _P, _P, _P, _P, _P, ctypes.c_int,
                                           _P, _P, _P, _P, _P, _P, _P]
    for name in ("gcl_create", "gcl_destroy", "gcl_sync", "gcl_canon_one", "gcl_canon_batch",
                 "gcl_canon_batch_device_async", "gcl_iso", "gcl_canon_batch_noalloc",
                 "gcl_set_option", "gcl_canon_wide_device_async", "gcl_group_order",
                 "gcl_perm_group_order", "gcl_autotune", "gcl_set_tuning",
                 "gcl_canon_files", "gcl_format_adjacency_device_async", "gcl_wide_counters",
                 "gcl_host_alloc", "gcl_host_free", "gcl_canon_batch_mapped",
                 "gcl_canon_one_rows"):
        getattr(lib, name).restype = ctypes.c_int
    _lib = lib
    return lib


def _check(rc: int, what: str):
    if rc != GCL_OK:
        raise GclError(rc, what)


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_P)


class Context:
    """A device context (workspace, stream, staging buffers) on one GPU."""

    def __init__(self, device: int = 0, wide_min_n: Optional[int] = None):
        self.lib = load_library()
        h = _P()
        _check(self.lib.gcl_create(device, ctypes.byref(h)), "gcl_create")
        self.handle = h
        self.device = device
        if wide_min_n is not None:
            self.set_wide_min_n(wide_min_n)

    def autotune(self, graphs, max_aut: int = 10000, repeats: int = 2) -> dict:
        """Time the batched path's launch shapes on a sample (an Arena or a
        list of graphs), keep the fastest per size bucket for this context
        and return the choice (gcl_autotune)."""
        arena = graphs if isinstance(graphs, Arena) else pack(graphs)
        t = Tuning()
        col = arena.col if arena.col.size else np.zeros(1, np.int32)
        color = arena.color if arena.color.any() else None
        _check(self.lib.gcl_autotune(self.handle, arena.count, _ptr(arena.voff), _ptr(arena.eoff),
                                     _ptr(arena.rowptr), _ptr(col), _ptr(color), max_aut, repeats,
                                     ctypes.byref(t)), "gcl_autotune")
        return t.as_dict()

    def set_tuning(self, d: dict):
        """Apply a choice returned by autotune (gcl_set_tuning)."""
        t = Tuning()
        t.w64_blocks_per_sm = int(d.get("w64_blocks_per_sm", 0))
        for k in range(4):
            t.sp_blocks_per_sm[k] = int(d.get("sp_blocks_per_sm", [0] * 4)[k])
            t.sp_stage[k] = int(d.get("sp_stage", [-1] * 4)[k])
        _check(self.lib.gcl_set_tuning(self.handle, ctypes.byref(t)), "gcl_set_tuning")

    def set_wide_min_n(self, n: int):
        """Single graphs with at least n vertices use the wide search
        (GCL_OPT_WIDE_MIN_N); GCL_MAX_N + 1 keeps the sequential traversal."""
        _check(self.lib.gcl_set_option(self.handle, GCL_OPT_WIDE_MIN_N, int(n)),
               "gcl_set_option")

    def set_option(self, option: int, value: int):
        """gcl_set_option: one of the GCL_OPT_* constants."""
        _check(self.lib.gcl_set_option(self.handle, int(option), int(value)), "gcl_set_option")

    def close(self):
        if getattr(self, "handle", None):
            self.lib.gcl_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return int(self.lib.gcl_stream(self.handle) or 0)

    def sync(self):
        _check(self.lib.gcl_sync(self.handle), "gcl_sync")

    def host_array(self, shape, dtype) -> np.ndarray:
        """A numpy array in mapped host memory of this context (gcl_host_alloc),
        for gcl_canon_batch_mapped; freed with the context."""
        dt = np.dtype(dtype)
        count = int(np.prod(shape))
        p = _P()
        _check(self.lib.gcl_host_alloc(self.handle, max(count * dt.itemsize, 1), ctypes.byref(p)),
               "gcl_host_alloc")
        buf = (ctypes.c_uint8 * max(count * dt.itemsize, 1)).from_address(p.value)
        return np.frombuffer(buf, dtype=dt, count=count).reshape(shape)

    def host_free(self, a: np.ndarray):
        """Frees an array from host_array (gcl_host_free); it must not be used after."""
        _check(self.lib.gcl_host_free(self.handle, ctypes.c_void_p(a.ctypes.data)), "gcl_host_free")

    def wide_counters(self) -> dict:
        """Counters of the last wide search on this context, by name
        (gcl_wide_counters; needs GCL_OPT_COUNTERS set before that search)."""
        out = np.zeros(len(WIDE_COUNTERS), dtype=np.int64)
        k = self.lib.gcl_wide_counters(self.handle, _ptr(out), len(out))
        if k < 0:
            _check(k, "gcl_wide_counters")
        return {name: int(out[i]) for i, name in enumerate(WIDE_COUNTERS[:k])}


_default: Optional[Context] = None


def default_context() -> Context:
    global _default
    if _default is None:
        _default = Context(0)
    return _default


@dataclass
class CanonResult:
    matrix: np.ndarray  # n x n uint8
    nodes: int
    num_aut: int


def _csr(g: Graph):
    rp = np.ascontiguousarray(g.rowptr, dtype=np.int32)
    cl = np.ascontiguousarray(g.col, dtype=np.int32)
    if cl.size == 0:
        cl = np.zeros(1, np.int32)
    co = None if g.color is None else np.ascontiguousarray(g.color, dtype=np.int32)
    return rp, cl, co


def canon(g: Graph, max_aut: int = 10000, ctx: Optional[Context] = None) -> CanonResult:
    """Canonical form of one graph (one launch)."""
    ctx = ctx or default_context()
    rp, cl, co = _csr(g)
    out = np.zeros((g.n, g.n), dtype=np.uint8)
    nodes = ctypes.c_int64()
    naut = ctypes.c_int64()
    rc = ctx.lib.gcl_canon_one(ctx.handle, _ptr(rp), _ptr(cl), _ptr(co), g.n, max_aut,
                               _ptr(out if out.size else np.zeros(1, np.uint8)),
                               ctypes.byref(nodes), ctypes.byref(naut))
    _check(rc, "gcl_canon_one")
    return CanonResult(out, int(nodes.value), int(naut.value))


def canon_rows(g: Graph, max_aut: int = 10000, ctx: Optional[Context] = None):
    """(packed rows, nodes, num_aut) of one graph (gcl_canon_one_rows): the
    canonical matrix as n rows of ceil(n/64) words (unpack_rows gives it)."""
    ctx = ctx or default_context()
    rp, cl, co = _csr(g)
    rows = np.zeros(max(g.n * ((g.n + 63) // 64), 1), dtype=np.uint64)
    nodes = ctypes.c_int64()
    naut = ctypes.c_int64()
    rc = ctx.lib.gcl_canon_one_rows(ctx.handle, _ptr(rp), _ptr(cl), _ptr(co), g.n, max_aut,
                                    _ptr(rows), ctypes.byref(nodes), ctypes.byref(naut))
    _check(rc, "gcl_canon_one_rows")
    return rows[: g.n * ((g.n + 63) // 64)], int(nodes.value), int(naut.value)


@dataclass
class FileResult:
    status: int
    n: int
    rows: Optional[np.ndarray]   # packed canonical rows (n * ceil(n/64) words)
    label: Optional[np.ndarray]
    num_aut: int
    nodes: int


def canon_files(paths: Sequence[str], max_aut: int = 10000, ctx: Optional[Context] = None,
                chunk: int = 4096, threads: int = 0) -> List[FileResult]:
    """Canonize DIMACS files, parsing on host threads while the GPU works
    (gcl_canon_files); one FileResult per path, in order."""
    ctx = ctx or default_context()
    out: List[Optional[FileResult]] = [None] * len(paths)

    def cb(_user, index, status, n, rows, label, num_aut, nodes):
        r = l = None
        if status == 0:
            w = n * ((n + 63) // 64)
            r = np.ctypeslib.as_array(rows, shape=(max(w, 1),))[:w].copy() if w else np.zeros(0, np.uint64)
            l = np.ctypeslib.as_array(label, shape=(max(n, 1),))[:n].copy() if n else np.zeros(0, np.int32)
        out[index] = FileResult(int(status), int(n), r, l, int(num_aut), int(nodes))

    arr = (ctypes.c_char_p * max(len(paths), 1))(*[os.fsencode(p) for p in paths])
    fn = _FILE_CB(cb)
    _check(ctx.lib.gcl_canon_files(ctx.handle, len(paths), arr, max_aut, chunk, threads, fn, None),
           "gcl_canon_files")
    return out


def group_order(g: Graph, ctx: Optional[Context] = None, return_checked: bool = False):
    """|Aut(g)| (colour-preserving), exact, from the automorphisms the wide
    search finds (gcl_group_order).  With return_checked, (order, checked):
    checked is 1 when a Schreier-Sims completion confirmed the order, -1 when
    the completion's differing order was returned, 0 when no completion
    finished within its budget (the first path's orbit product, unchecked)."""
    ctx = ctx or default_context()
    rp, cl, co = _csr(g)
    lg = ctypes.c_double()
    ngen = ctypes.c_int64()
    chk = ctypes.c_int()
    buf = ctypes.create_string_buffer(1 << 20)
    rc = ctx.lib.gcl_group_order(ctx.handle, _ptr(rp), _ptr(cl), _ptr(co), g.n, ctypes.byref(lg),
                                 buf, len(buf), ctypes.byref(ngen), ctypes.byref(chk))
    _check(rc, "gcl_group_order")
    order = int(buf.value.decode())
    return (order, chk.value) if return_checked else order


def perm_group_order(perms) -> int:
    """Order of the group generated by the rows of `perms` (count x n
    permutations of 0..n-1), host Schreier-Sims (gcl_perm_group_order)."""
    lib = load_library()
    p = np.ascontiguousarray(perms, dtype=np.uint16)
    if p.ndim != 2:
        raise ValueError("perms must be count x n")
    lg = ctypes.c_double()
    buf = ctypes.create_string_buffer(1 << 20)
    rc = lib.gcl_perm_group_order(p.shape[1], _ptr(p) if p.size else None, p.shape[0],
                                  ctypes.byref(lg), buf, len(buf))
    _check(rc, "gcl_perm_group_order")
    return int(buf.value.decode())


def Nauty_Parallel(g: Graph, max_aut: int = 10000) -> bytes:  # noqa: N802 (reference name)
    """The n*n canonical adjacency bytes, as src/nauty_parallel.h:9-13 returns."""
    return canon(g, max_aut).matrix.tobytes()


def rows_offsets(arena: Arena) -> np.ndarray:
    """Offsets (in 64-bit words) of each graph's packed rows."""
    n = arena.sizes()
    o = np.zeros(arena.count + 1, dtype=np.int64)
    np.cumsum(n * ((n + 63) // 64), out=o[1:])
    return o


def unpack_rows(rows: np.ndarray, n: int) -> np.ndarray:
    """n x n 0/1 matrix from n packed rows of ceil(n/64) words."""
    w = (n + 63) // 64
    bits = np.unpackbits(rows.reshape(n, w).view(np.uint8), axis=1, bitorder="little")
    return bits[:, :n].astype(np.uint8)


@dataclass
class BatchResult:
    dense: Optional[np.ndarray]  # concatenated n_g*n_g blocks
    ooff: np.ndarray
    label: Optional[np.ndarray]  # concatenated per-graph labels
    stats: np.ndarray  # (count, 2): num_aut, nodes
    status: np.ndarray
    arena: Arena
    rows: Optional[np.ndarray] = None  # concatenated packed rows
    roff: Optional[np.ndarray] = None

    def packed(self, g: int) -> np.ndarray:
        return self.rows[self.roff[g]: self.roff[g + 1]]

    def matrix(self, g: int) -> np.ndarray:
        n = int(self.arena.voff[g + 1] - self.arena.voff[g])
        return self.dense[self.ooff[g]: self.ooff[g + 1]].reshape(n, n)

    def labeling(self, g: int) -> np.ndarray:
        return self.label[self.arena.voff[g]: self.arena.voff[g + 1]]


def canon_batch(graphs: Union[Arena, Sequence[Graph]], max_aut: int = 10000,
                ctx: Optional[Context] = None, dense: bool = True,
                label: bool = True, rows: bool = False,
                per_graph_errors: bool = False) -> BatchResult:
    """Canonize every graph of a ragged arena in one batched call.  The call
    fails (GclError) when a graph has no result; with per_graph_errors the
    result comes back anyway and `status` says which graphs have none
    (1 ring outgrown, 2 too large, 3 bad input, 4 internal, 5 time budget)."""
    ctx = ctx or default_context()
    arena = graphs if isinstance(graphs, Arena) else pack(graphs)
    ooff = arena.out_offsets()
    roff = rows_offsets(arena)
    out = np.zeros(max(int(ooff[-1]), 1), dtype=np.uint8) if dense else None
    prow = np.zeros(max(int(roff[-1]), 1), dtype=np.uint64) if rows else None
    lab = np.zeros(max(int(arena.voff[-1]), 1), dtype=np.int32) if label else None
    stats = np.zeros((max(arena.count, 1), 2), dtype=np.int64)
    status = np.zeros(max(arena.count, 1), dtype=np.int32)
    col = arena.col if arena.col.size else np.zeros(1, np.int32)
    color = arena.color if arena.color.any() else None
    rc = ctx.lib.gcl_canon_batch(ctx.handle, arena.count, _ptr(arena.voff), _ptr(arena.eoff),
                                 _ptr(arena.rowptr), _ptr(col), _ptr(color), max_aut, _ptr(out),
                                 _ptr(ooff), _ptr(prow), _ptr(roff), _ptr(lab), _ptr(stats),
                                 _ptr(status))
    per_graph = rc in (-4, -5, -6, -7) and (status[:arena.count] != 0).any()
    if not (per_graph_errors and per_graph):
        _check(rc, "gcl_canon_batch")
    return BatchResult(out, ooff, lab, stats[:arena.count], status[:arena.count], arena,
                       prow, roff)


def canon_batch_mapped(graphs: Union[Arena, Sequence[Graph]], max_aut: int = 10000,
                       ctx: Optional[Context] = None, dense: bool = True, label: bool = True,
                       rows: bool = False) -> BatchResult:
    """canon_batch through gcl_canon_batch_mapped: the arena is copied into
    mapped host memory of the context and the results come back there (no
    staging copies for graphs up to 64 vertices)."""
    ctx = ctx or default_context()
    arena = graphs if isinstance(graphs, Arena) else pack(graphs)
    held = []

    def alloc(shape, dtype):
        held.append(ctx.host_array(shape, dtype))
        return held[-1]

    def mapped(a):
        m = alloc(a.shape, a.dtype)
        m[...] = a
        return m
    ooff = arena.out_offsets()
    roff = rows_offsets(arena)
    voff, eoff, rp = mapped(arena.voff), mapped(arena.eoff), mapped(arena.rowptr)
    col = mapped(arena.col) if arena.col.size else None
    color = mapped(arena.color) if arena.color.any() else None
    m_ooff, m_roff = mapped(ooff), mapped(roff)
    out = alloc((max(int(ooff[-1]), 1),), np.uint8) if dense else None
    prow = alloc((max(int(roff[-1]), 1),), np.uint64) if rows else None
    lab = alloc((max(int(arena.voff[-1]), 1),), np.int32) if label else None
    stats = alloc((max(arena.count, 1), 2), np.int64)
    status = alloc((max(arena.count, 1),), np.int32)
    try:
        rc = ctx.lib.gcl_canon_batch_mapped(ctx.handle, arena.count, _ptr(voff), _ptr(eoff),
                                            _ptr(rp), _ptr(col), _ptr(color), max_aut, _ptr(out),
                                            _ptr(m_ooff), _ptr(prow), _ptr(m_roff), _ptr(lab),
                                            _ptr(stats), _ptr(status))
        _check(rc, "gcl_canon_batch_mapped")
        cp = lambda a: None if a is None else np.array(a)  # noqa: E731  (off the mapped buffers)
        return BatchResult(cp(out), ooff, cp(lab), cp(stats[:arena.count]),
                           cp(status[:arena.count]), arena, cp(prow), roff)
    finally:
        for a in held:
            ctx.host_free(a)


def is_isomorphic(g1: Graph, g2: Graph, max_aut: int = 10000,
                  ctx: Optional[Context] = None) -> bool:
    """main.cpp:172-197: canonize both, compare the upper triangles."""
    ctx = ctx or default_context()
    a, b = _csr(g1), _csr(g2)
    v = ctypes.c_int()
    rc = ctx.lib.gcl_iso(ctx.handle, _ptr(a[0]), _ptr(a[1]), _ptr(a[2]), g1.n, _ptr(b[0]),
                         _ptr(b[1]), _ptr(b[2]), g2.n, max_aut, ctypes.byref(v))
    _check(rc, "gcl_iso")
    return bool(v.value)


# ---------------------------------------------------------------------------
# Serving (gcl_serve_*): continuous batching over several device contexts.
# ---------------------------------------------------------------------------

REQ_CANON = 0
REQ_ISO = 1


class ServeConfig(ctypes.Structure):
    _fields_ = [("lanes", ctypes.c_int), ("mid_lanes", ctypes.c_int), ("big_lanes", ctypes.c_int),
                ("large_lanes", ctypes.c_int), ("max_batch", ctypes.c_int),
                ("mid_batch", ctypes.c_int), ("big_batch", ctypes.c_int), ("mid_n", ctypes.c_int),
                ("big_n", ctypes.c_int), ("large_n", ctypes.c_int), ("max_aut", ctypes.c_int),
                ("lane_bytes", ctypes.c_int64), ("table_slots", ctypes.c_int64),
                ("store_bytes", ctypes.c_int64), ("memo_bytes", ctypes.c_int64),
                ("big_wide", ctypes.c_int)]


class ServeResult(ctypes.Structure):
    _fields_ = [("id", ctypes.c_int64), ("status", ctypes.c_int32), ("verdict", ctypes.c_int32),
                ("repeat", ctypes.c_int32), ("batch", ctypes.c_int32),
                ("class_id", ctypes.c_int64), ("canon_hash", ctypes.c_uint64),
                ("latency_s", ctypes.c_double), ("admit_s", ctypes.c_double),
                ("launch_s", ctypes.c_double), ("gpu_done_s", ctypes.c_double)]


class ServeStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in ("submitted", "completed", "batches", "graphs",
                                              "memo_hits", "class_repeats", "classes",
                                              "large_graphs")] + [
        ("class_batches", ctypes.c_int64 * 4), ("class_batch_ns", ctypes.c_int64 * 4),
        ("class_queue_ns", ctypes.c_int64 * 4), ("class_max_launch_ns", ctypes.c_int64 * 4),
        ("class_max_complete_ns", ctypes.c_int64 * 4), ("enqueue_part_max_ns", ctypes.c_int64 * 6)]


def _serve_sigs(lib):
    if getattr(lib, "_serve_sigs", False):
        return
    lib.gcl_serve_create.argtypes = [ctypes.c_int, ctypes.POINTER(ServeConfig), ctypes.POINTER(_P)]
    lib.gcl_serve_destroy.argtypes = [_P]
    lib.gcl_serve_submit.argtypes = [_P, ctypes.c_int64, ctypes.c_int, _P, _P, _P, ctypes.c_int,
                                     _P, _P, _P, ctypes.c_int, _P, _P]
    lib.gcl_serve_poll.argtypes = [_P, ctypes.POINTER(ServeResult), ctypes.c_int, ctypes.c_int]
    lib.gcl_serve_stats_get.argtypes = [_P, ctypes.POINTER(ServeStats)]
    lib.gcl_serve_replay.argtypes = [_P, ctypes.c_int, _P, _P, _P, _P, ctypes.c_int, _P, _P, _P,
                                     _P, _P, ctypes.c_double, ctypes.POINTER(ServeResult)]
    for name in ("gcl_serve_create", "gcl_serve_destroy", "gcl_serve_submit", "gcl_serve_poll",
                 "gcl_serve_stats_get", "gcl_serve_replay"):
        getattr(lib, name).restype = ctypes.c_int
    lib._serve_sigs = True


class Server:
    """A request loop on one GPU (gcl_serve_create): submit canonization and
    isomorphism requests as they arrive, poll finished results."""

    def __init__(self, device: int = 0, **cfg):
        self.lib = load_library()
        _serve_sigs(self.lib)
        c = ServeConfig()
        for k, v in cfg.items():
            setattr(c, k, v)
        h = _P()
        _check(self.lib.gcl_serve_create(device, ctypes.byref(c), ctypes.byref(h)),
               "gcl_serve_create")
        self.handle = h
        self._keep = {}  # output buffers of requests in flight, by id

    def close(self):
        if getattr(self, "handle", None):
            self.lib.gcl_serve_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit_canon(self, rid: int, g: Graph, want_form: bool = True):
        rp, cl, co = _csr(g)
        rows = np.zeros(max(g.n * ((g.n + 63) // 64), 1), np.uint64) if want_form else None
        lab = np.zeros(max(g.n, 1), np.int32) if want_form else None
        self._keep[rid] = (rows, lab, g.n)
        rc = self.lib.gcl_serve_submit(self.handle, rid, REQ_CANON, _ptr(rp), _ptr(cl), _ptr(co),
                                       g.n, None, None, None, 0, _ptr(rows), _ptr(lab))
        _check(rc, "gcl_serve_submit")

    def submit_iso(self, rid: int, g1: Graph, g2: Graph):
        a, b = _csr(g1), _csr(g2)
        rc = self.lib.gcl_serve_submit(self.handle, rid, REQ_ISO, _ptr(a[0]), _ptr(a[1]),
                                       _ptr(a[2]), g1.n, _ptr(b[0]), _ptr(b[1]), _ptr(b[2]),
                                       g2.n, None, None)
        _check(rc, "gcl_serve_submit")

    def poll(self, max_results: int = 1024, timeout_ms: int = 10):
        """[(result, rows, label)] for finished requests; rows/label are the
        packed canonical form and labeling of canonization requests."""
        buf = (ServeResult * max_results)()
        k = self.lib.gcl_serve_poll(self.handle, buf, max_results, timeout_ms)
        if k < 0:
            _check(k, "gcl_serve_poll")
        out = []
        for i in range(k):
            r = buf[i]
            rows, lab, n = self._keep.pop(r.id, (None, None, 0))
            out.append((r, None if rows is None else rows[: n * ((n + 63) // 64)],
                        None if lab is None else lab[:n]))
        return out

    def stats(self) -> dict:
        s = ServeStats()
        _check(self.lib.gcl_serve_stats_get(self.handle, ctypes.byref(s)), "gcl_serve_stats_get")
        out = {}
        for k, _ in ServeStats._fields_:
            v = getattr(s, k)
            out[k] = [int(x) for x in v] if hasattr(v, "__len__") else int(v)
        return out

    def replay(self, arena: Arena, kind, g1, g2, arrival_s, timeout_s: float = 600.0):
        """Open-loop load (gcl_serve_replay): request i is submitted at
        arrival_s[i]; returns the results in request order (latency from the
        scheduled arrival)."""
        nreq = len(kind)
        kind = np.ascontiguousarray(kind, np.int32)
        g1 = np.ascontiguousarray(g1, np.int32)
        g2 = np.ascontiguousarray(g2, np.int32)
        arr = np.ascontiguousarray(arrival_s, np.float64)
        res = (ServeResult * max(nreq, 1))()
        col = arena.col if arena.col.size else np.zeros(1, np.int32)
        color = arena.color if arena.color.any() else None
        rc = self.lib.gcl_serve_replay(self.handle, nreq, _ptr(arr), _ptr(kind), _ptr(g1),
                                       _ptr(g2), arena.count, _ptr(arena.voff), _ptr(arena.eoff),
                                       _ptr(arena.rowptr), _ptr(col), _ptr(color), timeout_s, res)
        _check(rc, "gcl_serve_replay")
        return [res[i] for i in range(nreq)]
