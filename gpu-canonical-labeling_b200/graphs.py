"""Graph model, DIMACS-style I/O, seeded generators and the ragged CSR arena.

The in-memory graph is the reference's ``CSRGraph`` (CSRGraph.h:6-39):
``rowptr[n+1]`` / ``col[2m]`` int32 with both directions stored, every row
sorted ascending, no self loops, plus ``color[n]`` int32 (0 = uncoloured).

``read_dimacs`` follows ``CSRGraph::fromDIMACS`` (CSRGraph.cpp:40-119)
line for line in behaviour: ``c`` lines and empty lines are skipped, ``p``
sets the vertex count (the edge count on that line is ignored), ``n v c``
sets a colour (1-based, vertex 0 ignored, out-of-range ignored), ``e u v``
is 1-based, self loops are dropped and both directions are inserted.  The
reference keeps duplicate ``e`` lines as parallel edges, which its
refinement does not handle (partition_refinement.cpp:296-303 assumes a
singleton splitter yields counts in {0, 1}); this module reports them as
``ValueError`` instead of producing undefined output.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Iterable, List, Optional, Sequence, Tuple

import numpy as np


@dataclass
class Graph:
    """Undirected, optionally vertex-coloured graph in CSR form."""

    n: int
    rowptr: np.ndarray  # int32[n+1]
    col: np.ndarray  # int32[2m]
    color: Optional[np.ndarray] = None  # int32[n] or None (all zero)

    @property
    def m(self) -> int:
        return int(self.rowptr[-1]) // 2

    def edges(self) -> np.ndarray:
        """Undirected edge list (u < v), shape (m, 2), lexicographic order."""
        src = np.repeat(np.arange(self.n, dtype=np.int32), np.diff(self.rowptr))
        mask = src < self.col
        return np.stack([src[mask], self.col[mask]], axis=1)

    def colors(self) -> np.ndarray:
        if self.color is None:
            return np.zeros(self.n, dtype=np.int32)
        return self.color

    def adjacency(self) -> np.ndarray:
        """Dense n x n uint8 adjacency matrix."""
        a = np.zeros((self.n, self.n), dtype=np.uint8)
        src = np.repeat(np.arange(self.n), np.diff(self.rowptr))
        a[src, self.col] = 1
        return a


def from_edges(n: int, edges: Iterable[Tuple[int, int]] | np.ndarray,
               color: Optional[Sequence[int]] = None) -> Graph:
    """Build the CSR the way CSRGraph::fromDIMACS does (0-based edges)."""
    e = np.asarray(list(edges) if not isinstance(edges, np.ndarray) else edges,
                   dtype=np.int64).reshape(-1, 2)
    if e.size and (e.min() < 0 or e.max() >= n):
        raise ValueError("edge endpoint out of range")
    e = e[e[:, 0] != e[:, 1]]  # self loops dropped (CSRGraph.cpp:74)
    both = np.concatenate([e, e[:, ::-1]], axis=0)
    order = np.lexsort((both[:, 1], both[:, 0]))
    both = both[order]
    if len(both) > 1:
        dup = np.all(both[1:] == both[:-1], axis=1)
        if dup.any():
            raise ValueError("duplicate edge (parallel edges are not supported)")
    deg = np.bincount(both[:, 0], minlength=n) if len(both) else np.zeros(n, np.int64)
    rowptr = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(deg, out=rowptr[1:])
    col = both[:, 1].astype(np.int32)
    c = None
    if color is not None:
        c = np.asarray(color, dtype=np.int32).copy()
        if c.shape != (n,):
            raise ValueError("color must have n entries")
        if not c.any():
            c = None
    return Graph(n, rowptr, col, c)


_BLANK = " \t\r\v\f\n"
_UINT_MAX = 2**32 - 1
_INT_MAX = 2**31 - 1


class _LineReader:
    """Extractions from one line with the rules of std::istringstream >> x,
    which CSRGraph::fromDIMACS applies to every line (CSRGraph.cpp:50-79):
    blanks skipped; at the end of the line an extraction fails and leaves its
    target alone; a number is an optional sign and decimal digits up to the
    first non-digit, no digits store 0 and an overflow the type's limit; a
    failed extraction stops the rest of the line."""

    def __init__(self, line: str):
        self.s, self.i, self.failed = line, 0, False

    def _sentry(self) -> bool:
        if self.failed:
            return False
        while self.i < len(self.s) and self.s[self.i] in _BLANK:
            self.i += 1
        if self.i == len(self.s):
            self.failed = True
            return False
        return True

    def char(self, default: str) -> str:
        if not self._sentry():
            return default
        self.i += 1
        return self.s[self.i - 1]

    def word(self) -> None:
        if self._sentry():
            while self.i < len(self.s) and self.s[self.i] not in _BLANK:
                self.i += 1

    def _number(self):
        neg = False
        if self.s[self.i] in "+-":
            neg = self.s[self.i] == "-"
            self.i += 1
        j = self.i
        while self.i < len(self.s) and "0" <= self.s[self.i] <= "9":
            self.i += 1
        return neg, (int(self.s[j:self.i]) if self.i > j else None)

    def uint(self, default: int) -> int:
        if not self._sentry():
            return default
        neg, mag = self._number()
        if mag is None or mag > _UINT_MAX:
            self.failed = True
            return 0 if mag is None else _UINT_MAX
        return (-mag) % 2**32 if neg else mag

    def int(self, default: int) -> int:
        if not self._sentry():
            return default
        neg, mag = self._number()
        if mag is None:
            self.failed = True
            return 0
        v = -mag if neg else mag
        if v > _INT_MAX or v < -_INT_MAX - 1:
            self.failed = True
            return _INT_MAX if v > 0 else -_INT_MAX - 1
        return v


def parse_dimacs(text: str) -> Graph:
    """Parse DIMACS text with CSRGraph::fromDIMACS semantics (CSRGraph.cpp:40-119):
    'c' lines and empty lines skipped, the first non-blank character is the
    line type, 'p <word> <n> <m>' sets n, 'n <v> <colour>' colours vertex v
    (1-based, 0 or > n ignored), 'e <u> <v>' adds an edge (1-based, self loops
    dropped), other types ignored.  Where the reference is undefined -- an
    endpoint of 0 or above n, a repeated edge -- ValueError is raised, as the
    C++ reader of the library (csrc/gcl_dimacs.h) rejects the file."""
    n = 0
    edges: List[Tuple[int, int]] = []
    colors: List[Tuple[int, int]] = []
    for line in text.split("\n"):
        if not line or line[0] == "c":
            continue
        r = _LineReader(line)
        t = r.char("\0")
        if t == "p":
            r.word()
            n = r.uint(n)
            r.uint(0)
        elif t == "n":
            vid = r.uint(0)
            col = r.int(0)
            if vid != 0:
                colors.append((vid - 1, col))
        elif t == "e":
            u = r.uint(0)
            v = r.uint(0)
            if u == v:
                continue
            if u == 0 or v == 0 or u > n or v > n:
                raise ValueError("edge endpoint out of range")
            edges.append((u - 1, v - 1))
    color = np.zeros(n, dtype=np.int32)
    for v, c in colors:
        if v < n:
            color[v] = c
    return from_edges(n, edges, color)


def read_dimacs(path: str) -> Graph:
    with open(path, "r", newline="") as f:
        return parse_dimacs(f.read())


def to_dimacs(g: Graph) -> str:
    e = g.edges()
    out = [f"p edge {g.n} {len(e)}"]
    if g.color is not None:
        out += [f"n {v + 1} {int(c)}" for v, c in enumerate(g.color) if c != 0]
    out += [f"e {u + 1} {v + 1}" for u, v in e]
    return "\n".join(out) + "\n"


def write_dimacs(g: Graph, path: str) -> None:
    with open(path, "w") as f:
        f.write(to_dimacs(g))


def relabel(g: Graph, perm: np.ndarray) -> Graph:
    """Graph with vertex v renamed perm[v] (colours move with vertices)."""
    perm = np.asarray(perm, dtype=np.int64)
    e = g.edges()
    ne = perm[e] if len(e) else e
    col = None
    if g.color is not None:
        col = np.zeros(g.n, dtype=np.int32)
        col[perm] = g.color
    return from_edges(g.n, ne, col)


def random_relabel(g: Graph, rng: np.random.Generator) -> Graph:
    return relabel(g, rng.permutation(g.n))


# --------------------------------------------------------------------------
# Seeded generators for the benchmark workloads.
# --------------------------------------------------------------------------

def erdos_renyi(n: int, p: float, rng: np.random.Generator) -> Graph:
    iu, ju = np.triu_indices(n, 1)
    keep = rng.random(len(iu)) < p
    return from_edges(n, np.stack([iu[keep], ju[keep]], axis=1))


def move_one_edge(g: Graph, rng: np.random.Generator) -> Graph:
    """Copy with one random edge moved to a random non-edge."""
    e = g.edges().tolist()
    adj = set(map(tuple, e))
    k = int(rng.integers(len(e)))
    del e[k]
    while True:
        u, v = sorted(int(x) for x in rng.choice(g.n, 2, replace=False))
        if (u, v) not in adj:
            break
    e.append((u, v))
    return from_edges(g.n, e, g.color)


def random_regular(n: int, d: int, rng: np.random.Generator,
                   max_tries: int = 10000) -> Graph:
    """Random simple d-regular graph: configuration model rejected until
    simple, falling back (when the whole-pairing acceptance rate is tiny,
    e.g. d = 6) to pairing stubs one edge at a time among the pairs that keep
    the graph simple, restarting on a dead end (Steger-Wormald)."""
    if (n * d) % 2:
        raise ValueError("n*d must be even")
    stubs = np.repeat(np.arange(n), d)
    for _ in range(min(max_tries, 200)):
        p = rng.permutation(stubs).reshape(-1, 2)
        if np.any(p[:, 0] == p[:, 1]):
            continue
        a = np.sort(p, axis=1)
        key = a[:, 0].astype(np.int64) * n + a[:, 1]
        if len(np.unique(key)) != len(key):
            continue
        return from_edges(n, a)
    for _ in range(max_tries):
        free = list(stubs)
        edges = set()
        ok = True
        while free:
            for _attempt in range(100):
                i, j = rng.choice(len(free), 2, replace=False)
                u, v = free[i], free[j]
                if u != v and (min(u, v), max(u, v)) not in edges:
                    break
            else:
                ok = False
                break
            edges.add((min(u, v), max(u, v)))
            for k in sorted((i, j), reverse=True):
                free[k] = free[-1]
                free.pop()
        if ok:
            return from_edges(n, np.array(sorted(edges)))
    raise RuntimeError("no simple regular graph found")


def torus(k1: int, k2: Optional[int] = None) -> Graph:
    """Toroidal grid C_k1 x C_k2 (k >= 3)."""
    k2 = k1 if k2 is None else k2
    e = []
    for i in range(k1):
        for j in range(k2):
            v = i * k2 + j
            e.append((v, i * k2 + (j + 1) % k2))
            e.append((v, ((i + 1) % k1) * k2 + j))
    e = np.array([(min(a, b), max(a, b)) for a, b in e])
    e = np.unique(e, axis=0)
    return from_edges(k1 * k2, e)


def disjoint_union(g: Graph, k: int) -> Graph:
    e = g.edges()
    parts = [e + i * g.n for i in range(k)]
    col = None if g.color is None else np.tile(g.color, k)
    return from_edges(g.n * k, np.concatenate(parts) if len(e) else e, col)


def cfi_graph(base_n: int, rng: np.random.Generator, twist: bool = False) -> Graph:
    """Cai-Fuerer-Immerman gadget graph over a random cubic base graph of
    `base_n` vertices (10 * base_n vertices).  Each base vertex becomes four
    middle vertices (the even subsets of its three edges) and a pair of end
    vertices per edge; a middle vertex joins end 1 of the edges in its subset
    and end 0 of the others; the ends of a base edge are joined 0-0 and 1-1
    (0-1 and 1-0 on the first edge when `twist`).  Colour refinement leaves
    these graphs nearly undivided, so their search trees are deep with many
    inequivalent leaves."""
    base = random_regular(base_n, 3, rng)
    be = [tuple(int(x) for x in e) for e in base.edges()]
    inc: List[List[int]] = [[] for _ in range(base_n)]
    for k, (u, v) in enumerate(be):
        inc[u].append(k)
        inc[v].append(k)
    ends = {}
    nid = 4 * base_n
    for v in range(base_n):
        for k in inc[v]:
            for bit in (0, 1):
                ends[(v, k, bit)] = nid
                nid += 1
    edges = []
    subsets = [(), (0, 1), (0, 2), (1, 2)]
    for v in range(base_n):
        for si, sub in enumerate(subsets):
            m = 4 * v + si
            for t, k in enumerate(inc[v]):
                edges.append((m, ends[(v, k, 1 if t in sub else 0)]))
    for k, (u, v) in enumerate(be):
        flip = 1 if (twist and k == 0) else 0
        for bit in (0, 1):
            edges.append((ends[(u, k, bit)], ends[(v, k, bit ^ flip)]))
    return from_edges(nid, edges)


def prufer_tree(n: int, rng: np.random.Generator, max_deg: int = 4) -> List[Tuple[int, int]]:
    """Uniform labelled tree (Pruefer sequence) rejected until max degree <= max_deg."""
    if n <= 2:
        return [(0, 1)] if n == 2 else []
    while True:
        seq = rng.integers(0, n, n - 2)
        deg = np.bincount(seq, minlength=n) + 1
        if deg.max() <= max_deg:
            break
    deg = deg.tolist()
    edges = []
    import heapq
    leaves = [v for v in range(n) if deg[v] == 1]
    heapq.heapify(leaves)
    for x in seq.tolist():
        leaf = heapq.heappop(leaves)
        edges.append((leaf, x))
        deg[x] -= 1
        if deg[x] == 1:
            heapq.heappush(leaves, x)
    u = heapq.heappop(leaves)
    v = heapq.heappop(leaves)
    edges.append((u, v))
    return edges


def recursive_tree(n: int, rng: np.random.Generator, max_deg: int = 4) -> List[Tuple[int, int]]:
    """Random tree with max degree <= max_deg for sizes where rejecting
    Pruefer sequences is hopeless (the chance that a uniform tree on n
    vertices has max degree <= 4 falls like exp(-0.019 n)): vertices arrive in
    a random order and each attaches to a uniformly chosen earlier vertex of
    degree < max_deg."""
    if n <= 1:
        return []
    order = rng.permutation(n)
    deg = np.zeros(n, dtype=np.int64)
    open_ = [int(order[0])]  # vertices with spare degree
    edges = []
    for i in range(1, n):
        v = int(order[i])
        j = int(rng.integers(len(open_)))
        u = open_[j]
        edges.append((u, v))
        deg[u] += 1
        deg[v] += 1
        if deg[u] >= max_deg:
            open_[j] = open_[-1]
            open_.pop()
        open_.append(v)
    return edges


def tree_plus_edges(n: int, rng: np.random.Generator, max_deg: int = 4,
                    max_extra: int = 6) -> Graph:
    """Pruefer tree (max degree 4) plus U{0..max_extra} ring-closing edges
    drawn uniformly among non-edges that keep the max degree <= max_deg.
    Above 128 vertices the tree comes from ``recursive_tree`` and the extra
    edges from rejection sampling (same distribution of extra edges)."""
    tree = prufer_tree(n, rng, max_deg) if n <= 128 else recursive_tree(n, rng, max_deg)
    edges = [(min(a, b), max(a, b)) for a, b in tree]
    deg = np.zeros(n, dtype=np.int64)
    adj = set(edges)
    for a, b in edges:
        deg[a] += 1
        deg[b] += 1
    extra = int(rng.integers(0, max_extra + 1))
    adjm = None
    if n <= 128:
        adjm = np.zeros((n, n), dtype=bool)
        for a, b in edges:
            adjm[a, b] = True
    for _ in range(extra):
        free = np.nonzero(deg < max_deg)[0]
        if n <= 128:
            # every non-adjacent pair of free vertices, in (i, j) row order
            iu, ju = np.triu_indices(len(free), 1)
            ca, cb = free[iu], free[ju]
            keep = ~adjm[ca, cb]
            ca, cb = ca[keep], cb[keep]
            if ca.size == 0:
                break
            k = int(rng.integers(ca.size))
            a, b = int(ca[k]), int(cb[k])
        else:
            if len(free) < 2:
                break
            while True:  # uniform over non-adjacent pairs of free vertices
                i, j = rng.choice(len(free), 2, replace=False)
                a, b = int(min(free[i], free[j])), int(max(free[i], free[j]))
                if (a, b) not in adj:
                    break
        adj.add((a, b))
        if adjm is not None:
            adjm[a, b] = True
        edges.append((a, b))
        deg[a] += 1
        deg[b] += 1
    return from_edges(n, edges)


def small_batch(count: int = 10000, seed: int = 3000, n_lo: int = 10, n_hi: int = 64,
                relabel_frac: float = 0.2) -> List[Graph]:
    """Batched small-graph workload: ``count`` graphs, n ~ U[n_lo, n_hi],
    Pruefer tree (max degree 4) + 0-6 extra edges; ``relabel_frac`` of them
    are random relabelings of earlier graphs (to exercise deduplication)."""
    rng = np.random.default_rng(seed)
    out: List[Graph] = []
    for i in range(count):
        if i > 0 and rng.random() < relabel_frac:
            src = out[int(rng.integers(len(out)))]
            out.append(random_relabel(src, rng))
        else:
            n = int(rng.integers(n_lo, n_hi + 1))
            out.append(tree_plus_edges(n, rng))
    return out


def mixed_batch(count: int = 2000, seed: int = 4000, n_lo: int = 64,
                n_hi: int = 4096) -> List[Graph]:
    """Mixed-size workload: n log-uniform in [n_lo, n_hi], four families in
    equal shares (ER mean degree 8, random d-regular d in {3,4,6}, toroidal
    grids, disjoint unions of 2-4 copies of one random regular component)."""
    rng = np.random.default_rng(seed)
    out: List[Graph] = []
    for i in range(count):
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        fam = i % 4
        if fam == 0:
            out.append(erdos_renyi(n, min(1.0, 8.0 / max(n - 1, 1)), rng))
        elif fam == 1:
            d = int(rng.choice([3, 4, 6]))
            if (n * d) % 2:
                n += 1
            out.append(random_regular(n, d, rng))
        elif fam == 2:
            k1 = max(3, int(round(math.sqrt(n) * rng.uniform(0.7, 1.3))))
            k2 = max(3, int(round(n / k1)))
            out.append(torus(k1, k2))
        else:
            # a few copies of one larger component: the reference's search
            # (first-leaf and per-level orbit pruning only) grows exponentially
            # in the number of identical components
            k = int(rng.choice([2, 3, 4]))
            c = max(8, n // k)
            d = 3 if c % 2 == 0 else 4
            comp = random_regular(c, d, rng)
            out.append(disjoint_union(comp, k))
    return out


@dataclass
class ServingWorkload:
    """An open-loop request stream over a pool of graphs: request i arrives
    at ``arrival[i]`` seconds and is a canonization of ``graphs[g1[i]]``
    (kind 0) or an isomorphism query between ``graphs[g1[i]]`` and
    ``graphs[g2[i]]`` (kind 1)."""

    graphs: List[Graph]
    kind: np.ndarray
    g1: np.ndarray
    g2: np.ndarray
    arrival: np.ndarray


def serving_size(rng: np.random.Generator, n_lo: int = 10, n_mid: int = 128,
                 n_big: int = 2048, n_max: int = 20000) -> int:
    """Heavy-tailed request size: 90% uniform on [n_lo, n_mid], 9%
    log-uniform on (n_mid, n_big], 1% log-uniform on (n_big, n_max]."""
    u = rng.random()
    if u < 0.90:
        return int(rng.integers(n_lo, n_mid + 1))
    lo, hi = (n_mid, min(n_big, n_max)) if u < 0.99 else (min(n_big, n_max), n_max)
    if hi <= lo + 1:
        return int(hi)
    return int(min(hi, max(lo + 1, round(math.exp(rng.uniform(math.log(lo + 1), math.log(hi)))))))


def serving_workload(count: int, rate: float, seed: int = 5000, iso_frac: float = 0.3,
                     repeat_frac: float = 0.2, n_max: int = 20000) -> ServingWorkload:
    """Poisson arrivals at ``rate`` requests/s.  Graphs are the batched
    workload's family (tree of max degree 4 plus 0-6 extra edges) with the
    heavy-tailed sizes of ``serving_size``.  ``iso_frac`` of the requests are
    isomorphism pairs, half of them a random relabeling (isomorphic) and half
    a copy with one edge moved (almost always not); ``repeat_frac`` of the
    canonization requests re-ask an earlier graph under a random relabeling
    (the canonical-hash table's repeats)."""
    rng = np.random.default_rng(seed)
    graphs: List[Graph] = []
    kind = np.zeros(count, np.int32)
    g1 = np.zeros(count, np.int32)
    g2 = np.zeros(count, np.int32)
    canon_ids: List[int] = []
    for i in range(count):
        if rng.random() < iso_frac:
            a = tree_plus_edges(serving_size(rng, n_max=n_max), rng)
            b = random_relabel(a, rng) if rng.random() < 0.5 else move_one_edge(a, rng)
            graphs += [a, b]
            kind[i], g1[i], g2[i] = 1, len(graphs) - 2, len(graphs) - 1
            continue
        if canon_ids and rng.random() < repeat_frac:
            src = graphs[canon_ids[int(rng.integers(len(canon_ids)))]]
            graphs.append(random_relabel(src, rng))
        else:
            graphs.append(tree_plus_edges(serving_size(rng, n_max=n_max), rng))
        g1[i] = g2[i] = len(graphs) - 1
        canon_ids.append(len(graphs) - 1)
    arrival = np.cumsum(rng.exponential(1.0 / rate, count))
    return ServingWorkload(graphs, kind, g1, g2, arrival - arrival[0])


# --------------------------------------------------------------------------
# Ragged CSR arena (the batched input format).
# --------------------------------------------------------------------------

@dataclass
class Arena:
    """Many graphs packed back to back.

    Graph g owns vertices ``[voff[g], voff[g+1])`` and CSR entries
    ``[eoff[g], eoff[g+1])``; its local rowptr (n_g + 1 entries, starting at
    0) sits at ``rowptr[voff[g] + g : voff[g+1] + g + 1]``.  ``color`` is
    vertex-indexed like ``voff`` (all zero when uncoloured).
    """

    count: int
    voff: np.ndarray  # int64[count+1]
    eoff: np.ndarray  # int64[count+1]
    rowptr: np.ndarray  # int32[voff[-1] + count]
    col: np.ndarray  # int32[eoff[-1]]
    color: np.ndarray  # int32[voff[-1]]

    def sizes(self) -> np.ndarray:
        return np.diff(self.voff)

    def graph(self, g: int) -> Graph:
        a, b = int(self.voff[g]), int(self.voff[g + 1])
        rp = self.rowptr[a + g: b + g + 1].copy()
        col = self.col[int(self.eoff[g]): int(self.eoff[g + 1])].copy()
        c = self.color[a:b].copy()
        return Graph(b - a, rp, col, c if c.any() else None)

    def out_offsets(self) -> np.ndarray:
        """Offsets of each graph's n*n output block in a dense output arena."""
        n = self.sizes()
        o = np.zeros(self.count + 1, dtype=np.int64)
        np.cumsum(n * n, out=o[1:])
        return o


def shard_ranges(sizes: Sequence[int], world: int) -> List[Tuple[int, int]]:
    """Split graphs 0..len(sizes) into `world` contiguous ranges of nearly
    equal cost, the cost of a graph taken as n^2 + 1 (its canonical matrix and
    a search that grows with n).  Each rank canonizes its range on its own
    GPU; the only exchange is gathering the results."""
    cost = np.asarray(sizes, dtype=np.float64) ** 2 + 1.0
    cum = np.concatenate([[0.0], np.cumsum(cost)])
    cuts = [0]
    for r in range(1, world):
        cuts.append(int(np.searchsorted(cum, cum[-1] * r / world, side="left")))
    cuts.append(len(sizes))
    cuts = np.maximum.accumulate(np.asarray(cuts))
    return [(int(cuts[r]), int(cuts[r + 1])) for r in range(world)]


def pack(graphs: Sequence[Graph]) -> Arena:
    count = len(graphs)
    ns = np.array([g.n for g in graphs], dtype=np.int64)
    ms = np.array([len(g.col) for g in graphs], dtype=np.int64)
    voff = np.zeros(count + 1, dtype=np.int64)
    eoff = np.zeros(count + 1, dtype=np.int64)
    np.cumsum(ns, out=voff[1:])
    np.cumsum(ms, out=eoff[1:])
    rowptr = (np.concatenate([g.rowptr for g in graphs]).astype(np.int32)
              if count else np.zeros(0, np.int32))
    col = (np.concatenate([g.col for g in graphs]).astype(np.int32)
           if count else np.zeros(0, np.int32))
    color = (np.concatenate([g.colors() for g in graphs]).astype(np.int32)
             if count else np.zeros(0, np.int32))
    return Arena(count, voff, eoff, rowptr, col, color)
