"""Lane-parallel reformulations in the kernels, restated in Python and
checked on the CPU against the serial forms they replace:

* `mash_fold_mask` (csrc/gcl_device.cuh): the reference's invariant hash
  mash(l, i) = ((l ^ 065435) + i) & 077777 (partition_refinement.h:9-19)
  folded over up to 32 items one bit position at a time -- each item's flip
  of bit j is 065435_j ^ i_j ^ carry_j, the bit before item k is bit j of
  the start value xor the parity of the earlier flips (a ballot's prefix
  popcount), and that gives the carries into bit j + 1;
* the warp kernel's active set after a non-singleton split
  (csrc/canon_warp64.cuh, w64_refine; partition_refinement.cpp:436-460):
  every new fragment enters; for a split cell that was not active, its
  first fragment enters and its first largest fragment leaves -- computed
  from one maximum of (size, -position) per cell instead of a walk over the
  fragments;
* the warp kernel's orbit computation (w64_orbits): union-find over packed
  parent words with one hook round per automorphism, against plain
  component labelling;
* the warp kernel's singleton splitter step (w64_refine): the split cells
  handled lane-parallel, against the serial per-cell loop it replaced.
"""
import random

C, M = 0o65435, 0o77777


def mash(l, i):
    return ((l ^ C) + i) & M


def fold_bits(lc, items, mask):
    """mash_fold_mask: lane k holds items[k]; lanes outside mask are ignored."""
    carry = [0] * 32
    out = 0
    for j in range(15):
        cj, x0 = (C >> j) & 1, (lc >> j) & 1
        flip = [((cj ^ ((items[k] >> j) & 1) ^ carry[k]) if (mask >> k) & 1 else 0)
                for k in range(32)]
        ballot = sum(f << k for k, f in enumerate(flip))
        for k in range(32):
            vj = (items[k] >> j) & 1
            y = x0 ^ (bin(ballot & ((1 << k) - 1)).count("1") & 1) ^ cj
            carry[k] = (y & vj) | (y & carry[k]) | (vj & carry[k])
        out |= (x0 ^ (bin(ballot).count("1") & 1)) << j
    return out


def test_mash_fold_equals_serial_chain():
    rng = random.Random(3)
    for _ in range(1500):
        mask = rng.getrandbits(32) or 1
        items = [rng.randrange(0, 1 << 17) for _ in range(32)]
        lc = rng.randrange(0, 1 << 17)
        ref = lc
        for k in range(32):
            if (mask >> k) & 1:
                ref = mash(ref, items[k])
        assert fold_bits(lc, items, mask) == ref & M


def _ctz(x):
    return (x & -x).bit_length() - 1


def _msb(x):
    return x.bit_length() - 1


def _low(k):
    return (1 << k) - 1


def _ge(k):
    return ((1 << 64) - 1) & ~_low(k) if k < 64 else 0


def active_serial(n, starts, ns, active):
    all_ = starts | ns
    was = active
    active |= ns
    t = ns
    while t:
        c = _msb(starts & _low(_ctz(t)))
        nc = starts & _ge(c + 1)
        end = _ctz(nc) if nc else n
        t &= ~_low(end)
        if (was >> c) & 1:
            continue
        fr = all_ & _ge(c) & _low(end)
        maxsz, maxp = 0, c
        while fr:
            f = _ctz(fr)
            fr &= fr - 1
            sz = (_ctz(fr) if fr else end) - f
            if sz > maxsz:
                maxsz, maxp = sz, f
        active |= 1 << c
        active &= ~(1 << maxp)
    return active


def active_parallel(n, starts, ns, active):
    all_ = starts | ns
    best, frags = {}, []
    for v in range(n):
        if not (all_ >> v) & 1:
            continue
        cell = _msb(starts & _low(v + 1))
        nc = starts & _ge(cell + 1)
        end = _ctz(nc) if nc else n
        nf = all_ & _ge(v + 1)
        fr = not (active >> cell) & 1 and (ns & _low(end) & _ge(cell + 1)) != 0
        key = ((min(_ctz(nf) if nf else n, end) - v) << 6) | (63 - v)
        frags.append((v, cell, fr, key))
        if fr:
            best[cell] = max(best.get(cell, 0), key)
    out = sum(1 << v for v, c, fr, key in frags if fr and best[c] == key)
    inn = sum(1 << v for v, c, fr, key in frags if fr and c == v)
    return (active | ns | inn) & ~out


def test_w64_active_set_equals_serial_walk():
    rng = random.Random(1)
    for _ in range(5000):
        n = rng.randint(1, 64)
        starts = 1 | sum(1 << p for p in range(1, n) if rng.random() < 0.3)
        ns = sum(1 << p for p in range(1, n) if not (starts >> p) & 1 and rng.random() < 0.2)
        active = sum(1 << p for p in range(n) if rng.random() < 0.4)
        assert active_serial(n, starts, ns, active) == active_parallel(n, starts, ns, active)


# ---------------------------------------------------------------------------
# w64_orbits (csrc/canon_warp64.cuh; compute_orbits_fast, perm_group.cpp:5-116):
# the components of the graph joining every vertex v to its previous orbit's
# label L(v) and to pi(v) for each selected automorphism pi, labelled by their
# least vertex -- computed by union-find with parent(v) = L(v) to start, a
# hook round per automorphism (each disagreeing edge offers min(root) to
# par[max(root)], atomicMin) and pointer jumping after every round.
# ---------------------------------------------------------------------------

def _components(n, L, perms):
    adj = [set() for _ in range(n)]
    for v in range(n):
        adj[v].add(L[v])
        adj[L[v]].add(v)
        for p in perms:
            adj[v].add(p[v])
            adj[p[v]].add(v)
    lab = [-1] * n
    for s in range(n):
        if lab[s] >= 0:
            continue
        comp, stack = [s], [s]
        lab[s] = s
        while stack:
            x = stack.pop()
            for y in adj[x]:
                if lab[y] < 0:
                    lab[y] = s
                    comp.append(y)
                    stack.append(y)
        m = min(comp)
        for x in comp:
            lab[x] = m
    return lab


def _union_find_lanes(n, L, perms):
    fp = list(L)

    def compress():
        for _ in range(10):
            nxt = [fp[fp[v]] for v in range(n)]
            changed = nxt != fp
            fp[:] = nxt
            if not changed:
                return True
        return False

    assert compress()
    for p in perms:
        for _ in range(n + 1):
            ra = list(fp)
            rb = [fp[p[v]] for v in range(n)]
            if all(a == b for a, b in zip(ra, rb)):
                break
            par = list(fp)
            for v in range(n):
                if ra[v] != rb[v]:
                    hi, lo = max(ra[v], rb[v]), min(ra[v], rb[v])
                    par[hi] = min(par[hi], lo)
            fp[:] = par
            assert compress()
        else:
            raise AssertionError("hook rounds did not converge")
    return fp


def test_w64_orbit_union_find_equals_components():
    rng = random.Random(7)
    for _ in range(3000):
        n = rng.randint(1, 64)
        # previous orbits: a random partition, each block labelled by its least vertex
        blocks = list(range(n))
        for v in range(n):
            if rng.random() < 0.5:
                blocks[v] = blocks[rng.randrange(0, v + 1)]
        least = {}
        for v in range(n):
            least.setdefault(blocks[v], v)
        L = [least[blocks[v]] for v in range(n)]
        perms = []
        for _ in range(rng.randint(1, 3)):
            p = list(range(n))
            # a random permutation made of a few random cycles (automorphism-like)
            pts = rng.sample(range(n), rng.randint(0, n))
            for i, x in enumerate(pts):
                p[x] = pts[(i + 1) % len(pts)]
            perms.append(p)
        assert _union_find_lanes(n, L, perms) == _components(n, L, perms)


# ---------------------------------------------------------------------------
# w64_refine's singleton splitter step (csrc/canon_warp64.cuh;
# partition_refinement.cpp:296-465): the split cells handled serially in
# position order, against the lane-parallel form (each cell split by the lane
# owning its start; active, start and singleton additions OR-ed; the hash over
# the split cells in position order; the hint from the last split cell in
# position order that sets one).
# ---------------------------------------------------------------------------

def _split_serial(n, starts, cmask, active, hint, sing, lc, N):
    cmask = dict(cmask)
    split = sorted(c for c in range(n) if (starts >> c) & 1
                   and cmask[c] & N and cmask[c] & ~N & ((1 << n) - 1))
    cs = {}
    for c in split:
        C = cmask[c]
        CN, CR = C & N, C & ~N
        nb, nn = bin(CN).count("1"), bin(CR).count("1")
        p = c + nb
        lc = mash(lc, p - 1)
        if (active >> c) & 1 or nb >= nn:
            active |= 1 << p
            if nn == 1:
                hint = p
        else:
            active |= 1 << c
            if nb == 1:
                hint = c
        starts |= 1 << p
        if nb == 1:
            sing |= CN
        if nn == 1:
            sing |= CR
        cmask[c], cmask[p] = CN, CR
        for v in range(n):
            if (CR >> v) & 1:
                cs[v] = p
    return starts, active, hint, sing, lc, cmask, cs


def _split_parallel(n, starts, cmask, active, hint, sing, lc, N):
    owner = {}
    addA = addS = addG = 0
    hv = {}
    nb_of = {}
    for c in range(n):  # lane-parallel: the lane owning start c
        if not ((starts >> c) & 1) or not (cmask[c] & N and cmask[c] & ~N & ((1 << n) - 1)):
            continue
        C = cmask[c]
        CN, CR = C & N, C & ~N
        nb, nn = bin(CN).count("1"), bin(CR).count("1")
        p = c + nb
        if (active >> c) & 1 or nb >= nn:
            addA |= 1 << p
            if nn == 1:
                hv[c] = p
        else:
            addA |= 1 << c
            if nb == 1:
                hv[c] = c
        addS |= 1 << p
        if nb == 1:
            addG |= CN
        if nn == 1:
            addG |= CR
        owner[c] = (CN, CR, p)
        nb_of[c] = nb
    for c in sorted(owner):
        lc = mash(lc, c + nb_of[c] - 1)
    if hv:
        hint = hv[max(hv)]
    cmask = dict(cmask)
    cs = {}
    for c, (CN, CR, p) in owner.items():
        cmask[c], cmask[p] = CN, CR
        for v in range(n):
            if (CR >> v) & 1:
                cs[v] = p
    return starts | addS, active | addA, hint, sing | addG, lc, cmask, cs


def test_w64_singleton_split_parallel_equals_serial():
    rng = random.Random(11)
    for _ in range(3000):
        n = rng.randint(2, 64)
        # a random ordered partition: cells are runs of positions, members random vertices
        verts = list(range(n))
        rng.shuffle(verts)
        starts, cmask, pos = 1, {}, 0
        while pos < n:
            size = rng.randint(1, max(1, min(n - pos, rng.choice((1, 2, 3, 8, 64)))))
            starts |= 1 << pos
            cmask[pos] = sum(1 << v for v in verts[pos:pos + size])
            pos += size
        sing = 0
        for c, m in cmask.items():
            if bin(m).count("1") == 1:
                sing |= m
        for c in range(n):
            cmask.setdefault(c, rng.getrandbits(64) & ((1 << n) - 1))  # stale entries
        active = sum(1 << c for c in range(n) if (starts >> c) & 1 and rng.random() < 0.4)
        hint = rng.randrange(n)
        lc = rng.randrange(1 << 15)
        N = sum(1 << v for v in range(n) if rng.random() < 0.3)
        a = _split_serial(n, starts, cmask, active, hint, sing, lc, N)
        b = _split_parallel(n, starts, cmask, active, hint, sing, lc, N)
        assert a == b
