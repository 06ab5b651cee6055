"""Two lane-parallel reformulations in the kernels, restated in Python and
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
  fragments.
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
