"""Group order of graphs whose automorphism groups have large orbits, where
the Schreier-Sims check of gcl_group_order (general, then on the first
path's base images) may exceed its budget and the first path's basic orbits
give the order unchecked.  The host part is checked on the CPU
(tests/test_group_base.py)."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = [pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA GPU")]


@pytest.mark.gpu
def test_group_order_large_vertex_transitive(pkg, G):
    ctx = pkg.Context(0)
    # checked: 1 confirmed by a completion, 0 unchecked within the budget;
    # never -1 (a completion that disagrees with the orbit product)
    order, checked = pkg.group_order(G.torus(100), ctx=ctx, return_checked=True)
    assert order == 8 * 100 * 100 and checked in (0, 1)
    d = 12
    cube = G.from_edges(1 << d, [(a, a ^ (1 << b)) for a in range(1 << d) for b in range(d)
                                 if a < a ^ (1 << b)])
    order, checked = pkg.group_order(cube, ctx=ctx, return_checked=True)
    assert order == (1 << d) * math.factorial(d) and checked in (0, 1)


@pytest.mark.gpu
def test_group_order_long_base(pkg, G):
    # S_200 (about 8 s on a B200; S_300 takes 35 s, S_600 minutes: the wide
    # search of an empty graph visits O(n^2) nodes per level): both
    # Schreier-Sims checks run out of budget, and the first path's basic
    # orbits give the order, reported as unchecked
    ctx = pkg.Context(0)
    order, checked = pkg.group_order(G.from_edges(200, []), ctx=ctx, return_checked=True)
    assert order == math.factorial(200) and checked == 0
