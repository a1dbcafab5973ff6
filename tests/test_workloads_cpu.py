"""CPU checks of the host-side workload builders that the batched, learned and
serving configurations use: instance sizes and kinds, successive batches that
are valid on the capacities left by the previous ones, the union of many
instances' batches in one vertex numbering, and the R-MAT instances with
reserved insert slots."""
import math

import numpy as np


def _kind(g, s, t):
    """Grids have side * side vertices with s and t at opposite corners;
    R-MAT graphs have 2^scale vertices."""
    n = g.num_nodes()
    side = int(round(math.sqrt(n)))
    if side * side == n and (s, t) == (0, n - 1):
        return "grid"
    assert n & (n - 1) == 0, n
    return "rmat"


def test_batched_instances_follow_the_spec(dmf):
    from dyn_maxflow_b200 import workloads
    lo, hi = 500, 8000
    inst = workloads.batched(count=8, steps=3, seed=5, median=2000, lo=lo, hi=hi)
    assert len(inst) == 8
    assert [_kind(g, s, t) for g, s, t, _ in inst] == ["grid", "rmat"] * 4
    for i, (g, s, t, batches) in enumerate(inst):
        n = g.num_nodes()
        # sizes: clipped to [lo, hi] before a grid side or an R-MAT scale is rounded
        assert lo / 2 <= n <= 2 * hi and s != t and 0 <= s < n and 0 <= t < n
        assert len(batches) == 3
        off, adj, w, par = g.arrays()
        cur = w.copy()
        for src, dst, nw in batches:
            arcs = np.array([g.find_arc(int(a), int(b)) for a, b in zip(src, dst)])
            assert arcs.min() >= 0 and len(set(arcs.tolist())) == len(arcs)  # existing, distinct
            pos = int((cur > 0).sum())
            # fractions drawn from U[0.5%, 5%] of the arcs with capacity
            assert 0.005 * pos - 2 <= len(arcs) <= 0.05 * pos + 2
            old = cur[arcs]
            assert (old > 0).all()  # half increases, half decreases, no inserts
            assert (nw >= 0).all() and (nw != old).any()
            cur[arcs] = nw  # the next batch is drawn on these capacities
    # reproducible from the seed
    again = workloads.batched(count=8, steps=3, seed=5, median=2000, lo=lo, hi=hi)
    for (g, s, t, b), (g2, s2, t2, b2) in zip(inst, again):
        assert (s, t) == (s2, t2)
        for x, y in zip(g.arrays(), g2.arrays()):
            np.testing.assert_array_equal(x, y)
        for bb, bb2 in zip(b, b2):
            for x, y in zip(bb, bb2):
                np.testing.assert_array_equal(x, y)


def test_union_steps_renumber_and_concatenate(dmf):
    from dyn_maxflow_b200 import workloads
    inst = workloads.batched(count=4, steps=2, seed=1, median=1500, lo=500, hi=4000)
    base = np.cumsum([0] + [g.num_nodes() for g, _, _, _ in inst])[:-1]
    ofs, src, dst, w = workloads.union_steps(inst, base)
    assert ofs.tolist()[0] == 0 and len(ofs) == 3 and ofs[-1] == len(src) == len(dst) == len(w)
    assert src.dtype == dst.dtype == w.dtype == np.int32
    for b in range(2):
        pos = ofs[b]
        for i, (g, _, _, batches) in enumerate(inst):
            s, d, c = batches[b]
            k = len(s)
            np.testing.assert_array_equal(src[pos:pos + k], s + base[i])
            np.testing.assert_array_equal(dst[pos:pos + k], d + base[i])
            np.testing.assert_array_equal(w[pos:pos + k], c)
            # every renumbered update stays inside its instance's vertex range
            assert (src[pos:pos + k] >= base[i]).all() and (src[pos:pos + k] < base[i] + g.num_nodes()).all()
            pos += k
        assert pos == ofs[b + 1]


def test_rmat_instance_reserves_insert_slots_and_mixes_batches(dmf):
    from dyn_maxflow_b200 import sched
    g, s, t = sched.rmat_instance(10, 7)
    off, adj, w, par = g.arrays()
    n = g.num_nodes()
    assert n == 1024 and s != t
    tail = np.repeat(np.arange(n), np.diff(off))
    outdeg = np.bincount(tail[w > 0], minlength=n)
    assert outdeg[s] == outdeg.max()
    # reserved slots: zero-capacity arcs whose partner is zero too, at least the requested count
    assert ((w == 0) & (w[par] == 0)).sum() // 2 >= int(0.02 * (16 << 10)) + 16
    src, dst, nw = sched.next_batch(g, 0.05, 11)
    arcs = np.array([g.find_arc(int(a), int(b)) for a, b in zip(src, dst)])
    assert arcs.min() >= 0 and len(set(arcs.tolist())) == len(arcs)
    old = w[arcs]
    ins = int(((old == 0) & (nw > 0)).sum())
    dele = int(((old > 0) & (nw == 0)).sum())
    # the 40/40/10/10 mix: inserts about a tenth; capacities that end at zero
    # are the tenth of deletes plus the decreases (by U[1,500] on caps
    # U[1,1000]) that reach zero, a quarter of them: ~20% in all
    assert 0.05 * len(arcs) <= ins <= 0.15 * len(arcs)
    assert 0.12 * len(arcs) <= dele <= 0.28 * len(arcs)
    assert (nw[old == 0] <= 1000).all() and (nw >= 0).all()
