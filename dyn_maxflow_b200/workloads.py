"""Seeded synthetic workloads beyond the single-graph benchmark.

batched(): independent instances with log-normal sizes (median 20k vertices,
clipped to [1k, 200k]), half 4-neighbour grids and half R-MAT graphs
(a, b, c = 0.57, 0.19, 0.19, average out-degree 8), capacities U[1,1000], each
with `steps` successive update batches touching U[0.5%, 5%] of its arcs
(half increases, half decreases).  Sizes, seeds and fractions all come from
`seed`, so a workload is reproducible.
"""
from __future__ import annotations

import math

import numpy as np

from . import gen_batches, gen_grid, gen_rmat


def batched(count=256, steps=5, seed=0, median=20000, lo=1000, hi=200000, sigma=1.0, out_degree=8):
    rng = np.random.default_rng(seed)
    sizes = np.clip(np.exp(rng.normal(math.log(median), sigma, count)), lo, hi).astype(np.int64)
    inst = []
    for i, nv in enumerate(sizes):
        iseed = int(rng.integers(1 << 31))
        if i % 2 == 0:
            side = max(2, int(round(math.sqrt(nv))))
            g, s, t = gen_grid(side, side, seed=iseed, cap_lo=1, cap_hi=1000, st_cap=1000)
        else:
            scale = max(2, int(round(math.log2(nv))))
            g, s, t = gen_rmat(scale, out_degree << scale, 0.57, 0.19, 0.19, seed=iseed, cap_lo=1, cap_hi=1000)
        fracs = rng.uniform(0.005, 0.05, steps)
        batches = []
        # successive batches: each is drawn on the capacities left by the previous ones
        cur = g
        for b in range(steps):
            (bt,) = gen_batches(cur, 1, frac=float(fracs[b]), p_inc=0.5, p_dec=0.5, p_ins=0.0, delta_hi=500,
                                seed=iseed + 7919 * (b + 1))
            batches.append(bt)
            if b + 1 < steps:
                cur = _with_caps(cur, bt)
        inst.append((g, s, t, batches))
    return inst


def _with_caps(g, batch):
    from . import Graph
    off, adj, w, par = g.arrays()
    h = Graph.from_csr(off, adj, w, par)
    h.set_caps(*batch)
    return h


def union_steps(instances, vertex_base):
    """Per step, the concatenated batch of every instance in union vertex ids:
    -> (ofs[steps+1], src, dst, w)."""
    steps = len(instances[0][3])
    S, D, W, ofs = [], [], [], [0]
    for b in range(steps):
        for i, (_, _, _, batches) in enumerate(instances):
            s, d, w = batches[b]
            S.append(s + vertex_base[i])
            D.append(d + vertex_base[i])
            W.append(w)
        ofs.append(ofs[-1] + sum(len(x[3][b][0]) for x in instances))
    cat = lambda xs: np.ascontiguousarray(np.concatenate(xs), dtype=np.int32)
    return np.array(ofs, np.int64), cat(S), cat(D), cat(W)
