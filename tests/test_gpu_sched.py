"""The learned schedule picker on the GPU: its features equal a numpy
computation from the solver's state, every action yields the oracle's exact
flow (certified), state copies are exact, the CUDA inference matches the numpy
forward pass of the same bf16 weights, the CUDA training learns a synthetic
rule, and scheduled batches give the same flows as the plain schedule."""
import numpy as np
import pytest

from make_golden import make_config

pytestmark = pytest.mark.gpu


def certify(oracle, g, sv, s, t, want):
    off, adj, _, par = g.arrays()
    cap, res, ex, _ = sv.state()
    rc, val, cut = oracle.certify(g.num_nodes(), off, adj, cap, par, res, s, t)
    assert rc == 0 and val == want == cut


def numpy_features(g, sv, batch):
    """The 12 features of csrc/dmf_sched.cu (make_features) from the host side."""
    off, adj, _, par = g.arrays()
    cap, res, _, _ = sv.state()
    st = sv.stats()
    n, m = g.num_nodes(), g.num_edges()
    valid = dec = satdec = incsat = ins = dele = sdeg = mdeg = 0
    exc = 0
    for u, v, w in zip(*batch):
        u, v, w = int(u), int(v), int(w)
        if u == v or not (0 <= u < n and 0 <= v < n):
            continue
        e = g.find_arc(u, v)
        if e < 0:
            continue
        valid += 1
        c0, r = int(cap[e]), int(res[e])
        flow = c0 - r
        d = int(off[u + 1] - off[u])
        sdeg += d
        mdeg = max(mdeg, d)
        if w < c0:
            dec += 1
            if flow > w:
                satdec += 1
                exc += flow - w
        elif w > c0 and r == 0:
            incsat += 1
        if c0 == 0 and w > 0:
            ins += 1
        if c0 > 0 and w == 0:
            dele += 1
    k = len(batch[0])
    f32 = np.float32
    vd = max(1.0, valid)
    return np.array([
        k / max(1, m), np.log2(1 + k) / 24, dec / vd, satdec / vd, min(1.0, exc / max(1.0, st["flow"])),
        incsat / vd, ins / vd, dele / vd, np.log2(1 + sdeg / vd) / 16, np.log2(1 + mdeg) / 24,
        np.log2(1 + st["bfs_levels"] / max(1.0, st["outer_iters"])) / 16, np.log2(1 + n) / 32], f32)


def test_features_match_numpy(dmf):
    g, s, t, batches = make_config("rmat12")
    with dmf.Solver(g, s, t) as sv:
        sv.static_maxflow()
        for b in batches[:3]:
            got = sv.features(*b)
            np.testing.assert_allclose(got, numpy_features(g, sv, b), rtol=1e-5, atol=1e-6)
            sv.apply_updates(*b)


@pytest.mark.parametrize("name", ["rmat12", "grid256"])
def test_every_action_exact_and_copy_state(dmf, oracle, name):
    g, s, t, batches = make_config(name)
    off, adj, w, par = g.arrays()
    n = g.num_nodes()
    cur = w.copy()
    with dmf.Solver(g, s, t) as trunk, dmf.Solver(g, s, t) as scratch:
        trunk.static_maxflow()
        for b in batches[:2]:
            for a, c, x in zip(*b):
                if a != c:
                    cur[g.find_arc(int(a), int(c))] = x
            want = oracle.dinic(n, off, adj, cur, par, s, t)
            for action in range(dmf.N_ACTIONS):
                scratch.copy_state_from(trunk)
                for x, y in zip(scratch.state(), trunk.state()):
                    np.testing.assert_array_equal(x, y)
                assert scratch.apply_updates_action(action, *b) == want
                certify(oracle, g, scratch, s, t, want)
            trunk.copy_state_from(scratch)
            assert trunk.flow == want


def test_predict_matches_numpy_forward(dmf):
    from dyn_maxflow_b200 import sched
    rng = np.random.default_rng(3)
    X = rng.uniform(0, 1, size=(257, 12)).astype(np.float32)
    with dmf.Scheduler(seed=11) as sc:
        w, b = sc.get_weights()
        b = (b + rng.normal(0, 0.1, size=b.shape)).astype(np.float32)
        sc.set_weights(w, b)
        got = sc.predict(X)
        want = sched.forward_reference(w, b, X)
        # fp32 accumulation in a different order: agreement to fp32 rounding
        np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-4)
        w2, b2 = sc.get_weights()
        np.testing.assert_array_equal(w2, w)
        np.testing.assert_array_equal(b2, b)


def test_training_learns_a_rule(dmf):
    """Targets with a known cheapest action per region of feature space."""
    rng = np.random.default_rng(5)
    X = rng.uniform(0, 1, size=(4096, 12)).astype(np.float32)
    Y = np.stack([2.0 * X[:, 0] + 0.5,
                  2.0 - 2.0 * X[:, 0] + 0.3 * X[:, 3],
                  1.2 + 0.5 * X[:, 5],
                  3.0 - 2.5 * X[:, 1]], 1).astype(np.float32)
    with dmf.Scheduler(seed=1) as sc:
        loss = sc.train(X, Y, steps=3000, batch=64, lr=3e-3, seed=2)
        assert np.isfinite(loss).all()
        assert loss[-100:].mean() < 0.05 * loss[:20].mean()
        Xt = rng.uniform(0, 1, size=(1024, 12)).astype(np.float32)
        Yt = np.stack([2.0 * Xt[:, 0] + 0.5, 2.0 - 2.0 * Xt[:, 0] + 0.3 * Xt[:, 3], 1.2 + 0.5 * Xt[:, 5],
                       3.0 - 2.5 * Xt[:, 1]], 1)
        acc = (sc.predict(Xt).argmin(1) == Yt.argmin(1)).mean()
        assert acc > 0.85, acc


def test_scheduled_batches_equal_plain_and_records(dmf, oracle):
    g, s, t, batches = make_config("rmat12")
    off, adj, w, par = g.arrays()
    cur = w.copy()
    with dmf.Scheduler(seed=4) as sc:
        # a model that prefers recompute on large batches and the short interval otherwise
        X = np.random.default_rng(0).uniform(0, 1, size=(2048, 12)).astype(np.float32)
        Y = np.stack([np.full(2048, 1.0), 0.5 + 10 * X[:, 0], np.full(2048, 2.0), 1.5 - 10 * X[:, 0]], 1)
        sc.train(X, Y.astype(np.float32), steps=1500, seed=1)
        with dmf.Solver(g, s, t) as P, dmf.Solver(g, s, t) as L:
            P.static_maxflow()
            L.static_maxflow()
            picks = []
            for b in batches:
                for a, c, x in zip(*b):
                    if a != c:
                        cur[g.find_arc(int(a), int(c))] = x
                want = oracle.dinic(g.num_nodes(), off, adj, cur, par, s, t)
                fp, ap = P.apply_updates_scheduled(None, *b)
                fl, al = L.apply_updates_scheduled(sc, *b)
                assert ap == 0 and fp == fl == want
                picks.append(al)
            feat, act, ms, fl = L.sched_records()
            assert len(act) == len(batches) and list(act) == picks
            assert (ms > 0).all() and feat.shape == (len(batches), 12)
            assert L.sched_records()[1].size == 0  # drained
            certify(oracle, g, L, s, t, int(fl[-1]))
