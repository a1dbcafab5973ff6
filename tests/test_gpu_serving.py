"""Serving loop: graphs admitted by HBM budget, continuous batching of
update-batch requests; each result is the same alone and in the mix."""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _graphs(dmf):
    from dyn_maxflow_b200 import workloads
    return workloads.batched(count=8, steps=4, seed=11, median=600, lo=64, hi=3000)


def test_admission_by_budget(dmf):
    inst = _graphs(dmf)
    graphs = [x[0] for x in inst]
    # per arc: heads, partners, residuals, 8-byte capacity words (20 B) and the
    # arc table (16-byte slots, 2m + 64 of them); 64 B per vertex
    need = [20 * g.num_edges() + 16 * (2 * g.num_edges() + 64) + 64 * g.num_nodes() for g in graphs]
    budget = sum(need[:3]) + need[3] // 2  # room for the first three only
    with dmf.Server(graphs, [x[1] for x in inst], [x[2] for x in inst], budget) as srv:
        assert srv.admitted == 3 and srv.device_bytes == sum(need[:3])
        with pytest.raises(dmf.DmfError):
            srv.submit(3, [0], [1], [1])  # not admitted
    with pytest.raises(dmf.DmfError) as ei:
        dmf.Server(graphs, [x[1] for x in inst], [x[2] for x in inst], 16)
    assert ei.value.status == 5


def test_mixed_results_equal_alone(dmf, oracle):
    inst = _graphs(dmf)
    graphs, S, T = [x[0] for x in inst], [x[1] for x in inst], [x[2] for x in inst]
    # alone: each graph's request sequence on its own solver, one request at a time
    alone = []
    for g, s, t, batches in inst:
        with dmf.Solver(g, s, t) as sv:
            sv.static_maxflow()
            alone.append([sv.apply_updates(*b) for b in batches])
    # and independently: Dinic on the capacities after each request
    for i, (g, s, t, batches) in enumerate(inst):
        off, adj, w, par = g.arrays()
        cur = w.copy()
        for j, b in enumerate(batches):
            for a, c, x in zip(*b):
                cur[g.find_arc(int(a), int(c))] = x
            assert alone[i][j] == oracle.dinic(g.num_nodes(), off, adj, cur, par, s, t)
    # in the mix: every graph's requests submitted from its own thread, all at once
    got = [[None] * len(inst[0][3]) for _ in inst]
    lat = []
    with dmf.Server(graphs, S, T, 1 << 34) as srv:
        assert srv.admitted == len(inst)

        def client(i):
            tickets = [srv.submit(i, *b) for b in inst[i][3]]
            for j, tk in enumerate(tickets):
                got[i][j], l = srv.wait(tk)
                lat.append(l)

        th = [threading.Thread(target=client, args=(i,)) for i in range(len(inst))]
        for x in th:
            x.start()
        for x in th:
            x.join()
        st = srv.stats()
    assert got == alone
    assert st["served"] == sum(len(x[3]) for x in inst)
    assert st["mean_requests_per_tick"] > 1.0  # requests of different graphs shared launches
    assert min(lat) > 0


def test_bad_requests_are_rejected_alone(dmf):
    inst = _graphs(dmf)
    g, s, t, batches = inst[0]
    with dmf.Server([g], [s], [t], 1 << 30) as srv:
        n = g.num_nodes()
        missing = next((a, b) for a in range(n) for b in range(n) if a != b and g.find_arc(a, b) < 0)
        with pytest.raises(dmf.DmfError) as ei:
            srv.submit(0, [missing[0]], [missing[1]], [3])
        assert ei.value.status == 3
        tk = srv.submit(0, *batches[0])
        f, _ = srv.wait(tk)
        with dmf.Solver(g, s, t) as sv:
            sv.static_maxflow()
            assert f == sv.apply_updates(*batches[0])


def test_one_waiter_per_ticket(dmf):
    """Two threads waiting on one ticket: one gets the flow, the other an
    invalid-argument error (the ticket is taken, or already gone)."""
    inst = _graphs(dmf)
    g, s, t, batches = inst[0]
    with dmf.Solver(g, s, t) as sv:
        sv.static_maxflow()
        want = sv.apply_updates(*batches[0])
    with dmf.Server([g], [s], [t], 1 << 30) as srv:
        for _ in range(3):
            tk = srv.submit(0, *batches[0])
            out = []

            def waiter():
                try:
                    out.append(("flow", srv.wait(tk)[0]))
                except dmf.DmfError as e:
                    out.append(("error", e.status))

            th = [threading.Thread(target=waiter) for _ in range(2)]
            for x in th:
                x.start()
            for x in th:
                x.join()
            # updates set capacities, so the same batch again gives the same flow
            assert sorted(out) == [("error", 1), ("flow", want)]


def test_destroy_serves_pending_and_blocked_waiters(dmf):
    """close() serves every submitted request; a thread blocked in wait() gets
    its exact result, and tickets nobody waits for are freed."""
    inst = _graphs(dmf)
    alone = []
    for g, s, t, batches in inst:
        with dmf.Solver(g, s, t) as sv:
            sv.static_maxflow()
            alone.append([sv.apply_updates(*b) for b in batches])
    srv = dmf.Server([x[0] for x in inst], [x[1] for x in inst], [x[2] for x in inst], 1 << 34)
    tickets = [[srv.submit(i, *b) for b in x[3]] for i, x in enumerate(inst)]
    got, entered = [], threading.Event()

    def waiter():
        entered.set()
        got.append(srv.wait(tickets[0][-1])[0])

    th = threading.Thread(target=waiter)
    th.start()
    entered.wait()
    time.sleep(0.3)  # the waiter is inside wait() before close() starts
    srv.close()
    th.join(timeout=60)
    assert not th.is_alive() and got == [alone[0][-1]]


def test_large_requests_validated_in_parallel(dmf, oracle):
    """Requests of 16k+ updates take the parallel validation path: a repeated
    arc, an unknown arc, an out-of-range vertex and an out-of-range capacity
    are each rejected with their status, and nothing of a rejected request is
    applied; a valid large request is served with the exact flow."""
    g, s, t, (b,) = make_config_rmat14_one()
    k = len(b[0])
    assert k >= 16384
    off, adj, w, par = g.arrays()
    n = g.num_nodes()
    with dmf.Server([g], [s], [t], 1 << 31) as srv:
        src, dst, cap = (x.copy() for x in b)
        dup = (np.concatenate([src, src[:1]]), np.concatenate([dst, dst[:1]]), np.concatenate([cap, cap[:1]]))
        with pytest.raises(dmf.DmfError) as ei:
            srv.submit(0, *dup)
        assert ei.value.status == 4  # DMF_ERR_DUP_ARC
        missing = next((a, c) for a in range(n) for c in range(n) if a != c and g.find_arc(a, c) < 0)
        unk = (src.copy(), dst.copy(), cap.copy())
        unk[0][k // 2], unk[1][k // 2] = missing
        with pytest.raises(dmf.DmfError) as ei:
            srv.submit(0, *unk)
        assert ei.value.status == 3  # DMF_ERR_UNKNOWN_ARC
        oor = (src.copy(), dst.copy(), cap.copy())
        oor[1][k - 1] = n
        with pytest.raises(dmf.DmfError) as ei:
            srv.submit(0, *oor)
        assert ei.value.status == 1
        big = (src.copy(), dst.copy(), cap.copy())
        big[2][7] = 1 << 30
        with pytest.raises(dmf.DmfError) as ei:
            srv.submit(0, *big)
        assert ei.value.status == 1
        f, _ = srv.wait(srv.submit(0, src, dst, cap))
    cur = w.copy()
    for a, c, x in zip(src, dst, cap):
        if a != c:
            cur[g.find_arc(int(a), int(c))] = x
    assert f == oracle.dinic(n, off, adj, cur, par, s, t)


def make_config_rmat14_one():
    """R-MAT 14 with one batch of 8% of its arcs (about 40k updates)."""
    import dyn_maxflow_b200 as D
    narcs = 16 << 14
    g, s, t = D.gen_rmat(14, narcs, 0.57, 0.19, 0.19, seed=0, cap_lo=1, cap_hi=1000, reserve=narcs // 50)
    b = D.gen_batches(g, 1, frac=0.08, p_inc=0.4, p_dec=0.4, p_ins=0.1, delta_hi=500, ins_lo=1, ins_hi=1000, seed=3)
    return g, s, t, b


def test_small_request_overlaps_large_one(dmf, oracle):
    """A graph with most of the arcs gets a lane of its own; a request for a small
    graph, submitted while a large request (1M updates on a 1024 x 1024 grid, a
    solve of many latency-bound phases) is in flight on it, is served on the
    other lane and completes first, with the flow it has alone."""
    import dyn_maxflow_b200 as D
    big, bs, bt = D.gen_grid(1024, 1024, seed=5, cap_lo=1, cap_hi=100, st_cap=1000)
    positive = int((big.arrays()[2] > 0).sum())
    (bb,) = D.gen_batches(big, 1, frac=min(0.5, 1_050_000 / positive), p_inc=0.5, p_dec=0.5, p_ins=0.0,
                          delta_hi=50, seed=6)
    assert len(bb[0]) >= 1_000_000
    inst = _graphs(dmf)
    graphs = [big] + [x[0] for x in inst]
    S, T = [bs] + [x[1] for x in inst], [bt] + [x[2] for x in inst]
    # alone
    with dmf.Solver(big, bs, bt) as sv:
        sv.static_maxflow()
        capacity = sv.stats()["grid_blocks"]  # resident blocks of an uncapped solver
        want_big = sv.apply_updates(*bb)
    g1, s1, t1, b1 = inst[0]
    with dmf.Solver(g1, s1, t1) as sv:
        sv.static_maxflow()
        want_small = sv.apply_updates(*b1[0])
    off, adj, w, par = g1.arrays()
    cur = w.copy()
    for a, c, x in zip(*b1[0]):
        if a != c:
            cur[g1.find_arc(int(a), int(c))] = x
    assert want_small == oracle.dinic(g1.num_nodes(), off, adj, cur, par, s1, t1)
    with dmf.Server(graphs, S, T, 1 << 36) as srv:
        lb, ls = srv.lane(0), srv.lane(1)
        assert lb["lanes"] == 2 and lb["lane"] != ls["lane"]
        assert lb["grid_blocks"] + ls["grid_blocks"] <= capacity
        done = {}

        def waiter(name, tk):
            f, _ = srv.wait(tk)
            done[name] = (time.perf_counter(), f)

        tk_big = srv.submit(0, *bb)
        th_big = threading.Thread(target=waiter, args=("big", tk_big))
        th_big.start()
        tk_small = srv.submit(1, *b1[0])
        waiter("small", tk_small)
        th_big.join()
    assert done["small"][1] == want_small and done["big"][1] == want_big
    assert done["small"][0] < done["big"][0], done  # the small request finished first
