"""Parity of the sm_100a solver (through the C ABI) with the CPU oracle.

Every flow value must be bit-exact with the oracle's Dinic on the same
capacities, and every final device state must pass the oracle's certificate
(capacity bounds, pseudoflow accounting, no residual path from an active vertex
or from s to t/deficits, min-cut capacity == flow)."""
import os

import numpy as np
import pytest

from make_golden import make_config

pytestmark = pytest.mark.gpu

VARIANTS = ("data", "topo", "pp")


def certify(oracle, g, sv, s, t, want):
    off, adj, _, par = g.arrays()
    cap, res, ex, _ = sv.state()
    rc, val, cut = oracle.certify(g.num_nodes(), off, adj, cap, par, res, s, t)
    assert rc == 0, f"certificate failed with code {rc}"
    assert val == want == cut
    # the device excess equals the pseudoflow accounting of the residuals
    tail = np.repeat(np.arange(g.num_nodes()), np.diff(off))
    acc = np.zeros(g.num_nodes(), np.int64)
    np.add.at(acc, tail, res.astype(np.int64) - cap.astype(np.int64))
    np.testing.assert_array_equal(acc, ex)


def apply_host(g, cur, batch):
    for a, b, c in zip(*batch):
        if a != b:
            cur[g.find_arc(int(a), int(b))] = c


@pytest.mark.parametrize("variant", VARIANTS)
def test_johnson_static_and_each_file(dmf, oracle, golden_dir, variant):
    g = dmf.Graph.load(os.path.join(golden_dir, "johnson8-2-4.bin"))
    off, adj, w, par = g.arrays()
    n, m = g.num_nodes(), g.num_edges()
    for kc in (m // n - 1, m // n, m // n + 1):
        for i in range(1, 11):
            batch = dmf.load_updates(os.path.join(golden_dir, f"johnson_p{i}.bin"))
            cur = w.copy()
            apply_host(g, cur, batch)
            want = oracle.dinic(n, off, adj, cur, par, 25, 2)
            with dmf.Solver(g, 25, 2, variant=variant, kernel_cycles=kc) as sv:
                assert sv.static_maxflow() == 540
                certify(oracle, g, sv, 25, 2, 540)
                assert sv.apply_updates(*batch) == want
                certify(oracle, g, sv, 25, 2, want)
            assert dmf.recalculate_max_flow(g, batch, 25, 2, kc, variant) == want
            assert dmf.static_recalculate(g, batch, 25, 2, kc, variant) == want


@pytest.mark.parametrize("variant", VARIANTS)
def test_grid256_static_and_batch(dmf, oracle, variant):
    g, s, t, (batch,) = make_config("grid256")
    off, adj, w, par = g.arrays()
    n = g.num_nodes()
    want0 = oracle.dinic(n, off, adj, w, par, s, t)
    cur = w.copy()
    apply_host(g, cur, batch)
    want1 = oracle.dinic(n, off, adj, cur, par, s, t)
    with dmf.Solver(g, s, t, variant=variant) as sv:
        assert sv.static_maxflow() == want0
        certify(oracle, g, sv, s, t, want0)
        assert sv.apply_updates(*batch) == want1
        certify(oracle, g, sv, s, t, want1)
        assert sv.recompute() == want1


@pytest.mark.parametrize("fixed", [False, True])
@pytest.mark.parametrize("interval", [1, 24, 400])
def test_long_push_phases_keep_the_source_closed(dmf, oracle, interval, fixed):
    """Many push rounds between global relabels lift vertices far above their
    BFS distance; excess must still never drain back into s (a source with a
    finite label lets it, and the solve then ends with an augmenting path)."""
    g, s, t, (batch,) = make_config("grid256")
    off, adj, w, par = g.arrays()
    want0 = oracle.dinic(g.num_nodes(), off, adj, w, par, s, t)
    with dmf.Solver(g, s, t, relabel_interval=interval, fixed_interval=fixed) as sv:
        assert sv.static_maxflow() == want0
        certify(oracle, g, sv, s, t, want0)
        cap, res, ex, h = sv.state()
        assert h[s] >= g.num_nodes()


@pytest.mark.parametrize("name", ["rmat12", "rmat14"])
@pytest.mark.parametrize("variant", VARIANTS)
def test_rmat_successive_batches(dmf, oracle, name, variant):
    g, s, t, batches = make_config(name)
    off, adj, w, par = g.arrays()
    n = g.num_nodes()
    cur = w.copy()
    with dmf.Solver(g, s, t, variant=variant) as sv:
        assert sv.static_maxflow() == oracle.dinic(n, off, adj, cur, par, s, t)
        for b in batches:
            apply_host(g, cur, b)
            want = oracle.dinic(n, off, adj, cur, par, s, t)
            assert sv.apply_updates(*b) == want
            certify(oracle, g, sv, s, t, want)
        # from-scratch recompute on the final capacities agrees
        assert sv.recompute() == want


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("name", ["rmat14", "grid256", "rmat16"])
def test_kept_dead_set_matches_revived(dmf, oracle, name, variant):
    """Batches keep the dead set of the last solve (the deficits a batch leaves
    inside it are covered there); every flow equals Dinic and the flow of a
    solver that revives every vertex at each batch, and every kept state is
    certified."""
    g, s, t, batches = make_config(name)
    if name == "grid256":  # more than the one configured batch
        batches = batches + dmf.gen_batches(g, 4, frac=0.01, p_inc=0.4, p_dec=0.4, p_ins=0.0, delta_hi=50, seed=7)
    off, adj, w, par = g.arrays()
    n = g.num_nodes()
    cur = w.copy()
    kept_batches = 0
    with dmf.Solver(g, s, t, variant=variant) as kept, dmf.Solver(g, s, t, variant=variant, revive_dead=True) as rev:
        assert kept.static_maxflow() == rev.static_maxflow()
        for b in batches:
            apply_host(g, cur, b)
            want = oracle.dinic(n, off, adj, cur, par, s, t)
            assert kept.apply_updates(*b) == want
            assert rev.apply_updates(*b) == want
            kept_batches += kept.stats()["dead_kept"]
            assert rev.stats()["dead_kept"] == 0
            certify(oracle, g, kept, s, t, want)
    if name.startswith("rmat"):  # on a grid the deficits sit far from any excess: revived
        assert kept_batches > 0


@pytest.mark.parametrize("tile", [4, 8, 16, 32])
def test_tile_sizes_agree(dmf, oracle, tile):
    g, s, t, batches = make_config("rmat12")
    off, adj, w, par = g.arrays()
    cur = w.copy()
    with dmf.Solver(g, s, t, tile=tile, kernel_cycles=2, relabel_interval=2) as sv:
        sv.static_maxflow()
        for b in batches[:3]:
            apply_host(g, cur, b)
            assert sv.apply_updates(*b) == oracle.dinic(g.num_nodes(), off, adj, cur, par, s, t)


@pytest.mark.parametrize("seed", range(8))
def test_random_graphs_many_batches(dmf, oracle, seed):
    rng = np.random.default_rng(100 + seed)
    nv = int(rng.integers(20, 400))
    k = int(rng.integers(nv, 8 * nv))
    u, v = rng.integers(0, nv, k), rng.integers(0, nv, k)
    wt = rng.integers(0, 60, k)
    g = dmf.Graph.from_edges(u, v, wt)
    off, adj, w, par = g.arrays()
    n = g.num_nodes()
    s, t = 0, n - 1
    tail = np.repeat(np.arange(n), np.diff(off))
    variant = VARIANTS[seed % 3]
    cur = w.copy()
    with dmf.Solver(g, s, t, variant=variant, relabel_interval=1 + seed % 4) as sv:
        assert sv.static_maxflow() == oracle.dinic(n, off, adj, cur, par, s, t)
        for _ in range(6):
            idx = rng.choice(g.num_edges(), size=min(g.num_edges(), int(rng.integers(1, 40))), replace=False)
            nw = rng.integers(0, 80, len(idx))
            nw[rng.random(len(idx)) < 0.3] = 0
            b = (tail[idx], adj[idx], nw)
            apply_host(g, cur, b)
            want = oracle.dinic(n, off, adj, cur, par, s, t)
            assert sv.apply_updates(*b) == want
            certify(oracle, g, sv, s, t, want)


def test_cut_matches_flow(dmf, oracle):
    g, s, t, batches = make_config("rmat12")
    off, adj, w, par = g.arrays()
    tail = np.repeat(np.arange(g.num_nodes()), np.diff(off))
    with dmf.Solver(g, s, t) as sv:
        f = sv.static_maxflow()
        f = sv.apply_updates(*batches[0])
        side = sv.cut()
        cap, res, ex, _ = sv.state()
        assert side[s] == 0 and side[t] == 1
        crossing = (side[tail] == 0) & (side[adj] == 1)
        assert int(cap[crossing].astype(np.int64).sum()) == f
        assert (res[crossing] == 0).all()


def test_edge_cases(dmf, oracle, golden_dir):
    g = dmf.Graph.load(os.path.join(golden_dir, "johnson8-2-4.bin"))
    off, adj, w, par = g.arrays()
    n = g.num_nodes()
    tail = np.repeat(np.arange(n), np.diff(off))
    with dmf.Solver(g, 25, 2) as sv:
        with pytest.raises(dmf.DmfError) as ei:
            sv.apply_updates([1], [2], [3])
        assert ei.value.status == 10  # not solved yet
        assert sv.static_maxflow() == 540
        assert sv.apply_updates([], [], []) == 540          # empty batch
        assert sv.apply_updates([3, 3], [3, 3], [5, 9]) == 540  # self-loops ignored
        missing = next((a, b) for a in range(n) for b in range(n) if a != b and g.find_arc(a, b) < 0)
        e0 = int(np.flatnonzero(w > 0)[0])
        e1 = int(np.flatnonzero(w > 0)[1])
        cap0, res0, _, _ = sv.state()
        for bad, status in [(([missing[0]], [missing[1]], [5]), 3),
                            (([tail[e0], tail[e0]], [adj[e0], adj[e0]], [1, 2]), 4),
                            # a valid update beside a repeated arc: the batch is rejected whole
                            (([tail[e1], tail[e0], tail[e0], tail[e0]], [adj[e1], adj[e0], adj[e0], adj[e0]],
                              [7, 1, 2, 3]), 4),
                            (([n + 5], [0], [1]), 1),
                            (([tail[e0]], [adj[e0]], [-1]), 1),
                            (([tail[e0]], [adj[e0]], [2**30]), 1)]:
            with pytest.raises(dmf.DmfError) as ei:
                sv.apply_updates(*bad)
            assert ei.value.status == status
            assert sv.flow == 540  # rejected batches change nothing
            cap1, res1, _, _ = sv.state()
            np.testing.assert_array_equal(cap1, cap0)
            np.testing.assert_array_equal(res1, res0)
        assert sv.apply_updates([], [], []) == 540
        # delete every arc out of the source: flow 0
        src_arcs = np.arange(off[25], off[26])
        assert sv.apply_updates(np.full(len(src_arcs), 25), adj[src_arcs], np.zeros(len(src_arcs))) == 0
        certify(oracle, g, sv, 25, 2, 0)
        # restore them at the largest allowed capacity
        big = np.full(len(src_arcs), 2**30 - 1 - int(w[par[src_arcs]].max()))
        cur = w.copy()
        cur[src_arcs] = big
        want = oracle.dinic(n, off, adj, cur, par, 25, 2)
        assert sv.apply_updates(np.full(len(src_arcs), 25), adj[src_arcs], big) == want
        certify(oracle, g, sv, 25, 2, want)


def test_zero_graph_and_unreachable_sink(dmf, oracle):
    # two components: s in one, t in the other
    u = np.array([0, 1, 3, 4]); v = np.array([1, 2, 4, 5]); wt = np.array([5, 5, 5, 5])
    g = dmf.Graph.from_edges(u, v, wt)
    with dmf.Solver(g, 0, 5) as sv:
        assert sv.static_maxflow() == 0
        assert sv.apply_updates([1], [2], [0]) == 0
    # all capacities zero
    g0 = dmf.Graph.from_edges(u, v, np.zeros(4))
    with dmf.Solver(g0, 0, 2) as sv:
        assert sv.static_maxflow() == 0
        assert sv.apply_updates([0, 1], [1, 2], [3, 2]) == 2


def test_device_pointer_batches_match_host(dmf, oracle):
    torch = pytest.importorskip("torch")
    g, s, t, batches = make_config("rmat12")
    with dmf.Solver(g, s, t) as a, dmf.Solver(g, s, t) as b:
        assert a.static_maxflow() == b.static_maxflow()
        for bt in batches[:4]:
            d = [torch.as_tensor(x, dtype=torch.int32, device="cuda") for x in bt]
            torch.cuda.synchronize()
            fa = a.apply_updates(*bt)
            fb = b.apply_updates_device(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), len(bt[0]))
            assert fa == fb


def test_recorded_reference_flows_on_gpu(dmf, golden_dir):
    """Our flows equal the values the reference's CUDA binaries printed."""
    import json
    from make_golden import cumulative_files, sha256
    path = os.path.join(golden_dir, "reference_flows.json")
    if not os.path.exists(path):
        pytest.skip("reference_flows.json not recorded yet")
    rec = json.load(open(path))
    checked = 0
    for name, entry in rec.items():
        g, s, t, batches = make_config(name)
        assert (g.num_nodes(), g.num_edges()) == (entry["n"], entry["m"])
        files = batches if not entry["cumulative"] else cumulative_files(batches)
        for key, per_file in entry["runs"].items():
            variant = key.split("/")[0]
            for rf in per_file:
                if rf["rc"] != 0 or not rf["runs"]:
                    continue
                ref = {r["dynamic_flow"] for r in rf["runs"]} | {r["static_flow"] for r in rf["runs"]}
                assert len(ref) == 1, (name, key, rf)
                got = dmf.recalculate_max_flow(g, files[rf["file"] - 1], s, t, 0, variant)
                assert got == ref.pop(), (name, key, rf["file"])
                checked += 1
    assert checked > 0
