"""Batched instances (dmf_multi_*): many graphs in one device state and one
persistent launch per call; the CUDA-graph-captured batch loop; the autotuner."""
import numpy as np
import pytest

from make_golden import make_config

pytestmark = pytest.mark.gpu


def _instances(dmf):
    from dyn_maxflow_b200 import workloads
    return workloads.batched(count=6, steps=3, seed=5, median=400, lo=64, hi=2000)


def _dinic_after(dmf, oracle, g, s, t, batches):
    off, adj, w, par = g.arrays()
    cur = w.copy()
    out = []
    for b in batches:
        for a, c, x in zip(*b):
            cur[g.find_arc(int(a), int(c))] = x
        out.append(oracle.dinic(g.num_nodes(), off, adj, cur, par, s, t))
    return out, cur


def test_multi_static_and_batches_match_dinic(dmf, oracle):
    inst = _instances(dmf)
    graphs = [x[0] for x in inst]
    with dmf.MultiSolver(graphs, [x[1] for x in inst], [x[2] for x in inst]) as ms:
        stat = ms.static_maxflow_all()
        for i, (g, s, t, _) in enumerate(inst):
            off, adj, w, par = g.arrays()
            assert stat[i] == oracle.dinic(g.num_nodes(), off, adj, w, par, s, t)
        want = [_dinic_after(dmf, oracle, *x)[0] for x in inst]
        for b in range(3):
            I = np.concatenate([np.full(len(x[3][b][0]), i) for i, x in enumerate(inst)])
            S = np.concatenate([x[3][b][0] for x in inst])
            D = np.concatenate([x[3][b][1] for x in inst])
            W = np.concatenate([x[3][b][2] for x in inst])
            got = ms.apply_updates_all(I, S, D, W)
            assert got.tolist() == [want[i][b] for i in range(len(inst))]
        # per-instance certificate on the union state
        cap, res, _, _ = ms.state()
        base_arc = 0
        for i, (g, s, t, _) in enumerate(inst):
            off, adj, w, par = g.arrays()
            m = g.num_edges()
            rc, val, cut = oracle.certify(g.num_nodes(), off, adj, cap[base_arc:base_arc + m], par,
                                          res[base_arc:base_arc + m], s, t)
            assert rc == 0 and val == want[i][-1] == cut
            base_arc += m


@pytest.mark.parametrize("use_graph", [True, False])
def test_run_batches_loop(dmf, oracle, use_graph):
    torch = pytest.importorskip("torch")
    from dyn_maxflow_b200 import workloads
    inst = _instances(dmf)
    graphs = [x[0] for x in inst]
    want = np.array([_dinic_after(dmf, oracle, *x)[0] for x in inst]).T  # [steps, count]
    for stream in (None, torch.cuda.Stream()):
        with dmf.MultiSolver(graphs, [x[1] for x in inst], [x[2] for x in inst], stream=stream) as ms:
            ms.static_maxflow_all()
            ofs, S, D, W = workloads.union_steps(inst, ms.vertex_base)
            dS, dD, dW = (torch.as_tensor(a, device="cuda") for a in (S, D, W))
            torch.cuda.synchronize()
            flows, t_ms = ms.run_batches(ofs, dS.data_ptr(), dD.data_ptr(), dW.data_ptr(), use_graph=use_graph)
            assert flows.tolist() == want.tolist()
            assert t_ms > 0
            # the solver stays usable afterwards
            assert ms.recompute() == int(want[-1].sum())


def test_autotune_keeps_the_flow(dmf, oracle):
    g, s, t, batches = make_config("rmat12")
    off, adj, w, par = g.arrays()
    with dmf.Solver(g, s, t) as sv:
        f0 = sv.static_maxflow()
        chosen = sv.autotune(repeats=1)
        assert chosen["tile"] in (4, 8, 16, 32)
        assert sv.flow == f0
        cur = w.copy()
        for b in batches[:3]:
            for a, c, x in zip(*b):
                cur[g.find_arc(int(a), int(c))] = x
            assert sv.apply_updates(*b) == oracle.dinic(g.num_nodes(), off, adj, cur, par, s, t)


def test_every_autotune_configuration_is_exact(dmf, oracle):
    """Every launch configuration the autotuner can choose (tile width, per-thread
    degree bound, relabel interval, cycles), set on a live solver as the
    autotuner sets it: a recompute and three successive batches must equal
    Dinic.  The autotuner picks by timing, so this covers deterministically what
    its choices could be."""
    import itertools
    g, s, t, batches = make_config("rmat12")
    off, adj, w, par = g.arrays()
    n = g.num_nodes()
    want = [oracle.dinic(n, off, adj, w, par, s, t)]
    cur = w.copy()
    for b in batches[:3]:
        for a, c, x in zip(*b):
            if a != c:
                cur[g.find_arc(int(a), int(c))] = x
        want.append(oracle.dinic(n, off, adj, cur, par, s, t))
    for tile, sd, iv, cyc in itertools.product([4, 8, 16, 32], [-1, 4, 8, 16, 32], [2, 3, 6, 12], [1, 2, 4]):
        with dmf.Solver(g, s, t) as sv:
            sv.static_maxflow()
            sv.set_opts(variant=0, kernel_cycles=cyc, relabel_interval=iv, tile=tile, small_deg=sd)
            got = [sv.recompute()] + [sv.apply_updates(*b) for b in batches[:3]]
            assert got == want, dict(tile=tile, small_deg=sd, interval=iv, cycles=cyc)
