"""Failure paths of the solver, driven without faulting or hanging the GPU.

* A bound on global relabels that runs out: max_iters = 1 on graphs that need
  more ends the call with DMF_ERR_NO_CONVERGENCE.
* A grid barrier whose wait runs out: DMF_FLAG_TEST_BARRIER_TIMEOUT makes one
  block of the persistent grid leave at once (it never arrives) and drops the
  wait limit to 20 ms; the other blocks give up, set the error flag and leave at
  their next barrier, and the call returns DMF_ERR_TIMEOUT.

After either, the same solver must refuse batches until it is solved again, and
a static solve without the bound or the hook must be exact (Dinic) and certified.
"""
import time

import pytest

from make_golden import make_config

pytestmark = pytest.mark.gpu

DMF_ERR_NO_CONVERGENCE = 6
DMF_ERR_TIMEOUT = 8
DMF_ERR_NOT_SOLVED = 10
FLAG_TEST_BARRIER_TIMEOUT = 16


def _exact(oracle, g, s, t):
    off, adj, w, par = g.arrays()
    return oracle.dinic(g.num_nodes(), off, adj, w, par, s, t)


def _certified(oracle, g, sv, s, t, want):
    off, adj, _, par = g.arrays()
    cap, res, _, _ = sv.state()
    rc, val, cut = oracle.certify(g.num_nodes(), off, adj, cap, par, res, s, t)
    assert rc == 0 and val == want == cut, (rc, val, cut, want)


@pytest.mark.parametrize("name", ["grid256", "rmat14"])
def test_iteration_bound_reports_no_convergence(dmf, oracle, name):
    g, s, t, batches = make_config(name)
    want = _exact(oracle, g, s, t)
    with dmf.Solver(g, s, t, max_iters=1) as sv:
        with pytest.raises(dmf.DmfError) as ei:
            sv.static_maxflow()
        assert ei.value.status == DMF_ERR_NO_CONVERGENCE
        # the failed solve left no usable state: batches are refused
        with pytest.raises(dmf.DmfError) as ei:
            sv.apply_updates(*batches[0])
        assert ei.value.status == DMF_ERR_NOT_SOLVED
        sv.set_opts(max_iters=0)
        assert sv.static_maxflow() == want
        _certified(oracle, g, sv, s, t, want)


@pytest.mark.parametrize("variant", ["data", "pp"])
def test_barrier_timeout_returns_instead_of_hanging(dmf, oracle, variant):
    g, s, t, batches = make_config("rmat14")
    want = _exact(oracle, g, s, t)
    with dmf.Solver(g, s, t, variant=variant, test_barrier_timeout=True) as sv:
        t0 = time.perf_counter()
        with pytest.raises(dmf.DmfError) as ei:
            sv.static_maxflow()
        assert ei.value.status == DMF_ERR_TIMEOUT
        assert time.perf_counter() - t0 < 5.0  # 20 ms limit, not the 4 s default
        with pytest.raises(dmf.DmfError) as ei:
            sv.apply_updates(*batches[0])
        assert ei.value.status == DMF_ERR_NOT_SOLVED
        sv.set_opts(variant=variant, flags=0)
        assert sv.static_maxflow() == want
        _certified(oracle, g, sv, s, t, want)
        # a batch after recovery is exact too, and the hook on a batch times out again
        off, adj, w, par = g.arrays()
        cur = w.copy()
        for a, b, c in zip(*batches[0]):
            if a != b:
                cur[g.find_arc(int(a), int(b))] = c
        want1 = oracle.dinic(g.num_nodes(), off, adj, cur, par, s, t)
        sv.set_opts(variant=variant, flags=FLAG_TEST_BARRIER_TIMEOUT)
        with pytest.raises(dmf.DmfError) as ei:
            sv.apply_updates(*batches[0])
        assert ei.value.status == DMF_ERR_TIMEOUT
        sv.set_opts(variant=variant, flags=0)
        assert sv.static_maxflow() == want
        assert sv.apply_updates(*batches[0]) == want1
        _certified(oracle, g, sv, s, t, want1)
