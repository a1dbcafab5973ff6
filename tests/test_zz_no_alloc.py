"""dmf_static_maxflow_noalloc: the static solve for callers that cannot allocate
device memory while they run (a fixed memory pool or arena, or a host that
forbids cudaMalloc after start-up).  It keeps its scratch in a static device
array inside the library; the caller supplies the graph and the residual output.

Checked through the C ABI against the allocating entry point
(dmf_static_maxflow) on two calls in a row: equal flow values (exact, integer)
and residuals that pass the oracle's max-flow certificate.  This file is
collected last so that a failure here does not hide the other tests' results.
"""
import ctypes as C
import os

import numpy as np
import pytest

from make_golden import make_config

pytestmark = pytest.mark.gpu


def _device_csr(torch, g):
    off, adj, w, par = g.arrays()
    to = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32), device="cuda")
    return off, adj, w, par, to(off), to(adj), to(w), to(par)


def _noalloc(dmf, torch, g, s, t):
    off, adj, w, par, d_off, d_adj, d_cap, d_par = _device_csr(torch, g)
    d_res = torch.full((max(g.num_edges(), 1),), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    flow = C.c_int64(-1)
    st = dmf._L.dmf_static_maxflow_noalloc(g.num_nodes(), g.num_edges(), C.c_void_p(d_off.data_ptr()),
                                           C.c_void_p(d_adj.data_ptr()), C.c_void_p(d_cap.data_ptr()),
                                           C.c_void_p(d_par.data_ptr()), s, t, C.c_void_p(d_res.data_ptr()),
                                           C.byref(flow), None)
    assert st == 0, dmf._L.dmf_last_error().decode()
    return flow.value, d_res[: g.num_edges()].cpu().numpy()


@pytest.mark.parametrize("name", ["johnson", "rmat14", "grid256"])
def test_noalloc_matches_allocating_entry_point(dmf, oracle, name):
    torch = pytest.importorskip("torch")
    g, s, t, _ = make_config(name)
    off, adj, w, par = g.arrays()
    with dmf.Solver(g, s, t) as sv:
        want = sv.static_maxflow()
    for call in range(2):  # two calls in a row share (and reuse) the static scratch
        got, res = _noalloc(dmf, torch, g, s, t)
        assert got == want, (name, call)
        rc, val, cut = oracle.certify(g.num_nodes(), off, adj, w, par, res, s, t)
        assert rc == 0 and val == want == cut, (name, call, rc)


def test_noalloc_alternating_graphs_and_limits(dmf, oracle):
    torch = pytest.importorskip("torch")
    g1, s1, t1, _ = make_config("rmat12")
    g2, s2, t2, _ = make_config("johnson")
    with dmf.Solver(g1, s1, t1) as a, dmf.Solver(g2, s2, t2) as b:
        w1, w2 = a.static_maxflow(), b.static_maxflow()
    # a larger graph then a smaller one: stale contents of the scratch must not leak
    assert _noalloc(dmf, torch, g1, s1, t1)[0] == w1
    assert _noalloc(dmf, torch, g2, s2, t2)[0] == w2
    assert _noalloc(dmf, torch, g1, s1, t1)[0] == w1
    # beyond the static capacity: rejected before any device work
    flow = C.c_int64(-1)
    st = dmf._L.dmf_static_maxflow_noalloc((1 << 18) + 1, 0, C.c_void_p(8), None, None, None, 0, 1, None,
                                           C.byref(flow), None)
    assert st == 1 and b"exceeds" in dmf._L.dmf_last_error()
    assert flow.value == -1
