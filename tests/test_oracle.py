"""The CPU oracle, pinned against the reference's known answer, its own builder
output, and (when recorded) the flows printed by the reference's CUDA binaries."""
import json
import os

import numpy as np
import pytest

from make_golden import make_config


def _johnson(oracle, golden_dir):
    return oracle.read_graph(os.path.join(golden_dir, "johnson8-2-4.bin"))


def test_johnson_known_answer(oracle, golden_dir):
    # johnson8-2-4 -> weight.cpp (seed 42) -> create_bin, s=25, t=2 (input_create/README.md:60-63)
    n, m, off, adj, w, par = _johnson(oracle, golden_dir)
    assert (n, m) == (29, 420)
    assert oracle.dinic(n, off, adj, w, par, 25, 2) == 540
    for variant in ("data", "topo", "pp"):
        for kc in (m // n - 1, m // n, m // n + 1):
            assert oracle.ref_run(variant, n, off, adj, w, par, 25, 2, kc, [], [], []) == (540, 540, 540)


def test_builder_restatement_matches_reference_tool(oracle, golden_dir):
    # tests/golden/johnson8-2-4.bin was written by the reference's create_bin.cpp
    t = np.loadtxt(os.path.join(golden_dir, "johnson8-2-4.txt"), dtype=np.int64)
    got = oracle.build_csr(t[:, 0], t[:, 1], t[:, 2])
    want = _johnson(oracle, golden_dir)
    assert got[:2] == want[:2]
    for a, b in zip(got[2:], want[2:]):
        np.testing.assert_array_equal(a, b)


def _random_graph(oracle, rng, n, k, cap_hi=20, dup=True):
    u = rng.integers(0, n, k)
    v = rng.integers(0, n, k)
    if dup:  # duplicates and self-loops on purpose: merged / dropped by create_bin
        u[: k // 10] = u[k // 10: 2 * (k // 10)]
        v[: k // 10] = v[k // 10: 2 * (k // 10)]
    w = rng.integers(0, cap_hi + 1, k)
    return oracle.build_csr(u, v, w)


@pytest.mark.parametrize("seed", range(6))
def test_reference_restatement_equals_dinic(oracle, seed):
    rng = np.random.default_rng(seed)
    n, m, off, adj, w, par = _random_graph(oracle, rng, 60, 400)
    s, t = 0, n - 1
    want = oracle.dinic(n, off, adj, w, par, s, t)
    # one batch of capacity changes on existing arcs
    idx = rng.choice(m, size=40, replace=False)
    tail = np.repeat(np.arange(n), np.diff(off))
    src, dst = tail[idx], adj[idx]
    neww = rng.integers(0, 25, len(idx))
    w2 = w.copy()
    w2[idx] = neww
    want2 = oracle.dinic(n, off, adj, w2, par, s, t)
    for variant in ("data", "topo", "pp"):
        for nth in (1, 4):
            before, dyn, stat = oracle.ref_run(variant, n, off, adj, w, par, s, t, 3, src, dst, neww, nthreads=nth)
            assert before == want
            assert dyn == want2 and stat == want2, (variant, nth)


def test_certificate_accepts_max_and_rejects_non_max(oracle):
    rng = np.random.default_rng(11)
    n, m, off, adj, w, par = _random_graph(oracle, rng, 50, 300)
    val, flow = oracle.dinic(n, off, adj, w, par, 0, n - 1, want_flow=True)
    res = (w - flow).astype(np.int32)
    rc, v, cut = oracle.certify(n, off, adj, w, par, res, 0, n - 1)
    assert rc == 0 and v == val == cut
    # zero flow is a valid pseudoflow but not maximum (when val > 0)
    if val > 0:
        rc, v, _ = oracle.certify(n, off, adj, w, par, w.copy(), 0, n - 1)
        assert rc == 3 and v == 0
    # residual below zero is rejected
    bad = res.copy()
    bad[0] = -1
    assert oracle.certify(n, off, adj, w, par, bad, 0, n - 1)[0] in (1, 2)


def test_successive_batches_match_dinic(oracle):
    g, s, t, batches = make_config("rmat12")
    off, adj, w, par = g.arrays()
    n = g.num_nodes()
    static, flows, _ = oracle.ref_run_successive("data", n, off, adj, w, par, s, t, 8, batches[:4], nthreads=4)
    assert static == oracle.dinic(n, off, adj, w, par, s, t)
    cur = w.copy()
    for i, (a, b, c) in enumerate(batches[:4]):
        for x, y, z in zip(a, b, c):
            cur[g.find_arc(int(x), int(y))] = z
        assert flows[i] == oracle.dinic(n, off, adj, cur, par, s, t)


def test_pp_successive_matches_dinic(oracle):
    g, s, t, batches = make_config("rmat12")
    off, adj, w, par = g.arrays()
    n = g.num_nodes()
    _, flows, _ = oracle.ref_run_successive("pp", n, off, adj, w, par, s, t, 8, batches[:3], nthreads=4)
    cur = w.copy()
    for i, (a, b, c) in enumerate(batches[:3]):
        for x, y, z in zip(a, b, c):
            cur[g.find_arc(int(x), int(y))] = z
        assert flows[i] == oracle.dinic(n, off, adj, cur, par, s, t)


def test_recorded_reference_binary_flows_match_oracle(oracle, golden_dir):
    """Flows printed by the reference's own CUDA benches (run on a B200 by
    make_golden.py reference) equal the oracle's exact flows on the same files."""
    path = os.path.join(golden_dir, "reference_flows.json")
    if not os.path.exists(path):
        pytest.skip("reference_flows.json not recorded yet")
    with open(path) as f:
        rec = json.load(f)
    import dyn_maxflow_b200 as D
    from make_golden import cumulative_files, sha256
    checked = 0
    for name, entry in rec.items():
        if entry["m"] > 2_000_000:
            continue  # large configs are checked on the GPU
        g, s, t, batches = make_config(name)
        off, adj, w, par = g.arrays()
        n = g.num_nodes()
        files = batches if not entry["cumulative"] else cumulative_files(batches)
        for key, per_file in entry["runs"].items():
            for rec_file in per_file:
                if rec_file["rc"] != 0:
                    continue
                a, b, c = files[rec_file["file"] - 1]
                cur = w.copy()
                for x, y, z in zip(a, b, c):
                    if x != y:
                        cur[g.find_arc(int(x), int(y))] = z
                want = oracle.dinic(n, off, adj, cur, par, s, t)
                for run in rec_file["runs"]:
                    assert run["dynamic_flow"] == want, (name, key, rec_file["file"], run)
                    assert run["static_flow"] == want, (name, key, rec_file["file"], run)
                    checked += 1
        _ = D, sha256
    assert checked > 0
