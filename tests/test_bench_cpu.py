"""CPU checks of the benchmark's bookkeeping: percentiles, the algorithmic byte
counts behind `roofline` and `roofline_bfs`, the lookup of recorded reference
binary runs, and the reference arm's JSON line end to end on a small R-MAT
graph (that arm runs on the host cores only, so it needs no GPU)."""
import importlib.util
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("dmf_bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_percentiles_interpolate(bench):
    assert bench.pct([4, 1, 3, 2], 0.5) == pytest.approx(2.5)
    assert bench.pct([1, 2, 3, 4], 0.99) == pytest.approx(3.97)
    assert bench.pct([7], 0.99) == 7
    assert bench.pct([], 0.5) is None


def test_throughput_of_the_timed_batches(bench):
    batches = [([0] * 5, [1] * 5, [2] * 5), ([0] * 10, [1] * 10, [2] * 10), ([0] * 30, [1] * 30, [2] * 30)]
    # the warm-up batch (5 updates) is not counted; 40 updates in 2 + 3 ms
    r = bench.throughput(batches, 1, [2.0, 3.0])
    assert r == {"batches_per_s": 400.0, "updates_per_s": 8000.0}


def test_algorithmic_bytes_by_hand(bench):
    st = {"dead_vertices": 90, "outer_iters": 2, "arcs_scanned": 1000, "vertices_visited": 50, "pushes": 20,
          "dead_deficits": 0}
    # 10 updates, 5 source arcs, 10 live and 90 dead vertices, 2 relabels
    want = 64 * 10 + 16 * 5 + (36 * 10 + 2 * 90) * 2 + 12 * 1000 + 16 * 50 + 24 * 20 + 8 * 10 + 90
    assert bench.algorithmic_bytes(st, 100, 10, 5) == want
    # deficits left inside the kept dead set add the O(n) check
    assert bench.algorithmic_bytes(dict(st, dead_deficits=3), 100, 10, 5) == want + 9 * 100
    # a counter above n (dead vertices of several solves) is clipped to n
    assert bench.algorithmic_bytes(dict(st, dead_vertices=500), 100, 10, 5) == (
        64 * 10 + 16 * 5 + (2 * 100) * 2 + 12 * 1000 + 16 * 50 + 24 * 20 + 100)


def test_bfs_roofline_by_hand(bench):
    stats = [{"outer_iters": 2, "bfs_arcs": 1000, "dead_vertices": 90},
             {"outer_iters": 2, "bfs_arcs": 1000, "dead_vertices": 90}]
    phases = {"bfs_init": {"us": 1.0}, "bfs_td": {"us": 2.0}, "bfs_bu": {"us": 0.5}, "bfs_finalize": {"us": 0.5},
              "push": {"us": 100.0}}
    r = bench.bfs_roofline(stats, phases, 100, 1000.0)
    nbytes = (16 * 10 + 2 * 90) * 2 + 12 * 1000
    assert r["bytes_per_batch"] == nbytes
    assert r["bfs_us_per_batch"] == pytest.approx(4.0)
    assert r["achieved"] == pytest.approx(round(nbytes / 4e-6 / 1e9, 1))
    assert r["frac"] == pytest.approx(round(nbytes / 4e-6 / 1e9 / 1000.0, 4))
    assert bench.bfs_roofline([], phases, 100, 1000.0) is None
    assert bench.bfs_roofline(stats, {"push": {"us": 3.0}}, 100, 1000.0) is None


def test_recorded_reference_runs_match_only_their_graph(bench):
    rec = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_flows.json")))
    r20 = rec["rmat20"]

    class G:
        def __init__(self, n, m):
            self.n, self.m = n, m

        def num_nodes(self):
            return self.n

        def num_edges(self):
            return self.m

    out = bench.recorded_reference_cuda(G(r20["n"], r20["m"]), r20["source"], r20["sink"], 20)
    assert out is not None and out["graph_sha256"] == r20["sha256"]
    runs = [v for k, v in out.items() if isinstance(v, dict)]
    assert runs and all(v["dyn_per_batch_ms"] and v["static_update_ms"] for v in runs)
    # another graph of the same scale (a different reserve) gets no recorded numbers
    assert bench.recorded_reference_cuda(G(r20["n"], r20["m"] + 2), r20["source"], r20["sink"], 20) is None
    assert bench.recorded_reference_cuda(G(r20["n"], r20["m"]), r20["source"], r20["sink"], 13) is None


def test_reference_arm_line(oracle, dmf):
    """`bench.py --impl reference` on R-MAT scale 10: one JSON line with the
    keys the driver reads, and flows equal to an independent Dinic solve of
    every successive batch."""
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--scale", "10", "--steps", "3",
           "--warmup", "1", "--ref-budget-s", "30"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "ms" and d["higher_is_better"] is False
    assert d["metric"] == "ms to exact maxflow per update batch (p50)"
    assert d["config"]["workload"] == "rmat10-1pct-mixed-successive"
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"] > 0
    assert d["e2e"] == {"value": d["value"], "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["steps"] == len(d["flows"]) >= 1
    # the same workload, solved batch by batch with Dinic
    narcs = 16 << 10
    nb = 1 + 3
    g, s, t = dmf.gen_rmat(10, narcs, 0.57, 0.19, 0.19, seed=0, cap_lo=1, cap_hi=1000,
                           reserve=int(0.1 * 0.01 * narcs * nb) + 16)
    batches = dmf.gen_batches(g, nb, frac=0.01, p_inc=0.4, p_dec=0.4, p_ins=0.1, delta_hi=500, ins_lo=1,
                              ins_hi=1000, seed=1)
    assert d["config"]["vertices"] == g.num_nodes() and d["config"]["csr_arcs"] == g.num_edges()
    off, adj, w, par = g.arrays()
    cur = w.copy()
    want = []
    for src, dst, cap in batches:
        for a, b, c in zip(src, dst, cap):
            if a != b:
                cur[g.find_arc(int(a), int(b))] = c
        want.append(oracle.dinic(g.num_nodes(), off, adj, cur, par, s, t))
    warm = d["warmup"]
    assert d["flows"] == want[warm:warm + len(d["flows"])]
