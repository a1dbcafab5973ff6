"""The drop-in command-line entry points on the GPU: same argv and stdout lines
as the reference benches, flows equal to the oracle's."""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "dyn_maxflow_b200", "bin")


def expected_flows(dmf, oracle, golden_dir):
    g = dmf.Graph.load(os.path.join(golden_dir, "johnson8-2-4.bin"))
    off, adj, w, par = g.arrays()
    out = []
    for i in range(1, 11):
        cur = w.copy()
        for a, b, c in zip(*dmf.load_updates(os.path.join(golden_dir, f"johnson_p{i}.bin"))):
            cur[g.find_arc(int(a), int(b))] = c
        out.append(oracle.dinic(g.num_nodes(), off, adj, cur, par, 25, 2))
    return out


@pytest.mark.parametrize("variant", ["data", "topo", "pp"])
def test_cli_all_files(dmf, oracle, golden_dir, variant):
    want = expected_flows(dmf, oracle, golden_dir)
    exe = os.path.join(BIN, f"dyn_{variant}_bench")
    r = subprocess.run([exe, os.path.join(golden_dir, "johnson8-2-4.bin"), os.path.join(golden_dir, "johnson"),
                        "25", "2"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = r.stdout
    assert out.startswith("source:25 sink:2\n")
    assert "PANIC" not in out
    files = re.findall(r"Processing file: .*johnson_p(\d+)\.bin", out)
    assert files == [str(i) for i in range(1, 11)]
    flows = [int(x) for x in re.findall(r"Dynamic flow:(-?\d+)", out)]
    # three kernel_cycles values per file (avg_deg-1, avg_deg, avg_deg+1)
    assert flows == [f for f in want for _ in range(3)]
    assert len(re.findall(r"=======kernel cycles (\d+) =======", out)) == 30
    assert len(re.findall(r"DYN TIME:[0-9.]+ms true_cnt=1 cnt=1 per batch time:[0-9.]+", out)) == 30
    upd = re.findall(r"updates size:(\d+)", out)
    sizes = [len(dmf.load_updates(os.path.join(golden_dir, f"johnson_p{i}.bin"))[0]) for i in range(1, 11)]
    assert [int(x) for x in upd] == [2 * k for k in sizes]
    if variant == "pp":
        assert "static  UPDATE GPU Time:" in out and "static main push cnt:" in out
    else:
        assert "STATIC UPDATE GPU Time:" in out and "static GPU Time:" in out
    if variant == "topo":
        assert "V:29\nE:420\n" in out


def test_cli_large_single_file_and_json(dmf, oracle, golden_dir):
    want = expected_flows(dmf, oracle, golden_dir)
    exe = os.path.join(BIN, "dyn_data_bench_large")
    env = dict(os.environ, DMF_CLI_JSON="1")
    r = subprocess.run([exe, os.path.join(golden_dir, "johnson8-2-4.bin"), os.path.join(golden_dir, "johnson"),
                        "25", "2", "7"], capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stderr
    assert re.findall(r"Processing file: .*johnson_p(\d+)\.bin", r.stdout) == ["7"]
    import json
    recs = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(recs) == 3 and all(x["dynamic_flow"] == x["recompute_flow"] == want[6] for x in recs)
    assert all(x["static_flow"] == 540 for x in recs)


def test_cli_bad_graph(tmp_path):
    (tmp_path / "bad.bin").write_bytes(b"\x01\x02")
    r = subprocess.run([os.path.join(BIN, "dyn_data_bench"), str(tmp_path / "bad.bin"), str(tmp_path / "x"), "0", "1"],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "bad file" in r.stderr
