"""dmf_tool (input tooling, host only) against the reference's own tool outputs."""
import os
import subprocess

import numpy as np
import pytest

from oracle.build import reference_root

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOOL = os.path.join(ROOT, "dyn_maxflow_b200", "bin", "dmf_tool")
MTX = os.path.join(reference_root(), "data", "raw_dataset", "johnson8-2-4.mtx")

pytestmark = pytest.mark.skipif(not os.path.exists(TOOL), reason="dmf_tool not built")


def run(*args):
    return subprocess.run([TOOL, *map(str, args)], capture_output=True, text=True)


@pytest.mark.skipif(not os.path.exists(MTX), reason="reference dataset not present")
def test_weight_and_cb_reproduce_reference_tools(tmp_path, golden_dir):
    # tests/golden/johnson8-2-4.{txt,bin} were written by the reference's weight.cpp and create_bin.cpp
    assert run("weight", MTX, tmp_path / "w.txt").returncode == 0
    assert (tmp_path / "w.txt").read_bytes() == open(os.path.join(golden_dir, "johnson8-2-4.txt"), "rb").read()
    r = run("cb", tmp_path / "w.txt", tmp_path / "w.bin")
    assert r.returncode == 0 and "29 nodes, 420 edges" in r.stdout
    assert (tmp_path / "w.bin").read_bytes() == open(os.path.join(golden_dir, "johnson8-2-4.bin"), "rb").read()


def test_cb_from_golden_text(tmp_path, golden_dir):
    r = run("cb", os.path.join(golden_dir, "johnson8-2-4.txt"), tmp_path / "j.bin")
    assert r.returncode == 0
    assert (tmp_path / "j.bin").read_bytes() == open(os.path.join(golden_dir, "johnson8-2-4.bin"), "rb").read()


def test_cb_update_layout(tmp_path):
    (tmp_path / "u.txt").write_text("3\n1 2 5\n3 4 6\n5 6 7\n")
    assert run("cb_update", tmp_path / "u.txt", tmp_path / "u.bin").returncode == 0
    want = np.array([3, 1, 3, 5, 2, 4, 6, 5, 6, 7], np.int32).tobytes()  # k, src[], dst[], w[]
    assert (tmp_path / "u.bin").read_bytes() == want
    (tmp_path / "short.txt").write_text("4\n1 2 5\n")
    assert run("cb_update", tmp_path / "short.txt", tmp_path / "s.bin").returncode == 1


def test_generators_and_cumulative_batches(tmp_path, dmf):
    r = run("gen-grid", 16, 16, 0, tmp_path / "g.bin")
    assert r.returncode == 0 and "source:0 sink:255" in r.stdout
    g = dmf.Graph.load(str(tmp_path / "g.bin"))
    assert g.num_nodes() == 256
    assert run("gen-batches", tmp_path / "g.bin", 3, 0.05, 1, tmp_path / "g", "cumulative").returncode == 0
    files = [dmf.load_updates(str(tmp_path / f"g_p{i}.bin")) for i in (1, 2, 3)]
    sizes = [len(f[0]) for f in files]
    assert sizes[0] <= sizes[1] <= sizes[2]  # cumulative: later files hold earlier arcs
    batches = dmf.gen_batches(g, 3, frac=0.05, seed=1)
    net = {}
    for s, d, w in batches:
        net.update({(a, b): c for a, b, c in zip(s.tolist(), d.tolist(), w.tolist())})
    got = {(a, b): c for a, b, c in zip(*(x.tolist() for x in files[2]))}
    assert got == net
    r = run("gen-rmat", 10, 3, 20, tmp_path / "r.bin")
    assert r.returncode == 0 and dmf.Graph.load(str(tmp_path / "r.bin")).num_nodes() == 1024
