"""The C ABI library loads and exports every entry point include/dmf.h declares;
host-only calls behave without a GPU (no compute is issued here)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "dmf.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    names = re.findall(r"\b(dmf_[a-z0-9_]+)\s*\(", hdr)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("dmf_graph_load", "dmf_updates_load", "dmf_solver_create", "dmf_static_maxflow",
                 "dmf_apply_updates", "dmf_apply_updates_device", "dmf_recompute", "dmf_get_cut",
                 "dmf_solver_destroy", "dmf_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol(dmf):
    lib = ctypes.CDLL(dmf.lib_path)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", dmf.lib_path], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (dmf_[a-z0-9_]+)", out))
    assert set(declared_symbols()) <= exported


def test_status_strings_and_defaults(dmf):
    L = ctypes.CDLL(dmf.lib_path)
    L.dmf_status_string.restype = ctypes.c_char_p
    assert L.dmf_status_string(0) == b"ok"
    assert L.dmf_status_string(3) == b"unknown arc"
    o = dmf.Opts()
    dmf._L.dmf_opts_default(ctypes.byref(o))
    assert o.variant == 0 and o.device == -1


def test_host_failure_is_a_status(dmf):
    """No C++ exception leaves the C ABI: an R-MAT request for 2^62 arcs cannot
    be allocated and returns DMF_ERR_OOM instead of ending the process."""
    with pytest.raises(dmf.DmfError) as ei:
        dmf.gen_rmat(scale=10, narcs=1 << 62)
    assert ei.value.status == 5 and "allocation" in str(ei.value)
    L = ctypes.CDLL(dmf.lib_path)
    L.dmf_status_string.restype = ctypes.c_char_p
    assert L.dmf_status_string(11) == b"host runtime error"
    g, _, _ = dmf.gen_rmat(scale=6, seed=1)  # the library still works
    assert g.num_edges() > 0


def test_solver_requires_gpu_and_validates_args(dmf, golden_dir):
    g = dmf.Graph.load(os.path.join(golden_dir, "johnson8-2-4.bin"))
    with pytest.raises(dmf.DmfError) as ei:
        dmf.Solver(g, 25, 25)
    assert ei.value.status == 1
    with pytest.raises(dmf.DmfError):
        dmf.Solver(g, 25, 99)
    if dmf.device_count() == 0:
        with pytest.raises(dmf.DmfError) as ei:
            dmf.Solver(g, 25, 2)
        assert ei.value.status == 7  # DMF_ERR_CUDA: no CPU fallback


def test_cli_usage_without_args():
    exe = os.path.join(ROOT, "dyn_maxflow_b200", "bin", "dyn_data_bench")
    if not os.path.exists(exe):
        pytest.skip("CLI not built")
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 1 and "usage" in r.stderr


def test_cli_failure_names_the_cause(dmf, golden_dir):
    """A failing step prints the library's own message (the release of what the
    step held must not clear it) and exits 1; the reference's first stdout
    lines are already out."""
    exe = os.path.join(ROOT, "dyn_maxflow_b200", "bin", "dyn_pp_bench_large")
    if not os.path.exists(exe):
        pytest.skip("CLI not built")
    graph, prefix = os.path.join(golden_dir, "johnson8-2-4.bin"), os.path.join(golden_dir, "johnson")
    r = subprocess.run([exe, graph, prefix, "25", "25", "1"], capture_output=True, text=True)
    assert r.returncode == 1
    assert "solver create failed: [invalid argument] need n >= 2 and distinct s, t" in r.stderr
    assert r.stdout.startswith("source:25 sink:25\nProcessing file:")
    if dmf.device_count() == 0:  # without a GPU the solver itself cannot be created
        r = subprocess.run([exe, graph, prefix, "25", "2", "1"], capture_output=True, text=True)
        assert r.returncode == 1 and "solver create failed: [cuda error] no CUDA device is visible" in r.stderr
