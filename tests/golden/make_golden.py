"""Generates the golden fixtures under tests/golden/.

  python tests/golden/make_golden.py fixtures
      Builds the johnson8-2-4 fixture with the reference's own input tools
      (oracle/_ref/weightg + oracle/_ref/cb, compiled from input_create/weight.cpp
      and create_bin.cpp; needs the reference checkout) and ten seeded update
      files johnson_p{i}.bin (i% of the arcs, mixed increases/decreases/deletes,
      each applied to the original graph, as the reference benches apply every
      file).

  python tests/golden/make_golden.py reference [--configs a,b,...] [--timeout S]
      Runs the reference's CUDA benches (oracle/_ref/dyn_{data,topo,pp}_bench*,
      built from code/*.cu) on a GPU and records the flow values they print
      ("Dynamic flow:", and "PANIC NOT MATCHING" lines) and their timings in
      tests/golden/reference_flows.json.  Inputs: the johnson fixture and graphs
      made by this package's seeded generators (grid 256x256, R-MAT scales 12,
      14, 16 and 20) with successive batches written as cumulative update files
      (file k = net capacities of every arc touched in batches 1..k), so that the
      reference, which applies each file to the original graph, reports the flow
      after batch k.  The sha256 of every generated graph is recorded so a
      change in the generators is detected.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

REF_BIN = os.path.join(ROOT, "oracle", "_ref")
OUT_JSON = os.path.join(HERE, "reference_flows.json")


def sha256(path: str) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 20), b""):
            h.update(chunk)
    return h.hexdigest()


# ---------------------------------------------------------------------------
# configs (all seeded; shared with the tests)
# ---------------------------------------------------------------------------
def make_config(name: str):
    """-> (Graph, s, t, batches) for a named config."""
    import dyn_maxflow_b200 as D
    if name == "johnson":
        g = D.Graph.load(os.path.join(HERE, "johnson8-2-4.bin"))
        batches = [D.load_updates(os.path.join(HERE, f"johnson_p{i}.bin")) for i in range(1, 11)]
        return g, 25, 2, batches
    if name == "grid256":
        g, s, t = D.gen_grid(256, 256, seed=0, cap_lo=1, cap_hi=100, st_cap=1000)
        b = D.gen_batches(g, 1, frac=0.01, p_inc=0.5, p_dec=0.5, p_ins=0.0, delta_hi=50, seed=0)
        return g, s, t, b
    m = re.fullmatch(r"rmat(\d+)", name)
    if m:
        scale = int(m.group(1))
        narcs = 16 << scale
        # scale 24 is the benchmark's headline graph: its reserve is sized for
        # the benchmark's 3 + 10 batches, so that the graphs are the same
        nb = 13 if scale >= 24 else 10
        reserve = int(0.1 * 0.01 * narcs * nb) + 16
        g, s, t = D.gen_rmat(scale, narcs, 0.57, 0.19, 0.19, seed=0, cap_lo=1, cap_hi=1000, reserve=reserve)
        b = D.gen_batches(g, nb, frac=0.01, p_inc=0.4, p_dec=0.4, p_ins=0.1, delta_hi=500, ins_lo=1,
                          ins_hi=1000, seed=1)
        return g, s, t, b
    raise KeyError(name)


def cumulative_files(batches):
    """file k = net absolute capacities of all arcs touched in batches 1..k."""
    import numpy as np
    net = {}
    files = []
    for (s, d, w) in batches:
        for a, b, c in zip(s.tolist(), d.tolist(), w.tolist()):
            net[(a, b)] = c
        keys = list(net.keys())
        files.append((np.array([k[0] for k in keys], np.int32), np.array([k[1] for k in keys], np.int32),
                      np.array([net[k] for k in keys], np.int32)))
    return files


# ---------------------------------------------------------------------------
def cmd_fixtures() -> None:
    import numpy as np
    from oracle import build as OB
    import dyn_maxflow_b200 as D
    if not OB.build_ref(cuda=False):
        raise SystemExit("reference checkout not found (set DMF_REFERENCE)")
    mtx = os.path.join(OB.reference_root(), "data", "raw_dataset", "johnson8-2-4.mtx")
    txt = os.path.join(HERE, "johnson8-2-4.txt")
    binp = os.path.join(HERE, "johnson8-2-4.bin")
    subprocess.run([os.path.join(REF_BIN, "weightg"), mtx, txt], check=True, capture_output=True)
    subprocess.run([os.path.join(REF_BIN, "cb"), txt, binp], check=True, capture_output=True)
    g = D.Graph.load(binp)
    for i in range(1, 11):
        (b,) = D.gen_batches(g, 1, frac=i / 100.0, p_inc=0.4, p_dec=0.4, p_ins=0.0, delta_hi=50, seed=100 + i)
        D.save_updates(os.path.join(HERE, f"johnson_p{i}.bin"), *b)
    print("fixtures written; johnson n,m =", g.num_nodes(), g.num_edges(), "sha256", sha256(binp))
    _ = np


_FLOW = re.compile(r"Dynamic flow:(-?\d+)")
_PANIC = re.compile(r"PANIC NOT MATCHING dynflow:(-?\d+) statflow:(-?\d+)")
_DYN = re.compile(r"per batch time:([0-9.]+)")
_STAT = re.compile(r"(?:STATIC UPDATE|static  UPDATE) GPU Time: ([0-9.]+)")
_KC = re.compile(r"=======kernel cycles (-?\d+) =======")


def parse_bench(out: str):
    """Per kernel_cycles block: dynamic flow, static flow (equal unless PANIC), times."""
    runs = []
    parts = _KC.split(out)
    for i in range(1, len(parts), 2):
        kc, body = int(parts[i]), parts[i + 1]
        fl = _FLOW.search(body)
        pn = _PANIC.search(body)
        dy = _DYN.search(body)
        st = _STAT.search(body)
        dyn = int(fl.group(1)) if fl else None
        stat = int(pn.group(2)) if pn else dyn
        runs.append({"kernel_cycles": kc, "dynamic_flow": dyn, "static_flow": stat, "panic": bool(pn),
                     "dyn_ms": float(dy.group(1)) if dy else None, "recompute_ms": float(st.group(1)) if st else None})
    return runs


def cmd_reference(configs, timeout: float, variants, builds, files_sel=None) -> None:
    import dyn_maxflow_b200 as D
    results = {}
    if os.path.exists(OUT_JSON):
        with open(OUT_JSON) as f:
            results = json.load(f)
    tmp = tempfile.mkdtemp(prefix="dmf_ref_")
    for name in configs:
        g, s, t, batches = make_config(name)
        gpath = os.path.join(tmp, f"{name}.bin")
        g.save(gpath)
        files = batches if name in ("johnson",) else cumulative_files(batches)
        for i, (a, b, c) in enumerate(files, 1):
            D.save_updates(os.path.join(tmp, f"{name}_p{i}.bin"), a, b, c)
        entry = {"sha256": sha256(gpath), "n": g.num_nodes(), "m": g.num_edges(), "source": s, "sink": t,
                 "files": len(files), "cumulative": name != "johnson", "runs": {}}
        for variant in variants:
            for build in builds:
                exe = os.path.join(REF_BIN, f"dyn_{variant}_bench_large" + ("_sm100a" if build == "sm100a" else ""))
                per_file = []
                for i in (files_sel or range(1, len(files) + 1)):
                    t0 = time.time()
                    try:
                        r = subprocess.run([exe, gpath, os.path.join(tmp, name), str(s), str(t), str(i)],
                                           capture_output=True, text=True, timeout=timeout)
                        out, rc = r.stdout, r.returncode
                    except subprocess.TimeoutExpired as e:
                        out, rc = (e.stdout or b"").decode() if isinstance(e.stdout, bytes) else (e.stdout or ""), "timeout"
                    per_file.append({"file": i, "rc": rc, "wall_s": round(time.time() - t0, 3),
                                     "runs": parse_bench(out)})
                    print(name, variant, build, i, rc, per_file[-1]["runs"], flush=True)
                    if rc == "timeout":
                        break
                entry["runs"][f"{variant}/{build}"] = per_file
        old = results.get(name)
        if old and old.get("sha256") == entry["sha256"]:
            old["runs"].update(entry["runs"])
            entry = old
        results[name] = entry
        with open(OUT_JSON, "w") as f:
            json.dump(results, f, indent=1, sort_keys=True)
    print("wrote", OUT_JSON)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["fixtures", "reference"])
    ap.add_argument("--configs", default="johnson,grid256,rmat12,rmat14,rmat16")
    ap.add_argument("--variants", default="data,topo,pp")
    ap.add_argument("--builds", default="sm100a")
    ap.add_argument("--timeout", type=float, default=300)
    ap.add_argument("--files", default="", help="comma-separated file numbers (default: all)")
    a = ap.parse_args()
    if a.what == "fixtures":
        cmd_fixtures()
    else:
        sel = [int(x) for x in a.files.split(",")] if a.files else None
        cmd_reference(a.configs.split(","), a.timeout, a.variants.split(","), a.builds.split(","), sel)
