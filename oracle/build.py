"""Build recipe for the oracle (test infrastructure only).

* ``build_oracle()`` compiles oracle/oracle.c (the CPU restatement, Dinic and the
  certificate checker) into oracle/liboracle.so.
* ``build_ref()`` compiles the reference's own sources, read in place under the
  reference checkout (DMF_REFERENCE, else a `reference` directory beside the
  repository; nothing is built when neither exists), into
  oracle/_ref/: its input tools with g++ (input_create/weight.cpp, create_bin.cpp,
  create_update_bin.cpp) and its CUDA benches with nvcc, once with the flags of
  code/Makefile (no -arch) and once with -arch=sm_100a.  Nothing is copied from
  the reference; the outputs stay in oracle/_ref/ (git-ignored).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(HERE, "liboracle.so")


def reference_root() -> str:
    """The reference checkout: $DMF_REFERENCE, else `reference` beside the repository."""
    env = os.environ.get("DMF_REFERENCE")
    if env:
        return env
    return os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")


def _stale(out: str, srcs: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "oracle.c")
    hdr = os.path.join(HERE, "oracle.h")
    if force or _stale(ORACLE_SO, [src, hdr]):
        _run(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-Wall", "-o", ORACLE_SO, src])
    return ORACLE_SO


REF_TOOLS = {
    "weightg": "input_create/weight.cpp",
    "cb": "input_create/create_bin.cpp",
    "cb_update": "input_create/create_update_bin.cpp",
}
REF_BENCHES = [
    "dyn_data_bench", "dyn_topo_bench", "dyn_pp_bench",
    "dyn_data_bench_large", "dyn_topo_bench_large", "dyn_pp_bench_large",
]


def build_ref(force: bool = False, cuda: bool = True) -> bool:
    """Returns False (and builds nothing) when the reference checkout is absent."""
    root = reference_root()
    if not os.path.isdir(os.path.join(root, "code")):
        return False
    os.makedirs(REF_OUT, exist_ok=True)
    for name, rel in REF_TOOLS.items():
        src = os.path.join(root, rel)
        out = os.path.join(REF_OUT, name)
        if force or _stale(out, [src]):
            _run(["g++", "-O2", "-o", out, src])
    if not cuda:
        return True
    code = os.path.join(root, "code")
    deps = [os.path.join(code, f) for f in ("graph.hpp", "update.hpp", "dyn_data.h", "dyn_topo.h", "dyn_pp.h")]
    for b in REF_BENCHES:
        src = os.path.join(code, b + ".cu")
        out_default = os.path.join(REF_OUT, b)
        out_sm100 = os.path.join(REF_OUT, b + "_sm100a")
        if force or _stale(out_default, [src] + deps):
            _run(["nvcc", src, "-o", out_default])  # code/Makefile:9-25
        if force or _stale(out_sm100, [src] + deps):
            _run(["nvcc", "-arch=sm_100a", src, "-o", out_sm100])
    return True


if __name__ == "__main__":
    build_oracle(force="--force" in sys.argv)
    print("oracle:", ORACLE_SO)
    print("reference built:", build_ref(force="--force" in sys.argv, cuda="--no-cuda" not in sys.argv))
