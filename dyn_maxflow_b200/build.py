"""Build of the native parts of dyn_maxflow_b200 (in-tree).

* ``libdmf.so``  -- the C-ABI library: csrc/dmf_solver.cu (the solver's host
  side), csrc/dmf_kernel_t*.cu (the sm_100a solve kernel, csrc/dmf_kernel.cuh,
  one file per tile width), csrc/dmf_sched.cu (schedule picker),
  csrc/dmf_host.cpp (formats, builder, generators) and csrc/dmf_server.cpp
  (serving loop), compiled by nvcc for ``-gencode arch=compute_100a,code=sm_100a``
  only.
* ``bin/dyn_data_bench``, ``bin/dyn_topo_bench``, ``bin/dyn_pp_bench`` and the
  ``*_large`` forms -- the drop-in command-line entry points (csrc/dmf_cli.cpp),
  linked against libdmf.so.
* ``bin/dmf_tool`` -- input tooling (csrc/dmf_tool.cpp): weighting, text -> .bin
  graph and update conversion, seeded generators.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libdmf.so")
BIN = os.path.join(PKG, "bin")
CLI_NAMES = ["dyn_data_bench", "dyn_topo_bench", "dyn_pp_bench",
             "dyn_data_bench_large", "dyn_topo_bench_large", "dyn_pp_bench_large"]

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC,-fopenmp,-O3",
    "--expt-relaxed-constexpr",
]


def _sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))] + [os.path.join(INCLUDE, "dmf.h")]


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], verbose: bool = False) -> str:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


LIB_SOURCES = ["dmf_solver.cu", "dmf_kernel_t4.cu", "dmf_kernel_t8.cu", "dmf_kernel_t16.cu", "dmf_kernel_t32.cu",
               "dmf_sched.cu", "dmf_host.cpp", "dmf_server.cpp"]
OBJ_DIR = os.path.join(PKG, "_build")


def build_lib(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compiles every source of libdmf.so to an object file (in parallel: the
    solve kernel's instantiations sit in one file per tile width) and links."""
    from concurrent.futures import ThreadPoolExecutor
    deps = _sources()
    if not (force or ptxas_info or _stale(LIB, deps)):
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    jobs = []
    for src in LIB_SOURCES:
        obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
        cmd = ["nvcc", *NVCC_FLAGS, "-I", INCLUDE, "-I", CSRC, "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_info and src.endswith(".cu"):
            cmd[1:1] = ["-Xptxas", "-v"]
        jobs.append((cmd, obj))
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        outs = list(ex.map(lambda j: _run(j[0], verbose), jobs))
    _run(["nvcc", *NVCC_FLAGS, "-shared", *[o for _, o in jobs], "-o", LIB + ".tmp", "-lgomp"], verbose)
    os.replace(LIB + ".tmp", LIB)
    if ptxas_info:
        print("\n".join(outs))
    return LIB


def build_cli(force: bool = False, verbose: bool = False) -> list[str]:
    os.makedirs(BIN, exist_ok=True)
    src = os.path.join(CSRC, "dmf_cli.cpp")
    outs = []
    for name in CLI_NAMES:
        out = os.path.join(BIN, name)
        variant = name.split("_")[1]
        large = "1" if name.endswith("_large") else "0"
        if force or _stale(out, [src, LIB, os.path.join(INCLUDE, "dmf.h")]):
            _run(["g++", "-std=c++17", "-O2", f"-DDMF_CLI_VARIANT=\"{variant}\"", f"-DDMF_CLI_LARGE={large}",
                  "-I", INCLUDE, src, "-o", out, "-L", PKG, "-ldmf", "-Wl,-rpath,$ORIGIN/.."], verbose)
        outs.append(out)
    return outs


def build_tool(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BIN, exist_ok=True)
    src = os.path.join(CSRC, "dmf_tool.cpp")
    out = os.path.join(BIN, "dmf_tool")
    if force or _stale(out, [src, LIB, os.path.join(INCLUDE, "dmf.h")]):
        _run(["g++", "-std=c++17", "-O2", "-I", INCLUDE, src, "-o", out, "-L", PKG, "-ldmf",
              "-Wl,-rpath,$ORIGIN/.."], verbose)
    return out


def build(force: bool = False, verbose: bool = False) -> None:
    build_lib(force, verbose)
    build_cli(force, verbose)
    build_tool(force, verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    if "--ptxas" in sys.argv:
        build_lib(ptxas_info=True)
