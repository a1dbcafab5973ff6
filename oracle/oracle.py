"""ctypes wrapper over oracle/liboracle.so.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the
checker, and by bench.py's CPU-baseline leg / reference arm.  The product path
never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

_lib = None

I32P = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
I64P = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
F64P = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
ORC_DATA, ORC_TOPO, ORC_PP = 0, 1, 2
VARIANTS = {"data": ORC_DATA, "topo": ORC_TOPO, "pp": ORC_PP}


def lib():
    global _lib
    if _lib is None:
        path = _build.ORACLE_SO
        if not os.path.exists(path):
            _build.build_oracle()
        L = C.CDLL(path)
        L.orc_dinic.restype = C.c_int64
        L.orc_dinic.argtypes = [C.c_int32, C.c_int32, I32P, I32P, I32P, I32P, C.c_int32, C.c_int32, C.c_void_p]
        L.orc_certify.restype = C.c_int
        L.orc_certify.argtypes = [C.c_int32, C.c_int32, I32P, I32P, I32P, I32P, I32P, C.c_int32, C.c_int32,
                                  C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.orc_ref_run.restype = C.c_int
        L.orc_ref_run.argtypes = [C.c_int, C.c_int32, C.c_int32, I32P, I32P, I32P, I32P, C.c_int32, C.c_int32,
                                  C.c_int32, C.c_int32, I32P, I32P, I32P, C.c_int, C.c_int64,
                                  C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.orc_ref_run_successive.restype = C.c_int
        L.orc_ref_run_successive.argtypes = [C.c_int, C.c_int32, C.c_int32, I32P, I32P, I32P, I32P, C.c_int32,
                                             C.c_int32, C.c_int32, C.c_int32, I64P, I32P, I32P, I32P, C.c_int,
                                             C.c_int64, C.POINTER(C.c_int64), I64P, F64P, C.c_double,
                                             C.POINTER(C.c_int32)]
        L.orc_build_csr.restype = C.c_int
        L.orc_build_csr.argtypes = [C.c_int64, I32P, I32P, I32P, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                    C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                    C.POINTER(C.c_void_p)]
        L.orc_graph_read.restype = C.c_int
        L.orc_graph_read.argtypes = [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)] + [C.POINTER(C.c_void_p)] * 4
        L.orc_updates_read.restype = C.c_int
        L.orc_updates_read.argtypes = [C.c_char_p, C.POINTER(C.c_int32)] + [C.POINTER(C.c_void_p)] * 3
        L.orc_free.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def _take(ptr: C.c_void_p, count: int) -> np.ndarray:
    arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int32)), shape=(max(count, 1),))[:count].copy()
    lib().orc_free(ptr)
    return arr


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def read_graph(path: str):
    """code/graph.hpp:202-223 -> (n, m, off, adj, w, par)."""
    n, m = C.c_int32(), C.c_int32()
    ps = [C.c_void_p() for _ in range(4)]
    if lib().orc_graph_read(path.encode(), C.byref(n), C.byref(m), *[C.byref(p) for p in ps]):
        raise IOError(f"cannot read graph {path}")
    off = _take(ps[0], n.value + 1)
    return n.value, m.value, off, _take(ps[1], m.value), _take(ps[2], m.value), _take(ps[3], m.value)


def read_updates(path: str):
    """code/update.hpp:52-88 -> (src, dst, w)."""
    k = C.c_int32()
    ps = [C.c_void_p() for _ in range(3)]
    if lib().orc_updates_read(path.encode(), C.byref(k), *[C.byref(p) for p in ps]):
        raise IOError(f"cannot read updates {path}")
    return tuple(_take(p, k.value) for p in ps)


def build_csr(u, v, w):
    """input_create/create_bin.cpp:67-124 restated -> (n, m, off, adj, cap, par)."""
    u, v, w = _i32(u), _i32(v), _i32(w)
    n, m = C.c_int32(), C.c_int32()
    ps = [C.c_void_p() for _ in range(4)]
    if lib().orc_build_csr(len(u), u, v, w, C.byref(n), C.byref(m), *[C.byref(p) for p in ps]):
        raise ValueError("bad edge list")
    return n.value, m.value, _take(ps[0], n.value + 1), _take(ps[1], m.value), _take(ps[2], m.value), _take(ps[3], m.value)


def dinic(n, off, adj, cap, par, s, t, want_flow=False):
    off, adj, cap, par = _i32(off), _i32(adj), _i32(cap), _i32(par)
    m = len(adj)
    fl = np.zeros(max(m, 1), dtype=np.int32) if want_flow else None
    val = lib().orc_dinic(n, m, off, adj, cap, par, s, t, fl.ctypes.data if want_flow else None)
    return (val, fl[:m]) if want_flow else val


def certify(n, off, adj, cap, par, res, s, t):
    """Returns (code, value, cut_capacity); code 0 means the pseudoflow is maximum."""
    off, adj, cap, par, res = _i32(off), _i32(adj), _i32(cap), _i32(par), _i32(res)
    val, cut = C.c_int64(), C.c_int64()
    rc = lib().orc_certify(n, len(adj), off, adj, cap, par, res, s, t, C.byref(val), C.byref(cut))
    return rc, val.value, cut.value


def ref_run(variant, n, off, adj, w, par, s, t, kernel_cycles, src, dst, wt, nthreads=1, max_iters=10_000_000):
    """One update file through the reference's algorithm: (static_before, dynflow, statflow)."""
    off, adj, w, par = _i32(off), _i32(adj), _i32(w), _i32(par)
    src, dst, wt = _i32(src), _i32(dst), _i32(wt)
    if len(src) == 0:
        src = dst = wt = np.zeros(1, np.int32)
        k = 0
    else:
        k = len(src)
    a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
    rc = lib().orc_ref_run(VARIANTS.get(variant, variant), n, len(adj), off, adj, w, par, s, t, kernel_cycles, k,
                           src, dst, wt, nthreads, max_iters, C.byref(a), C.byref(b), C.byref(c))
    if rc:
        raise RuntimeError(f"oracle ref_run failed rc={rc}")
    return a.value, b.value, c.value


def ref_run_successive(variant, n, off, adj, w, par, s, t, kernel_cycles, batches, nthreads=1,
                       max_iters=10_000_000, budget_ms=0.0):
    """Successive batches on one resident state -> (static_flow, flows[], batch_ms[]);
    with budget_ms > 0 the run stops once the batches' total time passes it (the
    lists then cover the batches that ran)."""
    off, adj, w, par = _i32(off), _i32(adj), _i32(w), _i32(par)
    bofs = np.zeros(len(batches) + 1, dtype=np.int64)
    for i, (bs, _, _) in enumerate(batches):
        bofs[i + 1] = bofs[i] + len(bs)
    cat = lambda j: _i32(np.concatenate([b[j] for b in batches]) if batches and bofs[-1] else np.zeros(1))
    src, dst, wt = cat(0), cat(1), cat(2)
    flows = np.zeros(max(len(batches), 1), dtype=np.int64)
    ms = np.zeros(max(len(batches), 1), dtype=np.float64)
    sf = C.c_int64()
    done = C.c_int32()
    rc = lib().orc_ref_run_successive(VARIANTS.get(variant, variant), n, len(adj), off, adj, w, par, s, t,
                                      kernel_cycles, len(batches), bofs, src, dst, wt, nthreads, max_iters,
                                      C.byref(sf), flows, ms, float(budget_ms), C.byref(done))
    if rc:
        raise RuntimeError(f"oracle ref_run_successive failed rc={rc}")
    return sf.value, flows[:done.value], ms[:done.value]
