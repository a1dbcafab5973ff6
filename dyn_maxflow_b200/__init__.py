"""dyn_maxflow_b200 -- Python view of libdmf.so, the B200 dynamic max-flow engine.

The compute path is the C ABI in include/dmf.h (sm_100a kernels); this module only
binds it with ctypes.  There is no CPU fallback: the solver raises DmfError when
no CUDA device is visible, and importing fails when libdmf.so has not been built.

Names mirror the reference (ShruthiKannappan/dyn_maxflow):
  Graph.load / num_nodes / num_edges ..... code/graph.hpp:18-233
  load_updates ........................... code/update.hpp:52-88
  recalculate_max_flow ................... code/dyn_data_bench.cu:171-298
  static_recalculate ..................... code/dyn_data_bench.cu:325-492
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

__all__ = [
    "DmfError", "Graph", "Solver", "Stats", "load_updates", "save_updates", "gen_grid", "gen_rmat",
    "gen_batches", "recalculate_max_flow", "static_recalculate", "device_count", "VARIANTS", "lib_path",
    "static_maxflow_noalloc", "MultiSolver", "Server", "Scheduler", "ACTIONS",
]

_PKG = os.path.dirname(os.path.abspath(__file__))
lib_path = os.path.join(_PKG, "libdmf.so")
if not os.path.exists(lib_path):
    raise ImportError(f"{lib_path} is missing: build it with `python -m dyn_maxflow_b200.build` "
                      "(or __graft_entry__.build()); there is no CPU fallback")
_L = C.CDLL(lib_path)

VARIANTS = {"data": 0, "topo": 1, "pp": 2}
I32P = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
U8P = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
I64P = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
VP = C.c_void_p
PP = C.POINTER(C.c_void_p)


class Opts(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("variant", "kernel_cycles", "relabel_interval", "tile", "max_iters",
                                          "device", "block_threads", "flags", "small_deg", "grid_blocks")]


class Stats(C.Structure):
    _fields_ = [("flow", C.c_int64), ("outer_iters", C.c_int64), ("bfs_levels", C.c_int64),
                ("push_rounds", C.c_int64), ("pushes", C.c_int64), ("relabels", C.c_int64),
                ("arcs_scanned", C.c_int64), ("vertices_visited", C.c_int64), ("dead_vertices", C.c_int64),
                ("last_ms", C.c_double), ("grid_blocks", C.c_int32), ("block_threads", C.c_int32),
                ("tile", C.c_int32), ("pad", C.c_int32), ("bfs_arcs", C.c_int64), ("dead_deficits", C.c_int64),
                ("dead_revived", C.c_int64), ("dead_kept", C.c_int32), ("pad2", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("pad")}


def _sig(name, res, *args):
    f = getattr(_L, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_sig("dmf_last_error", C.c_char_p)
_sig("dmf_status_string", C.c_char_p, C.c_int)
_sig("dmf_opts_default", None, C.POINTER(Opts))
_sig("dmf_free", None, VP)
_sig("dmf_graph_load", C.c_int, C.c_char_p, PP)
_sig("dmf_graph_from_csr", C.c_int, C.c_int32, C.c_int32, I32P, I32P, I32P, I32P, PP)
_sig("dmf_graph_from_edges", C.c_int, C.c_int64, I32P, I32P, I32P, PP)
_sig("dmf_graph_save", C.c_int, VP, C.c_char_p)
_sig("dmf_graph_info", C.c_int, VP, C.POINTER(C.c_int32), C.POINTER(C.c_int32))
_sig("dmf_graph_arrays", C.c_int, VP, PP, PP, PP, PP)
_sig("dmf_graph_find_arc", C.c_int64, VP, C.c_int32, C.c_int32)
_sig("dmf_graph_set_caps", C.c_int, VP, C.c_int32, I32P, I32P, I32P)
_sig("dmf_graph_free", None, VP)
_sig("dmf_updates_load", C.c_int, C.c_char_p, C.POINTER(C.c_int32), PP, PP, PP)
_sig("dmf_updates_save", C.c_int, C.c_char_p, C.c_int32, I32P, I32P, I32P)
_sig("dmf_gen_grid", C.c_int, C.c_int32, C.c_int32, C.c_uint64, C.c_int32, C.c_int32, C.c_int32, PP,
     C.POINTER(C.c_int32), C.POINTER(C.c_int32))
_sig("dmf_gen_rmat", C.c_int, C.c_int32, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_int32,
     C.c_int32, C.c_int64, PP, C.POINTER(C.c_int32), C.POINTER(C.c_int32))
_sig("dmf_gen_batches", C.c_int, VP, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32,
     C.c_int32, C.c_int32, C.c_uint64, PP, PP, PP, PP)
_sig("dmf_solver_create", C.c_int, VP, C.c_int32, C.c_int32, C.POINTER(Opts), VP, PP)
_sig("dmf_static_maxflow", C.c_int, VP, C.POINTER(C.c_int64))
_sig("dmf_apply_updates", C.c_int, VP, C.c_int32, I32P, I32P, I32P, C.POINTER(C.c_int64))
_sig("dmf_apply_updates_device", C.c_int, VP, C.c_int32, VP, VP, VP, C.POINTER(C.c_int64))
_sig("dmf_recompute", C.c_int, VP, C.c_int32, I32P, I32P, I32P, C.POINTER(C.c_int64))
_sig("dmf_recompute_device", C.c_int, VP, C.c_int32, VP, VP, VP, C.POINTER(C.c_int64))
_sig("dmf_flow_value", C.c_int, VP, C.POINTER(C.c_int64))
_sig("dmf_get_cut", C.c_int, VP, U8P)
_sig("dmf_get_state", C.c_int, VP, VP, VP, VP, VP)
_sig("dmf_stats_get", C.c_int, VP, C.POINTER(Stats))
_sig("dmf_trace_get", C.c_int, VP, C.c_int32, I32P, np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"),
     C.POINTER(C.c_int32))
_sig("dmf_trace_items", C.c_int, VP, C.c_int32, I64P, I64P, I64P, I64P)
_sig("dmf_trace_blocks", C.c_int, VP, C.c_int32, I64P)
_sig("dmf_solver_set_opts", C.c_int, VP, C.POINTER(Opts))
_sig("dmf_solver_destroy", C.c_int, VP)
_sig("dmf_device_count", C.c_int)
_sig("dmf_multi_create", C.c_int, C.c_int32, C.POINTER(C.c_void_p), I32P, I32P, C.POINTER(Opts), VP, PP)
_sig("dmf_multi_info", C.c_int, VP, C.POINTER(C.c_int32), I32P)
_sig("dmf_multi_static_maxflow", C.c_int, VP, I64P)
_sig("dmf_multi_apply_updates", C.c_int, VP, C.c_int32, I32P, I32P, I32P, I32P, I64P)
_sig("dmf_multi_run_batches", C.c_int, VP, C.c_int32, I64P, VP, VP, VP, C.c_int32, I64P, C.POINTER(C.c_double))
_sig("dmf_autotune", C.c_int, VP, C.c_int32, C.POINTER(Opts))
_sig("dmf_server_create", C.c_int, C.c_int32, C.POINTER(C.c_void_p), I32P, I32P, C.c_int64, C.POINTER(Opts), PP)
_sig("dmf_server_info", C.c_int, VP, C.POINTER(C.c_int32), C.POINTER(C.c_int64))
_sig("dmf_server_lane", C.c_int, VP, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32))
_sig("dmf_server_submit", C.c_int, VP, C.c_int32, C.c_int32, I32P, I32P, I32P, C.POINTER(C.c_int64))
_sig("dmf_server_wait", C.c_int, VP, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_double))
_sig("dmf_server_stats", C.c_int, VP, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_double))
_sig("dmf_server_destroy", C.c_int, VP)
F32P = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
U16P = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
_sig("dmf_sched_create", C.c_int, C.c_int32, C.c_uint64, PP)
_sig("dmf_sched_destroy", C.c_int, VP)
_sig("dmf_sched_set_weights", C.c_int, VP, U16P, F32P)
_sig("dmf_sched_get_weights", C.c_int, VP, U16P, F32P)
_sig("dmf_sched_set_margin", C.c_int, VP, C.c_float)
_sig("dmf_sched_train", C.c_int, VP, C.c_int32, F32P, F32P, C.c_int32, C.c_int32, C.c_float, C.c_uint64, F32P)
_sig("dmf_sched_predict", C.c_int, VP, C.c_int32, F32P, F32P)
_sig("dmf_solver_features", C.c_int, VP, C.c_int32, I32P, I32P, I32P, F32P)
_sig("dmf_apply_updates_action", C.c_int, VP, C.c_int32, C.c_int32, I32P, I32P, I32P, C.POINTER(C.c_int64))
_sig("dmf_apply_updates_scheduled", C.c_int, VP, VP, C.c_int32, I32P, I32P, I32P, C.POINTER(C.c_int64),
     C.POINTER(C.c_int32))
_sig("dmf_sched_records", C.c_int, VP, C.c_int32, F32P, I32P, F32P, I64P, C.POINTER(C.c_int32))
_sig("dmf_solver_copy_state", C.c_int, VP, VP)

# schedules the picker chooses from (DMF_ACTION_*); every one gives the same flow
ACTIONS = ("plain", "short_interval", "revive_dead", "recompute")
N_FEATURES, N_HIDDEN, N_ACTIONS, N_WEIGHTS, N_BIASES = 12, 64, 4, 5120, 132

_sig("dmf_static_maxflow_noalloc", C.c_int, C.c_int32, C.c_int32, VP, VP, VP, VP, C.c_int32, C.c_int32, VP,
     C.POINTER(C.c_int64), VP)


def static_maxflow_noalloc(n, m, d_index, d_adj, d_cap, d_par, s, t, d_res, stream=None) -> int:
    """dmf_static_maxflow_noalloc over caller-owned device buffers (raw pointers):
    the solver allocates nothing; its scratch is a static device array (n <= 262144)."""
    f = C.c_int64()
    st = None if stream is None else C.c_void_p(int(getattr(stream, "cuda_stream", stream)))
    _check(_L.dmf_static_maxflow_noalloc(n, m, C.c_void_p(d_index), C.c_void_p(d_adj), C.c_void_p(d_cap),
                                         C.c_void_p(d_par), s, t, C.c_void_p(d_res), C.byref(f), st))
    return f.value


class DmfError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{_L.dmf_status_string(status).decode()}] {msg}")
        self.status = status


def _check(st: int) -> None:
    if st:
        raise DmfError(st, (_L.dmf_last_error() or b"").decode())


def _i32(a) -> np.ndarray:
    """Contiguous int32 view or copy; values that int32 cannot hold exactly
    (out of range, fractional) raise instead of wrapping to another id."""
    a = np.asarray(a)
    if a.dtype != np.int32 and a.size:
        if a.dtype.kind not in "biuf":
            raise TypeError(f"expected integers, got {a.dtype}")
        if a.dtype.kind == "f" and not np.array_equal(a, np.trunc(a)):
            raise ValueError("expected integers, got fractional values")
        if a.min() < -2**31 or a.max() > 2**31 - 1:
            raise OverflowError("value outside the int32 range")
    return np.ascontiguousarray(a, dtype=np.int32)


def _take_i32(ptr: C.c_void_p, count: int) -> np.ndarray:
    if count == 0 or not ptr.value:
        _L.dmf_free(ptr)
        return np.zeros(0, np.int32)
    a = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int32)), shape=(count,)).copy()
    _L.dmf_free(ptr)
    return a


def device_count() -> int:
    return int(_L.dmf_device_count())


class Graph:
    """Host CSR in the reference's .bin layout (code/graph.hpp:18-233)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _L.dmf_graph_free(h)
            self._h = None

    @classmethod
    def load(cls, path: str) -> "Graph":
        """graph::loadGraph, code/graph.hpp:202-223."""
        h = C.c_void_p()
        _check(_L.dmf_graph_load(os.fsencode(path), C.byref(h)))
        return cls(h)

    loadGraph = load

    @classmethod
    def from_csr(cls, index, adj, w, par) -> "Graph":
        index, adj, w, par = _i32(index), _i32(adj), _i32(w), _i32(par)
        h = C.c_void_p()
        _check(_L.dmf_graph_from_csr(len(index) - 1, len(adj), index, adj, w, par, C.byref(h)))
        return cls(h)

    @classmethod
    def from_edges(cls, u, v, w) -> "Graph":
        """input_create/create_bin.cpp:67-124 semantics."""
        u, v, w = _i32(u), _i32(v), _i32(w)
        h = C.c_void_p()
        _check(_L.dmf_graph_from_edges(len(u), u, v, w, C.byref(h)))
        return cls(h)

    def save(self, path: str) -> None:
        _check(_L.dmf_graph_save(self._h, os.fsencode(path)))

    def num_nodes(self) -> int:
        n, m = C.c_int32(), C.c_int32()
        _check(_L.dmf_graph_info(self._h, C.byref(n), C.byref(m)))
        return n.value

    def num_edges(self) -> int:
        n, m = C.c_int32(), C.c_int32()
        _check(_L.dmf_graph_info(self._h, C.byref(n), C.byref(m)))
        return m.value

    def arrays(self):
        """(index[n+1], adj[m], w[m], par[m]) as numpy copies."""
        n, m = self.num_nodes(), self.num_edges()
        ps = [C.c_void_p() for _ in range(4)]
        _check(_L.dmf_graph_arrays(self._h, *[C.byref(p) for p in ps]))
        out = []
        for p, cnt in zip(ps, (n + 1, m, m, m)):
            out.append(np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_int32)), shape=(max(cnt, 1),))[:cnt].copy())
        return tuple(out)

    def find_arc(self, src: int, dst: int) -> int:
        return int(_L.dmf_graph_find_arc(self._h, src, dst))

    def set_caps(self, src, dst, w) -> None:
        """update_kernel (code/dyn_data_bench.cu:300-322) on the host copy."""
        src, dst, w = _i32(src), _i32(dst), _i32(w)
        _check(_L.dmf_graph_set_caps(self._h, len(src), src, dst, w))


def load_updates(path: str):
    """loadUpdateFile, code/update.hpp:52-88 -> (src, dst, w) int32 arrays."""
    k = C.c_int32()
    ps = [C.c_void_p() for _ in range(3)]
    _check(_L.dmf_updates_load(os.fsencode(path), C.byref(k), *[C.byref(p) for p in ps]))
    return tuple(_take_i32(p, k.value) for p in ps)


def save_updates(path: str, src, dst, w) -> None:
    src, dst, w = _i32(src), _i32(dst), _i32(w)
    _check(_L.dmf_updates_save(os.fsencode(path), len(src), src, dst, w))


def gen_grid(rows=256, cols=256, seed=0, cap_lo=1, cap_hi=100, st_cap=1000):
    """-> (Graph, s, t)."""
    h, s, t = C.c_void_p(), C.c_int32(), C.c_int32()
    _check(_L.dmf_gen_grid(rows, cols, seed, cap_lo, cap_hi, st_cap, C.byref(h), C.byref(s), C.byref(t)))
    return Graph(h), s.value, t.value


def gen_rmat(scale=20, narcs=None, a=0.57, b=0.19, c=0.19, seed=0, cap_lo=1, cap_hi=1000, reserve=0):
    """-> (Graph, s, t); narcs defaults to 16 * 2^scale."""
    if narcs is None:
        narcs = 16 << scale
    h, s, t = C.c_void_p(), C.c_int32(), C.c_int32()
    _check(_L.dmf_gen_rmat(scale, narcs, a, b, c, seed, cap_lo, cap_hi, reserve, C.byref(h), C.byref(s),
                           C.byref(t)))
    return Graph(h), s.value, t.value


def gen_batches(g: Graph, nbatches, frac=0.01, p_inc=0.4, p_dec=0.4, p_ins=0.1, delta_hi=500, ins_lo=1,
                ins_hi=1000, seed=1):
    """-> list of (src, dst, w) per batch (successive: batch b assumes batches < b applied)."""
    ofs, s, d, w = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
    _check(_L.dmf_gen_batches(g._h, nbatches, frac, p_inc, p_dec, p_ins, delta_hi, ins_lo, ins_hi, seed,
                              C.byref(ofs), C.byref(s), C.byref(d), C.byref(w)))
    o = np.ctypeslib.as_array(C.cast(ofs, C.POINTER(C.c_int64)), shape=(nbatches + 1,)).copy()
    _L.dmf_free(ofs)
    k = int(o[-1])
    S, D, W = _take_i32(s, k), _take_i32(d, k), _take_i32(w, k)
    return [(S[o[i]:o[i + 1]].copy(), D[o[i]:o[i + 1]].copy(), W[o[i]:o[i + 1]].copy()) for i in range(nbatches)]


class Solver:
    """Device-resident residual state of one graph on one GPU (dmf_solver)."""

    def __init__(self, g: Graph, source: int, sink: int, variant="data", kernel_cycles=0, relabel_interval=0,
                 tile=0, max_iters=0, device=-1, stream=None, trace=False, probe=False, fixed_interval=False,
                 revive_dead=False, test_barrier_timeout=False):
        o = Opts()
        _L.dmf_opts_default(C.byref(o))
        o.variant = VARIANTS[variant] if isinstance(variant, str) else int(variant)
        o.kernel_cycles, o.relabel_interval, o.tile, o.max_iters, o.device = (
            kernel_cycles, relabel_interval, tile, max_iters, device)
        o.flags = ((1 if trace or probe else 0) | (2 if probe else 0) | (4 if fixed_interval else 0)
                   | (8 if revive_dead else 0) | (16 if test_barrier_timeout else 0))
        self._h = C.c_void_p()
        self.n, self.m = g.num_nodes(), g.num_edges()
        stream_ptr = None if stream is None else C.c_void_p(int(getattr(stream, "cuda_stream", stream)))
        _check(_L.dmf_solver_create(g._h, source, sink, C.byref(o), stream_ptr, C.byref(self._h)))
        self.source, self.sink = source, sink

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _L.dmf_solver_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def static_maxflow(self) -> int:
        f = C.c_int64()
        _check(_L.dmf_static_maxflow(self._h, C.byref(f)))
        return f.value

    def apply_updates(self, src, dst, w) -> int:
        src, dst, w = _i32(src), _i32(dst), _i32(w)
        f = C.c_int64()
        _check(_L.dmf_apply_updates(self._h, len(src), src, dst, w, C.byref(f)))
        return f.value

    def apply_updates_device(self, d_src: int, d_dst: int, d_w: int, k: int) -> int:
        """Batch already on the device (raw device pointers, e.g. tensor.data_ptr())."""
        f = C.c_int64()
        _check(_L.dmf_apply_updates_device(self._h, k, C.c_void_p(d_src), C.c_void_p(d_dst), C.c_void_p(d_w),
                                           C.byref(f)))
        return f.value

    def features(self, src, dst, w) -> np.ndarray:
        """The schedule picker's 12 features of a batch against the current state (nothing applied)."""
        src, dst, w = _i32(src), _i32(dst), _i32(w)
        out = np.zeros(N_FEATURES, np.float32)
        _check(_L.dmf_solver_features(self._h, len(src), src, dst, w, out))
        return out

    def apply_updates_action(self, action: int, src, dst, w) -> int:
        """Applies a batch under one schedule (index into ACTIONS); same flow for every action."""
        src, dst, w = _i32(src), _i32(dst), _i32(w)
        f = C.c_int64()
        _check(_L.dmf_apply_updates_action(self._h, int(action), len(src), src, dst, w, C.byref(f)))
        return f.value

    def apply_updates_scheduled(self, sched, src, dst, w):
        """Applies a batch under the schedule `sched` (a Scheduler, or None for the plain
        one) picks; returns (flow, action)."""
        src, dst, w = _i32(src), _i32(dst), _i32(w)
        f, a = C.c_int64(), C.c_int32()
        _check(_L.dmf_apply_updates_scheduled(self._h, None if sched is None else sched._h, len(src), src, dst, w,
                                              C.byref(f), C.byref(a)))
        return f.value, a.value

    def sched_records(self, cap: int = 1 << 16):
        """Drains the per-batch records of the scheduled/action calls:
        (features[n,12], action[n], ms[n], flow[n])."""
        feat = np.zeros((cap, N_FEATURES), np.float32)
        act = np.zeros(cap, np.int32)
        ms = np.zeros(cap, np.float32)
        fl = np.zeros(cap, np.int64)
        cnt = C.c_int32()
        _check(_L.dmf_sched_records(self._h, cap, feat.reshape(-1), act, ms, fl, C.byref(cnt)))
        n = cnt.value
        return feat[:n], act[:n], ms[:n], fl[:n]

    def copy_state_from(self, other: "Solver") -> None:
        """Makes this solver's residual state an exact copy of `other`'s (same graph)."""
        _check(_L.dmf_solver_copy_state(self._h, other._h))

    def recompute(self, src=(), dst=(), w=()) -> int:
        src, dst, w = _i32(src), _i32(dst), _i32(w)
        f = C.c_int64()
        _check(_L.dmf_recompute(self._h, len(src), src, dst, w, C.byref(f)))
        return f.value

    def recompute_device(self, d_src: int, d_dst: int, d_w: int, k: int) -> int:
        f = C.c_int64()
        _check(_L.dmf_recompute_device(self._h, k, C.c_void_p(d_src), C.c_void_p(d_dst), C.c_void_p(d_w),
                                       C.byref(f)))
        return f.value

    @property
    def flow(self) -> int:
        f = C.c_int64()
        _check(_L.dmf_flow_value(self._h, C.byref(f)))
        return f.value

    def cut(self) -> np.ndarray:
        """1 = sink side (find_cut, code/dyn_pp.h:440-449)."""
        out = np.zeros(self.n, dtype=np.uint8)
        _check(_L.dmf_get_cut(self._h, out))
        return out

    def state(self):
        """(cap[m], res[m], excess[n], height[n]) copied from the device."""
        cap = np.zeros(max(self.m, 1), np.int32)
        res = np.zeros(max(self.m, 1), np.int32)
        ex = np.zeros(max(self.n, 1), np.int64)
        h = np.zeros(max(self.n, 1), np.int32)
        _check(_L.dmf_get_state(self._h, cap.ctypes.data, res.ctypes.data, ex.ctypes.data, h.ctypes.data))
        return cap[:self.m], res[:self.m], ex[:self.n], h[:self.n]

    TRACE_KINDS = {0: "start", 1: "init_res", 2: "saturate", 3: "lookup", 4: "apply", 5: "repair",
                   6: "cut_saturate", 7: "bfs_init", 8: "bfs_td", 9: "bfs_bu", 10: "bfs_finalize", 11: "push",
                   12: "flow", 13: "push_hub", 14: "push_hub_finish", 15: "pp_init", 16: "pp_bfs",
                   17: "pp_finalize", 18: "pp_round", 19: "reopen", 20: "dead_seed", 21: "dead_pull",
                   23: "dead_check", 24: "dead_revive", 25: "claim"}

    def trace(self):
        """[(phase kind, end time in us since kernel start)] of the last solve (trace=True)."""
        cnt = C.c_int32()
        _check(_L.dmf_trace_get(self._h, 0, np.zeros(1, np.int32), np.zeros(1), C.byref(cnt)))
        cap = max(cnt.value, 1)
        kinds = np.zeros(cap, np.int32)
        t = np.zeros(cap, np.float64)
        _check(_L.dmf_trace_get(self._h, cap, kinds, t, C.byref(cnt)))
        n = cnt.value
        items = np.zeros(max(n, 1), np.int64)
        hubs = np.zeros(max(n, 1), np.int64)
        sns = np.zeros(max(n, 1), np.int64)
        sv_ = np.zeros(max(n, 1), np.int64)
        _check(_L.dmf_trace_items(self._h, n, items, hubs, sns, sv_))
        blk = np.zeros(max(n, 1), np.int64)
        _check(_L.dmf_trace_blocks(self._h, n, blk))
        # per phase: (items, hub chunks, longest item ns, its vertex, longest block work ns)
        self.last_trace_items = list(zip(items[:n].tolist(), hubs[:n].tolist(), sns[:n].tolist(), sv_[:n].tolist(),
                                         blk[:n].tolist()))
        return [(self.TRACE_KINDS.get(int(k), str(k)), float(x)) for k, x in zip(kinds[:n], t[:n])]

    def stats(self) -> dict:
        st = Stats()
        _check(_L.dmf_stats_get(self._h, C.byref(st)))
        return st.as_dict()

    def autotune(self, repeats=2) -> dict:
        """dmf_autotune: picks tile / per-thread degree bound / relabel interval / cycles."""
        o = Opts()
        _check(_L.dmf_autotune(self._h, repeats, C.byref(o)))
        return {k: getattr(o, k) for k, _ in Opts._fields_}

    def set_opts(self, variant=None, kernel_cycles=None, relabel_interval=None, tile=None, max_iters=None,
                 small_deg=None, flags=None):
        """Replaces the solver's options (dmf_solver_set_opts); a field left None keeps the
        value a previous set_opts call gave it, else the library default."""
        o = Opts()
        _L.dmf_opts_default(C.byref(o))
        cur = getattr(self, "_opts", {})
        vals = dict(variant=variant, kernel_cycles=kernel_cycles, relabel_interval=relabel_interval, tile=tile,
                    max_iters=max_iters, small_deg=small_deg, flags=flags)
        for k_, v_ in vals.items():
            if v_ is None:
                v_ = cur.get(k_, 0 if k_ != "variant" else 0)
            if k_ == "variant" and isinstance(v_, str):
                v_ = VARIANTS[v_]
            setattr(o, k_, v_)
            cur[k_] = v_
        self._opts = cur
        _check(_L.dmf_solver_set_opts(self._h, C.byref(o)))


def recalculate_max_flow(g: Graph, updates, source: int, sink: int, kernel_cycles: int = 0, variant="data") -> int:
    """Dynamic path of the reference bench (code/dyn_data_bench.cu:171-298): a fresh
    device state of the ORIGINAL graph, static solve, one batch, flow readout."""
    with Solver(g, source, sink, variant=variant, kernel_cycles=kernel_cycles) as sv:
        sv.static_maxflow()
        return sv.apply_updates(*updates)


def static_recalculate(g: Graph, updates, source: int, sink: int, kernel_cycles: int = 0, variant="data") -> int:
    """From-scratch path of the reference bench (code/dyn_data_bench.cu:325-492)."""
    with Solver(g, source, sink, variant=variant, kernel_cycles=kernel_cycles) as sv:
        return sv.recompute(*updates)


class MultiSolver(Solver):
    """Many independent graphs in one device state (dmf_multi_*): one persistent
    launch per call serves every instance; flows come back per instance."""

    def __init__(self, graphs, sources, sinks, variant="data", kernel_cycles=0, relabel_interval=0, tile=0,
                 device=-1, stream=None, small_deg=0):
        o = Opts()
        _L.dmf_opts_default(C.byref(o))
        o.variant = VARIANTS[variant] if isinstance(variant, str) else int(variant)
        o.kernel_cycles, o.relabel_interval, o.tile, o.device, o.small_deg = (
            kernel_cycles, relabel_interval, tile, device, small_deg)
        self._h = C.c_void_p()
        self.graphs = list(graphs)
        arr = (C.c_void_p * len(self.graphs))(*[g._h.value for g in self.graphs])
        stream_ptr = None if stream is None else C.c_void_p(int(getattr(stream, "cuda_stream", stream)))
        _check(_L.dmf_multi_create(len(self.graphs), arr, _i32(sources), _i32(sinks), C.byref(o), stream_ptr,
                                   C.byref(self._h)))
        self.count = len(self.graphs)
        self.n = sum(g.num_nodes() for g in self.graphs)
        self.m = sum(g.num_edges() for g in self.graphs)
        cnt = C.c_int32()
        base = np.zeros(self.count, np.int32)
        _check(_L.dmf_multi_info(self._h, C.byref(cnt), base))
        self.vertex_base = base

    def static_maxflow_all(self) -> np.ndarray:
        out = np.zeros(self.count, np.int64)
        _check(_L.dmf_multi_static_maxflow(self._h, out))
        return out

    def apply_updates_all(self, inst, src, dst, w) -> np.ndarray:
        inst, src, dst, w = _i32(inst), _i32(src), _i32(dst), _i32(w)
        out = np.zeros(self.count, np.int64)
        _check(_L.dmf_multi_apply_updates(self._h, len(src), inst, src, dst, w, out))
        return out

    def run_batches(self, ofs, d_src: int, d_dst: int, d_w: int, use_graph=True):
        """Successive device-resident batches (union vertex ids); -> (flows[steps, count], ms)."""
        ofs = np.ascontiguousarray(ofs, dtype=np.int64)
        steps = len(ofs) - 1
        out = np.zeros(steps * self.count, np.int64)
        ms = C.c_double()
        _check(_L.dmf_multi_run_batches(self._h, steps, ofs, C.c_void_p(d_src), C.c_void_p(d_dst), C.c_void_p(d_w),
                                        1 if use_graph else 0, out, C.byref(ms)))
        return out.reshape(steps, self.count), ms.value


class Scheduler:
    """The learned schedule picker (dmf_sched): MLP 12-64-64-4 with bf16 weights and fp32
    accumulation; training and inference run in CUDA kernels on the device."""

    def __init__(self, device: int = -1, seed: int = 0):
        self._h = C.c_void_p()
        _check(_L.dmf_sched_create(device, seed, C.byref(self._h)))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _L.dmf_sched_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_margin(self, margin: float) -> None:
        """log2 units a non-plain action must be predicted to win by (default 0.1)."""
        _check(_L.dmf_sched_set_margin(self._h, float(margin)))

    def get_weights(self):
        """(weights[5120] as bf16 bit patterns in uint16, biases[132] fp32)."""
        w = np.zeros(N_WEIGHTS, np.uint16)
        b = np.zeros(N_BIASES, np.float32)
        _check(_L.dmf_sched_get_weights(self._h, w, b))
        return w, b

    def set_weights(self, weights, biases) -> None:
        _check(_L.dmf_sched_set_weights(self._h, np.ascontiguousarray(weights, np.uint16),
                                        np.ascontiguousarray(biases, np.float32)))

    def train(self, X, Y, steps=2000, batch=64, lr=3e-3, seed=0) -> np.ndarray:
        """Minibatch Adam on the device; returns the per-step minibatch MSE."""
        X = np.ascontiguousarray(X, np.float32).reshape(-1)
        Y = np.ascontiguousarray(Y, np.float32).reshape(-1)
        n = len(Y) // N_ACTIONS
        loss = np.zeros(max(steps, 1), np.float32)
        _check(_L.dmf_sched_train(self._h, n, X, Y, steps, batch, lr, seed, loss))
        return loss[:steps]

    def predict(self, X) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32).reshape(-1)
        n = len(X) // N_FEATURES
        Y = np.zeros(n * N_ACTIONS, np.float32)
        _check(_L.dmf_sched_predict(self._h, n, X, Y))
        return Y.reshape(n, N_ACTIONS)

    def save(self, path: str) -> None:
        w, b = self.get_weights()
        np.savez(path, weights=w, biases=b)

    @classmethod
    def load(cls, path: str, device: int = -1) -> "Scheduler":
        d = np.load(path)
        s = cls(device)
        s.set_weights(d["weights"], d["biases"])
        return s


class Server:
    """Serving loop (dmf_server_*): device-resident graphs admitted by HBM budget,
    continuous batching of update-batch requests.  submit() returns a ticket;
    wait(ticket) -> (flow, latency_ms).  Thread-safe."""

    def __init__(self, graphs, sources, sinks, hbm_budget_bytes, variant="data"):
        o = Opts()
        _L.dmf_opts_default(C.byref(o))
        o.variant = VARIANTS[variant] if isinstance(variant, str) else int(variant)
        self.graphs = list(graphs)  # kept alive for the server
        arr = (C.c_void_p * len(self.graphs))(*[g._h.value for g in self.graphs])
        self._h = C.c_void_p()
        _check(_L.dmf_server_create(len(self.graphs), arr, _i32(sources), _i32(sinks), int(hbm_budget_bytes),
                                    C.byref(o), C.byref(self._h)))
        adm, by = C.c_int32(), C.c_int64()
        _check(_L.dmf_server_info(self._h, C.byref(adm), C.byref(by)))
        self.admitted, self.device_bytes = adm.value, by.value

    def submit(self, graph, src, dst, w) -> int:
        src, dst, w = _i32(src), _i32(dst), _i32(w)
        tk = C.c_int64()
        _check(_L.dmf_server_submit(self._h, graph, len(src), src, dst, w, C.byref(tk)))
        return tk.value

    def wait(self, ticket):
        f, lat = C.c_int64(), C.c_double()
        _check(_L.dmf_server_wait(self._h, ticket, C.byref(f), C.byref(lat)))
        return f.value, lat.value

    def stats(self) -> dict:
        a, b, c = C.c_int64(), C.c_int64(), C.c_double()
        _check(_L.dmf_server_stats(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return {"ticks": a.value, "served": b.value, "mean_requests_per_tick": c.value}

    def lane(self, graph: int) -> dict:
        """dmf_server_lane: the lane serving `graph` and its share of resident blocks."""
        ln, lns, gb = C.c_int32(), C.c_int32(), C.c_int32()
        _check(_L.dmf_server_lane(self._h, graph, C.byref(ln), C.byref(lns), C.byref(gb)))
        return {"lane": ln.value, "lanes": lns.value, "grid_blocks": gb.value}

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _L.dmf_server_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
