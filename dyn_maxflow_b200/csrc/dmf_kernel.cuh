// dmf_kernel.cuh -- the persistent push-relabel solve kernel for sm_100a
// (k_solve), with its phases.  Each dmf_kernel_tN.cu instantiates it for one
// tile width, so the instantiations compile in parallel; dmf_solver.cu holds
// the host side.
//
// One cooperative launch runs a whole solve: the update prologue (arc lookup,
// capacity apply, over-capacity repair, source saturation), then rounds of
//   global relabel: direction-optimising reverse BFS from t and the deficit
//                   vertices over residual arcs, which also builds the active
//                   worklist and proves unreachable vertices dead;
//   push rounds:    discharge of every active vertex by a warp tile (or a whole
//                   block for hubs), multi-arc pushes per adjacency scan, with
//                   warp-aggregated worklist appends;
// until a global relabel finds no active vertex, then the flow readout
// excess(t) + sum of deficits (recalculate_max_flow_kernel_39,
// code/dyn_data.h:208-215).  Phases are separated by a bounded grid barrier, so
// no host round trip happens inside a solve (the reference syncs and copies a
// flag per BFS level, code/dyn_data_bench.cu:39-47).
//
// A dynamic batch keeps the dead set of the last solve (the vertices proven
// unable to reach t or a deficit): updated arcs that open residual from it to
// the live side are saturated at once (ph_reopen), the deficits this leaves
// inside the dead set are covered there by pulls from excess inside it
// (ph_dead_seed, ph_dead_pull), and the global relabels then only visit live
// vertices.  A deficit the pulls cannot cover revives the dead vertices that
// can reach it (ph_dead_check, ph_dead_revive), or every vertex when those are
// too many.
#pragma once
#include <cuda_runtime.h>

#include <climits>

#include "dmf_device.cuh"
#include "dmf.h"

namespace dmfk {

using namespace dmfd;

constexpr int kBlock = 512;
constexpr int kChunk = 256;  // arcs per hub chunk: one warp item, 8 arcs per lane
constexpr int kPPIters = 1;  // push-pull phase-1 relabel rounds before the general solve

enum Mode : int { MODE_STATIC = 0, MODE_DYNAMIC = 1, MODE_RECOMPUTE = 2, MODE_CUT = 3 };

// Phase kinds of the optional timeline (dmf_trace_get); values are part of the ABI.
enum TraceKind : int {
  TR_START = 0, TR_INIT_RES = 1, TR_SATURATE = 2, TR_LOOKUP = 3, TR_APPLY = 4, TR_REPAIR = 5,
  TR_CUT_SATURATE = 6, TR_BFS_INIT = 7, TR_BFS_TD = 8, TR_BFS_BU = 9, TR_BFS_FINALIZE = 10, TR_PUSH = 11,
  TR_FLOW = 12, TR_PUSH_HUB = 13, TR_PUSH_HUB_FINISH = 14, TR_PP_INIT = 15, TR_PP_BFS = 16, TR_PP_FINALIZE = 17,
  TR_PP_ROUND = 18, TR_REOPEN = 19, TR_DEAD_SEED = 20, TR_DEAD_PULL = 21, TR_DEAD_CHECK = 23,
  TR_DEAD_REVIVE = 24
};

// Local repair inside a kept dead set: at most this many pull rounds.
constexpr int kDeadRounds = 16;

// Largest capacity an update may set: keeps cap(e) + cap(partner) < 2^31 when
// both arcs of a pair change in one batch.
constexpr int kMaxUpdateCap = (1 << 30) - 1;

struct Params {
  int n, m, s, t;
  const int *__restrict__ off;
  const int *__restrict__ adj;
  const int *__restrict__ par;
  ArcSlot *atab;    // (tail, head) -> arc table with the per-arc batch stamps
  long long nslots;  // its slots
  int *cap;                  // capacities as a plain array (allocation-free static solve only)
  unsigned long long *capx;  // capacities of a solver: (epoch of the batch that set it << 32) | capacity
  int *res, *height, *stamp, *uarc;
  int *uold;  // per update: the capacity it replaced (-1: an earlier update of the batch named the arc)
  long long *excess;
  unsigned char *dead, *side;
  int *fq[2], *wq[2], *aq;     // non-hub vertex queues
  int *dq;                     // dead vertices whose excess the batch changed (kept dead set)
  int *dlab;                   // distance from excess inside the dead set, (wave << 4) | level
  int *pcur;                   // per vertex: where in its row its last pull found enough (long rows; may be null)
  int2 *fh[2], *wh[2], *ah;    // hub chunk queues
  const int2 *hch;             // every hub's chunks (bottom-up BFS, topology-driven rounds)
  int nhch;
  // per hub (indexed by hub_base), totals of the current push round:
  long long *hc_alloc;  // admissible residual claimed by the hub's chunks
  long long *hc_moved;  // excess pushed by them
  int *hc_min;          // minimum non-admissible head height
  int *hc_done;         // chunks that contributed to hc_min
  // Exhausted hub chunks: a chunk with no admissible arc at hub height h stays
  // so until the hub's height changes or the next global relabel (heights only
  // rise in between, and a reverse residual only opens from a higher head).
  // mark = (relabel epoch << 32) | h, indexed by hub_base[v] + chunk.
  const int *hub_base;
  unsigned long long *chunk_mark;
  int *chunk_tmin;
  unsigned relabel_base;
  const int *usrc, *udst, *uw;
  int k;
  // Several independent instances in one residual graph (batched mode): role
  // bit 0 = a source, bit 1 = a sink, inst = instance of each vertex, flows per
  // instance.  Single instance: role == nullptr, s and t above.
  const unsigned char *role;
  const int *inst;
  long long *inst_flow;
  const int *srcs;  // every source vertex (just s for one instance)
  // prefix sums of the sources' degrees (nsrc + 1 entries), or null: the
  // saturation then walks the sources one after the other
  const int *src_off;
  int nsrc;
  // instances a batched call works on (nullptr: all); the others are left as they
  // are: not seeded, not saturated, not read out
  const unsigned char *inst_active;
  Ctrl *ctrl;
  int mode, variant, cycles, interval, max_iters, hub_deg, small_deg, need_cut;
  // Dynamic batch with the dead set of the last solve kept: dead vertices stay
  // dead unless the batch gives them a deficit that cannot be covered inside
  // the dead set (then the first global relabel revives every vertex).
  int keep_dead;
  // every capacity is at most kMaxUpdateCap, so a pair's sum cannot overflow
  // and the lookup need not read the partner's capacity
  int caps_bounded;
  int bu_alpha;  // bottom-up when frontier arcs * bu_alpha > unexplored arcs (0: never)
  int adaptive;  // push rounds per relabel at least the depth of the last relabel BFS
  unsigned round_base;
  int epoch;
  unsigned long long *trace;  // optional phase timeline: 4 words per entry
  int trace_cap;
  int probe;                  // time work items (DMF_FLAG_PROBE)
  unsigned long long barrier_ns;  // grid-barrier wait limit
  // Failure-injection test hook (DMF_FLAG_TEST_BARRIER_TIMEOUT): this block
  // leaves at once and never arrives at a barrier (-1: none).
  int absent_block;
};

struct LStats {
  unsigned long long pushes = 0, relabels = 0, arcs = 0, visits = 0;
  unsigned long long barcs = 0;  // adjacency entries read by BFS levels
  unsigned long long probe = 0;  // (longest single item in ns << 32) | vertex, this phase
  unsigned long long t_phase = 0;  // thread 0: when this block left the last barrier
  long long to_sink = 0;  // flow pushed into the sink this push phase, not yet added
};

// Optional probe (DMF_FLAG_PROBE): times every work item and keeps the longest.
struct ItemTimer {
  unsigned long long t0;
  bool on;
  __device__ __forceinline__ ItemTimer(const Params &p) : t0(0), on(p.probe) {
    if (on) t0 = globaltimer();
  }
  __device__ __forceinline__ void done(LStats &ls, int v) {
    if (!on) return;
    unsigned long long dt = globaltimer() - t0;
    if (dt > 0xffffffffull) dt = 0xffffffffull;
    const unsigned long long key = (dt << 32) | (unsigned)v;
    if (key > ls.probe) ls.probe = key;
  }
};

__device__ __forceinline__ int deg_of(const Params &p, int v) { return __ldg(p.off + v + 1) - __ldg(p.off + v); }

__device__ __forceinline__ bool is_src(const Params &p, int v) { return p.role ? (p.role[v] & 1) : v == p.s; }
__device__ __forceinline__ bool is_snk(const Params &p, int v) { return p.role ? (p.role[v] & 2) : v == p.t; }
__device__ __forceinline__ bool is_term(const Params &p, int v) { return p.role ? p.role[v] != 0 : (v == p.s || v == p.t); }
// Whether v's instance takes part in this call (batched mode with a mask).
__device__ __forceinline__ bool inst_on(const Params &p, int v) {
  return !p.inst_active || p.inst_active[__ldg(p.inst + v)];
}

__device__ __forceinline__ void set_err(Ctrl *c, int bit, int info) {
  if (atomicOr(&c->err, bit) == 0) c->err_info = info;
}

// A dead vertex whose excess a batch lowers joins the candidate list once
// (stamp = round_base, a value no push round of this call uses).  The pull
// rounds later append the dead vertices they take below zero, so after them
// the list holds every dead vertex that can hold a deficit (dead vertices end
// every solve with excess >= 0).  The list has n + 1 entries; a count past
// that means some were dropped, and the dead check then sweeps every vertex.
__device__ __forceinline__ void add_dead_cand(const Params &p, int v) {
  if (atomicExch(p.stamp + v, (int)p.round_base) == (int)p.round_base) return;
  append_bounded(p.dq, &p.ctrl->dcand, v, p.n + 1);
}

// Capacities of a solver live in 8-byte words, capacity in the low half and
// in the high half the launch epoch of the batch that last set it (0 from the
// upload).  A batch swaps (epoch, w) in for every update; an update that gets
// back a word with this launch's epoch names an arc an earlier update of the
// batch named, so the batch is rejected (Ctrl::dup_at, read after the barrier)
// and ph_unclaim puts back what was changed.  The duplicate check thus rides on
// the capacity line the apply reads and writes anyway: no per-arc stamp, and
// no second write to clear a mark.  The caller-supplied capacities of the
// allocation-free static solve stay a plain int32 array (capx == nullptr).
__device__ __forceinline__ int cap_of(const Params &p, int e) {
  return p.capx ? (int)(unsigned)__ldcg(p.capx + e) : __ldcg(p.cap + e);
}

__device__ __forceinline__ unsigned long long cap_word(const Params &p, int w) {
  return ((unsigned long long)(unsigned)p.epoch << 32) | (unsigned)w;
}

// ---- prologue phases ----------------------------------------------------------

// staticMaxFlow_kernel_1 (code/dyn_data.h:25-35): residual = capacity, excess 0.
__device__ __forceinline__ void ph_init_res(const Params &p) {
  const int nt = gridDim.x * blockDim.x, gt = blockIdx.x * blockDim.x + threadIdx.x;
  for (int e = gt; e < p.m; e += nt) p.res[e] = cap_of(p, e);
  for (int v = gt; v < p.n; v += nt) p.excess[v] = 0;
}

// staticMaxFlow_kernel_7 (code/dyn_data.h:39-56) made parallel: every residual
// arc out of every source is saturated.  The arcs of all sources form one index
// space (src_off) walked grid-stride, so one source of very high degree (R-MAT's
// s) is spread over the whole grid and many small sources cost one pass.
__device__ __forceinline__ long long saturate_arc(const Params &p, int a) {
  const int r = __ldcg(p.res + a);
  if (r <= 0) return 0;
  p.res[a] = 0;
  atomicAdd(p.res + __ldg(p.par + a), r);
  atomic_add_ll(p.excess + __ldg(p.adj + a), r);
  return r;
}

__device__ __forceinline__ void ph_saturate(const Params &p) {
  const int nt = gridDim.x * blockDim.x, gt = blockIdx.x * blockDim.x + threadIdx.x;
  if (!p.src_off) {
    for (int i = 0; i < p.nsrc; i++) {
      if (p.inst_active && !p.inst_active[i]) continue;  // source i belongs to instance i
      const int s = p.srcs ? __ldg(p.srcs + i) : p.s;  // no list: the one source s
      const int beg = __ldg(p.off + s), end = __ldg(p.off + s + 1);
      long long sum = 0;
      for (int a = beg + gt; a < end; a += nt) sum += saturate_arc(p, a);
      agg_add_ll(p.excess + s, -sum);
    }
    return;
  }
  const int total = __ldg(p.src_off + p.nsrc);
  int cur = -1;  // source whose arcs this thread is summing
  long long sum = 0;
  for (int j = gt; j < total; j += nt) {
    int lo = 0, hi = p.nsrc;  // last i with src_off[i] <= j
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(p.src_off + mid) <= j) lo = mid;
      else hi = mid;
    }
    if (p.inst_active && !p.inst_active[lo]) continue;
    if (lo != cur) {
      if (sum) atomic_add_ll(p.excess + __ldg(p.srcs + cur), -sum);
      cur = lo;
      sum = 0;
    }
    const int s = __ldg(p.srcs + lo);
    sum += saturate_arc(p, __ldg(p.off + s) + (j - __ldg(p.src_off + lo)));
  }
  // threads of a warp that ended on the same source add once
  cg::coalesced_group g = cg::coalesced_threads();
  cg::coalesced_group same = cg::labeled_partition(g, cur);
  sum = cg::reduce(same, sum, cg::plus<long long>());
  if (same.thread_rank() == 0 && cur >= 0 && sum) atomic_add_ll(p.excess + __ldg(p.srcs + cur), -sum);
}

// Arc lookup of OnAdd_kernel (code/dyn_data.h:196-201), which scans the tail's
// adjacency for the head; here one probe of an open-addressing table keyed by
// (tail, head) (dmfd::ArcSlot, built once per solver by k_arc_table_build).
// A slot holds the key and the arc in one 16-byte line: a found update costs
// one DRAM sector (two when the probe crosses a sector) instead of a search of
// the tail's adjacency, and the line is only read.  Equal (tail, head) pairs
// in a CSR with duplicate arcs resolve to the last arc among them, as
// OnAdd_kernel's scan keeps the last match.  The lookup validates vertex ids,
// capacities and arcs; an arc named twice is found by the claim (ph_claim).

// Updates a thread looks up side by side: their probes are in flight together.
constexpr int kLookupBatch = 4;

__device__ __forceinline__ void ph_lookup(const Params &p) {
  const int nt = gridDim.x * blockDim.x, gt = spread_thread();
  for (int i0 = gt; i0 < p.k; i0 += kLookupBatch * nt) {
    int u[kLookupBatch], v[kLookupBatch], w[kLookupBatch], e[kLookupBatch];
    long long slot[kLookupBatch];
    bool on[kLookupBatch], pend[kLookupBatch];
#pragma unroll
    for (int j = 0; j < kLookupBatch; j++) {
      const int i = i0 + j * nt;
      on[j] = i < p.k;
      u[j] = on[j] ? __ldg(p.usrc + i) : 0;
      v[j] = on[j] ? __ldg(p.udst + i) : 0;
      w[j] = on[j] ? __ldg(p.uw + i) : 0;
    }
#pragma unroll
    for (int j = 0; j < kLookupBatch; j++) {
      e[j] = -1;
      pend[j] = false;
      if (!on[j]) continue;
      const int i = i0 + j * nt;
      p.uarc[i] = -1;
      if (u[j] < 0 || u[j] >= p.n || v[j] < 0 || v[j] >= p.n || w[j] < 0 || w[j] > kMaxUpdateCap) {
        set_err(p.ctrl, ERR_BAD_UPDATE, i);
        on[j] = false;
      } else if (u[j] == v[j]) {
        on[j] = false;  // ignored, as OnAdd_kernel does (code/dyn_data.h:194)
      } else {
        slot[j] = arc_slot0(u[j], v[j], p.nslots);
        pend[j] = true;
      }
    }
    // linear probing; the table always has an empty slot, so every probe
    // sequence ends (the bound only guards a corrupt table)
    for (long long probe = 0; probe < p.nslots; probe++) {
      ArcSlot s[kLookupBatch];
#pragma unroll
      for (int j = 0; j < kLookupBatch; j++)
        if (pend[j]) s[j] = load_slot(p.atab + slot[j]);
      bool any = false;
#pragma unroll
      for (int j = 0; j < kLookupBatch; j++) {
        if (!pend[j]) continue;
        if (s[j].tail == u[j] && s[j].head == v[j]) {
          e[j] = s[j].arc;
          pend[j] = false;
        } else if (s[j].tail == kEmptyTail) {
          pend[j] = false;
        } else {
          slot[j] = slot[j] + 1 == p.nslots ? 0 : slot[j] + 1;
          any = true;
        }
      }
      if (!any) break;
    }
#pragma unroll
    for (int j = 0; j < kLookupBatch; j++) {
      if (!on[j]) continue;
      const int i = i0 + j * nt;
      if (e[j] < 0) {
        set_err(p.ctrl, ERR_UNKNOWN_ARC, i);
        continue;
      }
      if (!p.caps_bounded && (long long)w[j] + cap_of(p, __ldg(p.par + e[j])) > INT_MAX) {
        set_err(p.ctrl, ERR_BAD_UPDATE, i);
        continue;
      }
      p.uarc[i] = e[j];
    }
  }
}

// Claim and capacity apply of OnAdd_kernel (code/dyn_data.h:202-205) in one
// pass: the new capacity goes in, the residual moves by the difference.  An
// arc whose residual went negative carries more flow than its new capacity;
// it is queued for the repair (ph_repair) rather than repaired here, so that a
// rejected batch only has to undo additions.  With the dead set kept, an arc
// from a dead tail to a live head that has residual now is queued for
// reopening.  In recompute mode only the capacity changes (update_kernel,
// code/dyn_data_bench.cu:300-322).
__device__ __forceinline__ void ph_claim_apply(const Params &p, bool residual) {
  const int nt = gridDim.x * blockDim.x, gt = spread_thread();
  const unsigned ep = (unsigned)p.epoch;
  for (int i = gt; i < p.k; i += nt) {
    const int e = __ldcg(p.uarc + i);
    if (e < 0) continue;
    const int w = __ldg(p.uw + i);
    bool du = false, dv = false;
    int u = 0, v = 0;
    if (residual && p.keep_dead) {
      u = __ldg(p.usrc + i);
      v = __ldg(p.udst + i);  // the lookup matched adj[e] == udst[i]
      du = __ldcg(p.dead + u) != 0;
      dv = __ldcg(p.dead + v) != 0;
    }
    const unsigned long long old = atomicExch(p.capx + e, cap_word(p, w));
    if ((unsigned)(old >> 32) == ep) {  // named twice: this update changes nothing
      p.uold[i] = -1;
      atomicCAS(&p.ctrl->dup_at, 0, i + 1);
      continue;
    }
    const int oc = (int)(unsigned)old;
    p.uold[i] = oc;
    const int delta = w - oc;
    if (!residual || !delta) continue;
    const int r = atomicAdd(p.res + e, delta) + delta;
    if (r < 0) append_bounded(p.wq[0], &p.ctrl->nrepair, i, p.n + 1);
    else if (r > 0 && du && !dv && !is_src(p, v)) append_bounded(p.aq, &p.ctrl->nreopen, i, p.n + 1);
  }
}

// A rejected batch: every update that changed its arc (the first to name it)
// puts the capacity and the residual back.
__device__ __forceinline__ void ph_unclaim(const Params &p, bool residual) {
  const int nt = gridDim.x * blockDim.x, gt = spread_thread();
  for (int i = gt; i < p.k; i += nt) {
    const int e = __ldcg(p.uarc + i);
    if (e < 0) continue;
    const int oc = __ldcg(p.uold + i);
    if (oc < 0) continue;
    p.capx[e] = (unsigned long long)(unsigned)oc;
    const int delta = __ldg(p.uw + i) - oc;
    if (residual && delta) atomicSub(p.res + e, delta);
  }
}

// Over-capacity repair of the queued arcs; replaces the O(m) sweeps
// incremental_kernel_20 / _22 (code/dyn_data.h:157-183): the overflow returns
// to the tail and is taken from the head.  Only an arc's own apply changed its
// residual, and at most one arc of a pair is negative (res(e) + res(partner) =
// cap(e) + cap(partner) >= 0), so the residual read here is the apply's.  Past
// the queue's capacity every update is looked at.
__device__ __forceinline__ void repair_update(const Params &p, int i) {
  const int e = __ldcg(p.uarc + i);
  if (e < 0) return;
  const int r = __ldcg(p.res + e);
  if (r >= 0) return;
  atomicAdd(p.res + e, -r);
  atomicAdd(p.res + __ldg(p.par + e), r);
  const int u = __ldg(p.usrc + i), v = __ldg(p.udst + i);
  atomic_add_ll(p.excess + u, -(long long)r);
  atomic_add_ll(p.excess + v, (long long)r);
  if (p.keep_dead) {  // the overflow returns to the tail: excess that can cover the head's deficit
    if (__ldcg(p.dead + v)) add_dead_cand(p, v);
    if (__ldcg(p.dead + u)) add_dead_cand(p, u);
  }
}

__device__ __forceinline__ void ph_repair(const Params &p, const Ctrl *sc) {
  const int nt = gridDim.x * blockDim.x, gt = spread_thread();
  const int nq = sc->nrepair;
  if (nq <= p.n + 1) {
    for (int j = gt; j < nq; j += nt) repair_update(p, __ldcg(p.wq[0] + j));
  } else {
    for (int i = gt; i < p.k; i += nt) repair_update(p, i);
  }
}

// Kept dead set D: after the last solve no residual arc leaves D (a complete
// BFS proved it, and pushes never enter D).  A batch can only add residual by
// raising a capacity; an updated arc u->v from D to a live v that has residual
// now is saturated at once: the flow goes to v (handled by the live solve) and
// u is charged with it (a deficit inside D, covered by the local repair).  D
// stays closed, so only the deficits inside it decide whether it stays dead.
__device__ __forceinline__ void reopen_update(const Params &p, int i) {
  const int e = __ldcg(p.uarc + i);
  if (e < 0) return;
  const int u = __ldg(p.usrc + i), v = __ldg(p.udst + i);  // adj[e] == udst[i]
  if (!__ldcg(p.dead + u) || __ldcg(p.dead + v) || is_src(p, v)) return;
  const int r = __ldcg(p.res + e);
  if (r <= 0) return;
  p.res[e] = 0;
  atomicAdd(p.res + __ldg(p.par + e), r);
  atomic_add_ll(p.excess + u, -(long long)r);
  atomic_add_ll(p.excess + v, (long long)r);
  add_dead_cand(p, u);
}

// The apply queued the updates that can need it (dead tail, live head,
// residual left); past the queue's capacity every update is looked at.
__device__ __forceinline__ void ph_reopen(const Params &p, const Ctrl *sc) {
  const int nt = gridDim.x * blockDim.x, gt = spread_thread();
  const int nq = sc->nreopen;
  if (nq <= p.n + 1) {
    for (int j = gt; j < nq; j += nt) reopen_update(p, __ldcg(p.aq + j));
  } else {
    for (int i = gt; i < p.k; i += nt) reopen_update(p, i);
  }
}

// Push-pull: an updated arc that now has residual from the source side A into
// the sink side B of the kept cut is saturated (the cut part of the fused
// incremental_kernel_20, code/dyn_pp.h:422-432, limited to touched arcs).
__device__ __forceinline__ void ph_cut_saturate(const Params &p) {
  const int nt = gridDim.x * blockDim.x, gt = spread_thread();
  for (int i = gt; i < p.k; i += nt) {
    int e = __ldcg(p.uarc + i);
    if (e < 0) continue;
    int u = __ldg(p.usrc + i), v = __ldg(p.udst + i);  // adj[e] == udst[i]
    if (is_term(p, u) || is_term(p, v)) continue;
    if (p.side[u] == 0 && p.side[v] == 1) {
      int r = __ldcg(p.res + e);
      if (r > 0) {
        p.res[e] = 0;
        atomicAdd(p.res + __ldg(p.par + e), r);
        atomic_add_ll(p.excess + u, -(long long)r);
        atomic_add_ll(p.excess + v, (long long)r);
      }
    }
  }
}

// ---- degree tiers ------------------------------------------------------------------
// Items of a vertex list (or all vertices when list == nullptr) in two passes:
// vertices of degree <= small_deg one per thread over the whole grid, then the
// larger ones (up to hub_deg; hubs are split into arc chunks and done by warps)
// one per tile.  `f(group, v)` does the work for one vertex.
// `pre(v)` is a per-vertex filter evaluated by one lane together with the degree
// read (a vertex it rejects costs one round of independent loads); it must not
// depend on writes of the current phase by other vertices' work.
template <int TILE, class F, class Pre>
__device__ __forceinline__ void for_tiered(const Params &p, LStats &ls, const int *list, int nn, F &&f, Pre &&pre) {
  const int nt = gridDim.x * blockDim.x;
  const int gt = list ? spread_thread(rot_threads()) : blockIdx.x * blockDim.x + threadIdx.x;
  for (int i = gt; i < nn; i += nt) {
    const int v = list ? __ldcg(list + i) : i;
    const bool keep = pre(v);
    if (deg_of(p, v) > p.small_deg || !keep) continue;
    ThreadGroup th;
    ItemTimer tm(p);
    f(th, v);
    tm.done(ls, v);
  }
  TileGroup<TILE> tg;
  if (!list) {
    // Sweep over every vertex: a tile checks TILE consecutive vertices per step
    // (one coalesced degree read, a ballot) and then works on the medium ones
    // it found, instead of one serial degree read per vertex.
    const int tiles = nt / TILE;
    for (int base = (int)((blockIdx.x * blockDim.x + threadIdx.x) / TILE) * TILE; base < nn; base += tiles * TILE) {
      const int v = base + tg.rank();
      const int d = v < nn ? deg_of(p, v) : 0;
      const bool keep = v < nn && pre(v);
      unsigned mask = tg.g.ballot(keep && d > p.small_deg && d <= p.hub_deg);
      while (mask) {  // tile-uniform
        const int vv = base + __ffs(mask) - 1;
        mask &= mask - 1;
        ItemTimer tm(p);
        f(tg, vv);
        tm.done(ls, vv);
      }
    }
    return;
  }
  const int gi = spread_group<TILE>(rot_tiles());
  for (int i = gi; i < nn; i += nt / TILE) {
    int v = 0, d = 0;
    if (tg.rank() == 0) {
      v = __ldcg(list + i);
      d = deg_of(p, v);
    }
    v = tg.g.shfl(v, 0);
    d = tg.g.shfl(d, 0);
    if (d <= p.small_deg || d > p.hub_deg) continue;  // tile-uniform
    ItemTimer tm(p);
    f(tg, v);
    tm.done(ls, v);
  }
}

template <int TILE, class F>
__device__ __forceinline__ void for_tiered(const Params &p, LStats &ls, const int *list, int nn, F &&f) {
  for_tiered<TILE>(p, ls, list, nn, f, [](int) { return true; });
}

// A hub (degree > hub_deg) enters a queue as ceil(deg / kChunk) consecutive
// items (v, c), chunk c covering arcs [off[v] + c*kChunk, +kChunk).  Every item
// is one warp's work, so a hub's adjacency is spread over many warps and no
// block-wide synchronisation is needed.
__device__ __forceinline__ int nchunks(int d) { return (d + kChunk - 1) / kChunk; }

__device__ __forceinline__ void append_hub(const Params &p, int2 *q, int *tail, int v) {
  const int k = nchunks(deg_of(p, v));
  const int base = atomicAdd(tail, k);
  for (int c = 0; c < k; c++) q[base + c] = make_int2(v, c);
}

__device__ __forceinline__ void chunk_range(const Params &p, int2 it, int &beg, int &end) {
  const int b0 = __ldg(p.off + it.x), e0 = __ldg(p.off + it.x + 1);
  beg = b0 + it.y * kChunk;
  end = min(e0, beg + kChunk);
}

// ---- global relabel ---------------------------------------------------------------

#define UNV (p.n + 1)

// Every vertex v of the call (instances outside the mask skipped) with its dead
// flag, f(v, dead): a thread takes vertices v0, v0 + nt, ... (coalesced across
// the warp), U at a time with their flag loads in flight together.  With a
// kept dead set nearly every vertex is dead and costs just that load, so the
// loop is bound by load latency unless several are outstanding.
template <int U, class F>
__device__ __forceinline__ void for_vertices(const Params &p, F &&f) {
  const int nt = gridDim.x * blockDim.x, gt = blockIdx.x * blockDim.x + threadIdx.x;
  for (int v0 = gt; v0 < p.n; v0 += U * nt) {
    unsigned char dd[U];
#pragma unroll
    for (int j = 0; j < U; j++) {
      const int v = v0 + j * nt;
      dd[j] = v < p.n ? __ldcg(p.dead + v) : 0;
    }
#pragma unroll
    for (int j = 0; j < U; j++) {
      const int v = v0 + j * nt;
      if (v < p.n && inst_on(p, v)) f(v, dd[j] != 0);
    }
  }
}

// Every live vertex of the call, f(v); returns how many dead vertices this
// thread passed over.  A warp takes windows of 512 vertices and first reads
// their dead flags as one 16-byte load per lane: a window with no live vertex
// (nearly all of them when a batch keeps the dead set) costs that load and a
// vote.  Other windows are walked like for_vertices (v = window + 32 j + lane,
// coalesced), the flags coming again from L2.  Calls with an instance mask
// take the plain per-vertex walk.
constexpr int kWindow = 512;

template <int U, class F>
__device__ __forceinline__ int for_live_vertices(const Params &p, F &&f) {
  int dead_seen = 0;
  if (p.inst_active) {
    for_vertices<U>(p, [&](int v, bool is_dead) {
      if (is_dead) dead_seen++;
      else f(v);
    });
    return dead_seen;
  }
  const int lane = threadIdx.x & 31;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long w0 = (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * kWindow; w0 < p.n;
       w0 += nw * kWindow) {
    const long long b = w0 + 16 * lane;  // this lane's 16 flags; b is 16-byte aligned
    bool all_dead;
    int mine;  // vertices < n among the 16
    if (b + 16 <= p.n) {
      const uint4 x = __ldcg(reinterpret_cast<const uint4 *>(p.dead + b));
      all_dead = (x.x & x.y & x.z & x.w) == 0x01010101u && (x.x | x.y | x.z | x.w) == 0x01010101u;
      mine = 16;
    } else {
      mine = b < p.n ? (int)(p.n - b) : 0;
      all_dead = true;
      for (int i = 0; i < mine; i++) all_dead &= __ldcg(p.dead + b + i) != 0;
    }
    if (__all_sync(0xffffffffu, all_dead)) {
      dead_seen += mine;
      continue;
    }
    for (int j0 = 0; j0 < kWindow / 32; j0 += U) {
      unsigned char dd[U];
#pragma unroll
      for (int j = 0; j < U; j++) {
        const long long v = w0 + (j0 + j) * 32 + lane;
        dd[j] = v < p.n ? __ldcg(p.dead + v) : 1;
      }
#pragma unroll
      for (int j = 0; j < U; j++) {
        const long long v = w0 + (j0 + j) * 32 + lane;
        if (v >= p.n) continue;
        if (dd[j]) dead_seen++;
        else f((int)v);
      }
    }
  }
  return dead_seen;
}

// Seeds (my_init_1, code/dyn_data.h:60-67): t and every deficit vertex other
// than s get height 0; all other live vertices become unvisited.  reset_dead
// revives every vertex (the first relabel of a solve that does not keep the
// dead set); count_kept adds the kept dead vertices to the dead-vertex
// statistic (first relabel of a batch that kept them).  Vertices of instances
// outside the call's mask are not touched at all: their labels and dead set
// stay as their own last solve left them.
__device__ __forceinline__ void ph_bfs_init(const Params &p, Slot *out, bool reset_dead, bool count_kept) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  Ctrl *c = p.ctrl;
  if (gt == 0) {
    c->act_q = 0;
    c->act_hq = 0;
    c->wtail[0] = c->whtail[0] = c->seen[0] = 0;  // written by push round 0
  }
  int pos = 0, kept = 0;
  long long unexpl = 0, seed_arcs = 0;
  auto seed = [&](int v) {
    long long ex = __ldcg(p.excess + v);
    int d = deg_of(p, v);
    if (d > p.hub_deg) {  // the hub's round totals start clean
      const int hid = __ldg(p.hub_base + v);
      p.hc_min[hid] = INT_MAX;
      p.hc_alloc[hid] = 0;
      p.hc_moved[hid] = 0;
      p.hc_done[hid] = 0;
    }
    if (is_snk(p, v) || (!is_src(p, v) && ex < 0)) {
      p.height[v] = 0;
      if (d > p.hub_deg) append_hub(p, p.fh[0], &out->hq, v);
      else append(p.fq[0], &out->q, v);
      seed_arcs += d;
    } else if (is_src(p, v)) {
      // Sources stay at height V and are never labelled: with a finite label
      // (the reference's BFS gives s its distance) a run of local relabels can
      // lift vertices above s while t is still reachable, excess drains back
      // into s, and the solve ends with an augmenting path open.  Excess that
      // cannot reach a sink or a deficit is parked on dead vertices instead,
      // so nothing ever has to return to s.
      p.height[v] = p.n;
    } else {
      p.height[v] = UNV;
      // a bottom-up level scans the arcs of every unvisited vertex, so the
      // direction heuristic weighs the frontier against all of them
      unexpl += d;
    }
    if (!is_term(p, v) && ex > 0) pos++;
  };
  if (reset_dead) {
    for_vertices<4>(p, [&](int v, bool is_dead) {
      if (is_dead) p.dead[v] = 0;
      seed(v);
    });
  } else {
    kept = for_live_vertices<4>(p, seed);
  }
  block_add_int(&c->pos_count, pos);
  block_add_ll(&c->unexplored, unexpl);
  block_add_ll(&out->arcs, seed_arcs);
  if (count_kept) block_add_ll((long long *)&c->st_dead, kept);
}

// Reserves `cnt` consecutive slots behind *tail for this thread with one atomic
// per group of threads that call it together.
__device__ __forceinline__ int reserve(int *tail, int cnt) {
  cg::coalesced_group g = cg::coalesced_threads();
  const int pre = cg::exclusive_scan(g, cnt, cg::plus<int>());
  int base = 0;
  if (g.thread_rank() == g.size() - 1) base = atomicAdd(tail, pre + cnt);
  return g.shfl(base, g.size() - 1) + pre;
}

struct VisitAcc {
  long long arcs = 0;
  int reached = 0;
};

__device__ __forceinline__ void bfs_visit(const Params &p, Slot *out, int nxt, int w, VisitAcc &acc) {
  int d = deg_of(p, w);
  const bool hub = d > p.hub_deg;
  if (hub) append_hub(p, p.fh[nxt], &out->hq, w);
  else append(p.fq[nxt], &out->q, w);
  acc.arcs += d;
  if (!is_term(p, w) && __ldcg(p.excess + w) > 0) {
    if (hub) append_hub(p, p.ah, &p.ctrl->act_hq, w);
    else append(p.aq, &p.ctrl->act_q, w);
    acc.reached++;
  }
}

// Counts go to the phase's own slot: a cross-phase counter would be read by a
// slow block after a fast block already added to it in the next phase.
__device__ __forceinline__ void flush_visits(const Params &p, Slot *out, VisitAcc &acc) {
  block_add_ll(&out->arcs, acc.arcs);
  block_add_int(&out->cnt, acc.reached);
}

// Top-down level (staticMaxFlow_kernel_11, code/dyn_data.h:72-87, run over the
// frontier queue instead of all V): x at level L labels w when arc w->x has
// residual, i.e. res[par[e]] > 0 for e = x->w.

// Arcs first, first+stride, ... < end of a frontier vertex, in register
// batches of kBatch so that the gathers of a batch are in flight together:
// heads, then head labels, then the reverse residuals, then the claims, then
// the claimed heads' degree and excess.
constexpr int kBatch = 8;   // arcs per lane per batch (a hub chunk is one batch)
constexpr int kTdBatch = 4;  // smaller for top-down, which keeps more state per arc
__device__ __forceinline__ void td_range(const Params &p, Slot *out, int nxt, int first, int end, int stride, int L,
                                         LStats &ls, VisitAcc &acc) {
  for (int a0 = first; a0 < end; a0 += kTdBatch * stride) {
    int w[kTdBatch];
    bool c[kTdBatch];
#pragma unroll
    for (int k = 0; k < kTdBatch; k++) {
      const int a = a0 + k * stride;
      w[k] = a < end ? __ldg(p.adj + a) : -1;
    }
#pragma unroll
    for (int k = 0; k < kTdBatch; k++) c[k] = w[k] >= 0 && __ldcg(p.height + w[k]) == UNV;
#pragma unroll
    for (int k = 0; k < kTdBatch; k++)
      if (c[k]) c[k] = __ldcg(p.res + __ldg(p.par + a0 + k * stride)) > 0;
#pragma unroll
    for (int k = 0; k < kTdBatch; k++)
      if (c[k]) c[k] = atomicCAS(p.height + w[k], UNV, L + 1) == UNV;
    int d[kTdBatch];
    long long ex[kTdBatch];
#pragma unroll
    for (int k = 0; k < kTdBatch; k++)
      if (c[k]) {
        d[k] = deg_of(p, w[k]);
        ex[k] = __ldcg(p.excess + w[k]);
      }
    // the batch's claimed heads go to the next frontier and, when active, to
    // the active list, with one reservation per list for the whole batch (a
    // large level claims hundreds of thousands of vertices: appends per arc
    // would serialise on the lists' tail counters)
    int nq = 0, na = 0;
    unsigned qmask = 0, amask = 0;
#pragma unroll
    for (int k = 0; k < kTdBatch; k++) {
      if (w[k] >= 0) ls.barcs++;
      if (!c[k]) continue;
      acc.arcs += d[k];
      const bool act = !is_term(p, w[k]) && ex[k] > 0;
      if (act) acc.reached++;
      if (d[k] > p.hub_deg) {
        append_hub(p, p.fh[nxt], &out->hq, w[k]);
        if (act) append_hub(p, p.ah, &p.ctrl->act_hq, w[k]);
      } else {
        qmask |= 1u << k;
        nq++;
        if (act) {
          amask |= 1u << k;
          na++;
        }
      }
    }
    if (nq) {
      int pos = reserve(&out->q, nq);
#pragma unroll
      for (int k = 0; k < kTdBatch; k++)
        if ((qmask >> k) & 1) p.fq[nxt][pos++] = w[k];
    }
    if (na) {
      int pos = reserve(&p.ctrl->act_q, na);
#pragma unroll
      for (int k = 0; k < kTdBatch; k++)
        if ((amask >> k) & 1) p.aq[pos++] = w[k];
    }
  }
}

template <int TILE>
__device__ __forceinline__ void ph_bfs_td(const Params &p, const Slot *in, Slot *out, int L, LStats &ls) {
  const int cur = L & 1, nxt = cur ^ 1;
  const int nn = ld_vol(&in->q), nh = ld_vol(&in->hq);
  VisitAcc acc;
  const int lane = threadIdx.x & 31, nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = spread_group<32>(); i < nh; i += nwarps) {
    int beg, end;
    const int2 it = __ldcg(p.fh[cur] + i);
    ItemTimer tm(p);
    chunk_range(p, it, beg, end);
    td_range(p, out, nxt, beg + lane, end, 32, L, ls, acc);
    tm.done(ls, it.x);
  }
  for_tiered<TILE>(p, ls, p.fq[cur], nn, [&](auto &g, int x) {
    const int beg = __ldg(p.off + x), end = __ldg(p.off + x + 1);
    td_range(p, out, nxt, beg + g.rank(), end, g.size(), L, ls, acc);
  });
  flush_visits(p, out, acc);
}

// Whether one of the arcs first, first+stride, ... < end (at most kBatch of them)
// has residual into a vertex labelled L; loads batched as in td_range.
__device__ __forceinline__ bool bu_batch(const Params &p, int first, int end, int stride, int L, LStats &ls) {
  int r[kBatch], w[kBatch];
#pragma unroll
  for (int k = 0; k < kBatch; k++) {
    const int a = first + k * stride;
    r[k] = a < end ? __ldcg(p.res + a) : 0;
    w[k] = a < end ? __ldg(p.adj + a) : -1;
  }
  bool hit = false;
#pragma unroll
  for (int k = 0; k < kBatch; k++) {
    if (w[k] >= 0) ls.barcs++;
    hit |= r[k] > 0 && __ldcg(p.height + w[k]) == L;
  }
  return hit;
}

// Bottom-up level: every unvisited vertex looks for a residual arc into level
// L and stops at the first one.  Hub chunks are searched by warps (the first
// chunk of a hub to succeed labels it); other vertices by a lane or a tile.
template <int TILE>
__device__ __forceinline__ void ph_bfs_bu(const Params &p, Slot *out, int L, LStats &ls) {
  const int nxt = (L & 1) ^ 1;
  VisitAcc acc;
  {
    TileGroup<32> wg;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = spread_group<32>(); i < p.nhch; i += nwarps) {
      const int2 it = __ldg(p.hch + i);
      int hv = 0;
      if (wg.rank() == 0) hv = __ldcg(p.height + it.x);
      if (wg.g.shfl(hv, 0) != UNV) continue;  // labelled already (possibly by another chunk)
      int beg, end;
      chunk_range(p, it, beg, end);
      const bool hit = bu_batch(p, beg + wg.rank(), end, 32, L, ls);  // 256 arcs = one batch
      if (wg.any(hit) && wg.rank() == 0 && atomicCAS(p.height + it.x, UNV, L + 1) == UNV)
        bfs_visit(p, out, nxt, it.x, acc);
    }
  }
  for_tiered<TILE>(p, ls, nullptr, p.n, [&](auto &g, int v) {
    if (__ldcg(p.height + v) != UNV) return;  // only v's group writes it in this phase
    const int beg = __ldg(p.off + v), end = __ldg(p.off + v + 1);
    bool found = false;
    for (int base = beg; base < end; base += kBatch * g.size()) {
      if (g.any(bu_batch(p, base + g.rank(), end, g.size(), L, ls))) {
        found = true;
        break;
      }
    }
    if (found && g.rank() == 0) {
      p.height[v] = L + 1;
      bfs_visit(p, out, nxt, v, acc);
    }
  }, [&](int v) { return __ldcg(p.height + v) == UNV; });
  flush_visits(p, out, acc);
}

// After the BFS: a complete BFS proves every unvisited vertex unreachable
// (dead for the rest of this solve; the reference gives them height V); an
// early-stopped BFS gives them the valid lower bound `floor`.
// Vertices already dead are skipped: they sit at height V and side 0 since the
// BFS that proved them dead.
__device__ __forceinline__ void ph_bfs_finalize(const Params &p, bool full, int floor_h, bool write_side) {
  int nd = 0;
  for_live_vertices<8>(p, [&](int v) {
    const int h = __ldcg(p.height + v);
    if (h == UNV) {
      if (full) {
        p.dead[v] = 1;
        p.height[v] = p.n;
        nd++;
      } else {
        p.height[v] = floor_h;
      }
    }
    if (write_side) p.side[v] = h < p.n ? 1 : 0;
  });
  block_add_ll((long long *)&p.ctrl->st_dead, nd);
}

// ---- local repair inside a kept dead set ------------------------------------------
// The batch changed the excess of some dead vertices (candidates in dq): the
// heads of repaired arcs got deficits, their tails the returned overflow, the
// tails of reopened arcs deficits.  The deficits are covered from excess inside
// the dead set, without reviving it, by pull-relabel rounds -- push-relabel run
// backwards, a deficit being moved instead of an excess.  A deficit y takes
// what it lacks over residual arcs x->y from dead in-neighbours holding excess
// (exactly the amount missing, so parked excess is not flooded around); it
// moves the rest to dead in-neighbours with a lower label, which pull in the
// next round; if some is still missing it relabels to 1 + the lowest label of
// its dead in-neighbours with residual and tries again next round.  Labels
// (dlab, tagged with the launch so nothing is reset; 0 until set, deficits
// start at 1) only rise, so deficits never cycle, and vertices can be passed
// through by many deficits.  Only dead vertices are pulled from, so every arc
// that gains residual (y->x) lies inside the dead set: it stays closed.
// Deficits left after kDeadRounds revive the dead vertices that can reach them
// (ph_dead_check, ph_dead_revive).

constexpr int kDeadRevived = 255;  // dlab label of a vertex the partial revival claimed

__device__ __forceinline__ unsigned dlab_tag(const Params &p) { return ((unsigned)p.epoch & 0xffffffu) << 8; }

// Label of dead vertex v in this launch's repair (0 when not set yet).
__device__ __forceinline__ int dead_label(const Params &p, int v) {
  const unsigned l = (unsigned)__ldcg(p.dlab + v);
  return (l & ~255u) == dlab_tag(p) ? (int)(l & 255u) : 0;
}

__device__ __forceinline__ void set_dead_label(const Params &p, int v, int h) {
  p.dlab[v] = (int)(dlab_tag(p) | (unsigned)(h < kDeadRevived - 1 ? h : kDeadRevived - 1));
}

// Seeds: the candidates with a deficit, at label 1.
__device__ __forceinline__ void ph_dead_seed(const Params &p, const Ctrl *sc, Slot *out) {
  const int nt = gridDim.x * blockDim.x, gt = spread_thread();
  Ctrl *c = p.ctrl;
  int seeds = 0;
  long long need = 0;
  const int nc = min(sc->dcand, p.n + 1);
  for (int i = gt; i < nc; i += nt) {
    const int v = __ldcg(p.dq + i);
    const long long ex = __ldcg(p.excess + v);
    if (ex >= 0 || is_term(p, v)) continue;
    set_dead_label(p, v, 1);
    append(p.fq[0], &out->q, v);
    seeds++;
    need -= ex;
  }
  block_add_int(&c->dseeds, seeds);
  block_add_ll(&c->dneed, need);
}

// One pull-relabel round: a warp per deficit of the list, lanes over its arcs.
// A vertex joins the next round's list once (stamp = this round's id).  A
// 32-arc step issues the supplier-side loads (the residual x->y, x's dead flag,
// excess and repair label) together once the arc's head and partner are
// known.  A row of at most 32 arcs is read once: pass 1 works on the loads of
// pass 0, with the residual pass 0 left on each arc (only y's warp changes the
// residual of an arc into y within a round).
struct PullArc {
  int x, pa, a, r, hx;
  long long ex;
  bool ok;  // residual x -> y from a dead vertex that is not a terminal
};

__device__ __forceinline__ PullArc pull_load(const Params &p, int a, int end) {
  PullArc q{-1, 0, a, 0, 0, 0, false};
  if (a < end) {
    q.x = __ldg(p.adj + a);
    q.pa = __ldg(p.par + a);
    q.r = __ldcg(p.res + q.pa);
    const bool dx = __ldcg(p.dead + q.x) != 0;
    q.ex = __ldcg(p.excess + q.x);
    q.hx = dead_label(p, q.x);
    q.ok = q.r > 0 && dx && !is_term(p, q.x);
  }
  return q;
}

// Pass 0 on one step: exact claims on parked excess (a claim bounded by an
// atomic on the supplier's excess; what another puller took first is handed
// back).  Returns what the warp moved.
__device__ __forceinline__ long long pull_excess(const Params &p, cg::thread_block_tile<32> &warp, PullArc &q,
                                                 long long need, LStats &ls) {
  const long long cand = q.ok && q.ex > 0 ? (q.ex < q.r ? q.ex : (long long)q.r) : 0;
  const long long pre = cg::exclusive_scan(warp, cand, cg::plus<long long>());
  long long take = need - pre;
  take = take < 0 ? 0 : (take > cand ? cand : take);
  if (take > 0) {
    const long long old = atomic_add_ll(p.excess + q.x, -take);
    if (old < take) {
      const long long back = take - (old > 0 ? old : 0);
      atomic_add_ll(p.excess + q.x, back);
      take -= back;
    }
    if (take > 0) {
      atomicSub(p.res + q.pa, (int)take);
      atomicAdd(p.res + q.a, (int)take);
      q.r -= (int)take;
      ls.pushes++;
    }
  }
  return cg::reduce(warp, take, cg::plus<long long>());
}

// Pass 1 on one step: the rest of the deficit moves to dead in-neighbours with
// a lower label (they pull it in the next round); hmin collects the labels of
// in-neighbours still residual.  Returns what the warp moved.
__device__ __forceinline__ long long pull_lower(const Params &p, cg::thread_block_tile<32> &warp, PullArc &q,
                                                long long need, int hy, int &hmin, int *nxt, int *ntail,
                                                unsigned round_id, LStats &ls) {
  long long cand = 0;
  if (q.ok && q.r > 0) {
    if (q.hx < hy) cand = q.r;
    else hmin = min(hmin, q.hx);
  }
  const long long pre = cg::exclusive_scan(warp, cand, cg::plus<long long>());
  long long take = need - pre;
  take = take < 0 ? 0 : (take > cand ? cand : take);
  if (take > 0) {
    const long long old = atomic_add_ll(p.excess + q.x, -take);
    if (old - take < 0 && atomicExch(p.stamp + q.x, (int)round_id) != (int)round_id) {
      append(nxt, ntail, q.x);  // x takes this part of the deficit over: it pulls next round
      append_bounded(p.dq, &p.ctrl->dcand, q.x, p.n + 1);  // and may keep it: the check looks at x
    }
    atomicSub(p.res + q.pa, (int)take);
    atomicAdd(p.res + q.a, (int)take);
    ls.pushes++;
  }
  if (cand > 0 && take < cand) hmin = min(hmin, q.hx);  // still residual
  return cg::reduce(warp, take, cg::plus<long long>());
}

// Warps first_warp, first_warp + nwarps, ... take the list's deficits; the next
// round's list is appended behind *ntail.
__device__ __forceinline__ void ph_dead_pull(const Params &p, const int *list, int nn, int *nxt, int *ntail,
                                             int first_warp, int nwarps, unsigned round_id, LStats &ls) {
  const int lane = threadIdx.x & 31;
  cg::thread_block_tile<32> warp = cg::tiled_partition<32>(cg::this_thread_block());
  for (int i = first_warp; i < nn; i += nwarps) {
    int y = 0;
    long long need = 0;
    if (lane == 0) {
      y = __ldcg(list + i);
      need = -__ldcg(p.excess + y);
    }
    y = warp.shfl(y, 0);
    need = warp.shfl(need, 0);
    if (need <= 0) continue;
    ItemTimer tm(p);
    const int hy = dead_label(p, y);
    const int beg = __ldg(p.off + y), end = __ldg(p.off + y + 1);
    long long got = 0;
    int hmin = INT_MAX;  // lowest label over the dead in-neighbours still residual
    if (end - beg <= 32) {
      PullArc q = pull_load(p, beg + lane, end);
      if (q.x >= 0) ls.arcs++;
      long long mv = pull_excess(p, warp, q, need, ls);
      need -= mv;
      got += mv;
      if (need > 0) {
        mv = pull_lower(p, warp, q, need, hy, hmin, nxt, ntail, round_id, ls);
        need -= mv;
        got += mv;
      }
    } else {
      // two steps' loads in flight at a time, starting at the row's cursor:
      // where the last pass 0 of this deficit was satisfied.  A hub deficit
      // that comes back batch after batch would otherwise rescan the in-arcs
      // whose suppliers it drained earlier (at R-MAT 24 the longest item of a
      // round, a hub of 60-165 k in-arcs, grew from 90 us to 550 us over 16
      // batches, and every round waits for it).
      const int deg = end - beg;
      int cur = p.pcur ? __ldcg(p.pcur + y) : 0;
      cur = (cur < 0 || cur >= deg) ? 0 : (cur & ~31);
      int stop = -1;
      for (int pass = 0; pass < 2 && need > 0; pass++) {
        for (int seg = 0; seg < 2 && need > 0; seg++) {
          const int sb = seg == 0 ? beg + cur : beg, se = seg == 0 ? end : beg + cur;
          for (int a0 = sb; a0 < se && need > 0; a0 += 64) {
            PullArc q0 = pull_load(p, a0 + lane, se);
            PullArc q1 = pull_load(p, a0 + 32 + lane, se);
            ls.arcs += (q0.x >= 0) + (q1.x >= 0);
            long long mv = pass == 0 ? pull_excess(p, warp, q0, need, ls)
                                     : pull_lower(p, warp, q0, need, hy, hmin, nxt, ntail, round_id, ls);
            need -= mv;
            got += mv;
            if (pass == 0 && need <= 0) stop = a0;
            if (need > 0 && a0 + 32 < se) {
              mv = pass == 0 ? pull_excess(p, warp, q1, need, ls)
                             : pull_lower(p, warp, q1, need, hy, hmin, nxt, ntail, round_id, ls);
              need -= mv;
              got += mv;
              if (pass == 0 && need <= 0) stop = a0 + 32;
            }
          }
        }
      }
      if (p.pcur && lane == 0 && stop >= 0) p.pcur[y] = stop - beg;
    }
    if (need > 0) {  // relabel and try again next round (nowhere to go: stays for the check)
      hmin = cg::reduce(warp, hmin, cg::less<int>());
      if (lane == 0 && hmin != INT_MAX) {
        set_dead_label(p, y, hmin + 1);
        ls.relabels++;
        if (atomicExch(p.stamp + y, (int)round_id) != (int)round_id) append(nxt, ntail, y);
      }
    }
    if (lane == 0 && got) atomic_add_ll(p.excess + y, got);
    tm.done(ls, y);
  }
}

// Pull rounds from round r0 on, in the calling block alone, once the list is
// short (at most kPullTail deficits): a block barrier between rounds instead of
// a grid barrier, at most kPullTailRounds of them.  Round r uses id round_base + (r - r0) + 1; the caller
// reserves the ids of every round up to kDeadRounds.  Deficits still open at the
// end are found by the dead check like any other.
constexpr int kPullTail = 64;
// Block rounds at most: a deficit still bouncing after them has no excess
// within reach inside the dead set (it relabels by one per round); the check
// revives it.
constexpr int kPullTailRounds = 6;

__device__ __forceinline__ void pull_tail_rounds(const Params &p, int r0, int nn, unsigned round_base, LStats &ls) {
  __shared__ int s_tail;
  const int r_end = min(kDeadRounds, r0 + kPullTailRounds);
  for (int r = r0; r < r_end && nn > 0; r++) {
    if (threadIdx.x == 0) s_tail = 0;
    __syncthreads();
    ph_dead_pull(p, p.fq[r & 1], nn, p.fq[(r + 1) & 1], &s_tail, threadIdx.x >> 5, blockDim.x >> 5,
                 round_base + (unsigned)(r - r0) + 1, ls);
    __syncthreads();
    nn = s_tail;
    __syncthreads();
  }
}

// Claims dead vertex v for the partial revival of this launch.
__device__ __forceinline__ bool revive_claim(const Params &p, int v) {
  const int tag = (int)(dlab_tag(p) | (unsigned)kDeadRevived);
  const int old = __ldcg(p.dlab + v);
  if (old == tag) return false;
  return atomicCAS(p.dlab + v, old, tag) == old;
}

// Counts the deficits left inside the dead set: the candidate list holds every
// dead vertex whose excess the batch or the pulls lowered (a vertex may appear
// more than once; the claim counts it once); past its capacity every vertex is
// looked at.  Each deficit found is revived (made live: it is a seed of the
// global relabels) and starts the partial revival.
__device__ __forceinline__ void ph_dead_check(const Params &p, const Ctrl *sc, Slot *out) {
  int left = 0;
  auto check = [&](int v, bool is_dead) {
    if (is_dead && !is_term(p, v) && __ldcg(p.excess + v) < 0 && revive_claim(p, v)) {
      left++;
      p.dead[v] = 0;
      if (deg_of(p, v) > p.hub_deg) append_hub(p, p.fh[0], &out->hq, v);
      else append(p.fq[0], &out->q, v);
    }
  };
  const int nc = sc->dcand;
  if (nc <= p.n + 1) {
    const int nt = gridDim.x * blockDim.x, gt = spread_thread();
    for (int i = gt; i < nc; i += nt) {
      const int v = __ldcg(p.dq + i);
      check(v, __ldcg(p.dead + v) != 0);
    }
  } else {
    for_vertices<8>(p, check);
  }
  block_add_int(&p.ctrl->dleft, left);
}

// Partial revival, one level: every dead vertex with a residual arc into the
// frontier can reach a revived deficit, so it is revived too (made live).  Run
// to completion, the dead vertices left cannot reach any revived vertex, and
// the dead set stays closed.  The arcs scanned go to out->arcs (the caller
// gives up past a budget and revives every vertex instead).
__device__ __forceinline__ void dead_revive_range(const Params &p, Slot *out, int nxt, int first, int end,
                                                  int stride, LStats &ls, long long &scanned, int &revived) {
  for (int a = first; a < end; a += stride) {
    const int x = __ldg(p.adj + a);
    ls.barcs++;
    scanned++;
    if (__ldcg(p.res + __ldg(p.par + a)) <= 0 || !__ldcg(p.dead + x) || is_term(p, x)) continue;
    if (!revive_claim(p, x)) continue;
    p.dead[x] = 0;
    revived++;
    if (deg_of(p, x) > p.hub_deg) append_hub(p, p.fh[nxt], &out->hq, x);
    else append(p.fq[nxt], &out->q, x);
  }
}

template <int TILE>
__device__ __forceinline__ void ph_dead_revive(const Params &p, const Slot *in, Slot *out, int L, LStats &ls) {
  const int cur = L & 1, nxt = cur ^ 1;
  const int nn = ld_vol(&in->q), nh = ld_vol(&in->hq);
  long long scanned = 0;
  int revived = 0;
  const int lane = threadIdx.x & 31, nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = spread_group<32>(); i < nh; i += nwarps) {
    int beg, end;
    const int2 it = __ldcg(p.fh[cur] + i);
    chunk_range(p, it, beg, end);
    dead_revive_range(p, out, nxt, beg + lane, end, 32, ls, scanned, revived);
  }
  for_tiered<TILE>(p, ls, p.fq[cur], nn, [&](auto &g, int z) {
    const int beg = __ldg(p.off + z), end = __ldg(p.off + z + 1);
    dead_revive_range(p, out, nxt, beg + g.rank(), end, g.size(), ls, scanned, revived);
  });
  block_add_ll(&out->arcs, scanned);
  block_add_ll((long long *)&p.ctrl->st_revived, revived);
}

// ---- push rounds ---------------------------------------------------------------
// Round r reads the worklists of round r-1 (the BFS active lists for r = 0) and
// appends to buffers r&1 with tails wtail/whtail[r%3]; tails are triple-buffered
// for the same reason as the phase slots.

__device__ __forceinline__ void enqueue(const Params &p, int r, unsigned round_id, int v) {
  if (atomicExch(p.stamp + v, (int)round_id) == (int)round_id) return;
  if (deg_of(p, v) > p.hub_deg) append_hub(p, p.wh[r & 1], &p.ctrl->whtail[r % 3], v);
  else append(p.wq[r & 1], &p.ctrl->wtail[r % 3], v);
}

// Adds d to the head's excess and returns the old value.  Pushes into the one
// sink of a single-instance solve are summed per thread instead and added once
// per block when the push phase ends (sink_flush): a high in-degree sink takes
// thousands of pushes a round, which would serialise on its excess word, and a
// terminal is never queued, so its old value is not needed.
__device__ __forceinline__ long long push_excess(const Params &p, int w, int d, LStats &ls) {
  if (!p.role && w == p.t) {
    ls.to_sink += d;
    return 0;
  }
  return atomic_add_ll(p.excess + w, d);
}

// Every thread of the block calls it at the end of the push phase.
__device__ __forceinline__ void sink_flush(const Params &p, LStats &ls) {
  if (p.role) return;  // uniform
  block_add_ll(p.excess + p.t, ls.to_sink);
  ls.to_sink = 0;
}

__device__ __forceinline__ void push_arc(const Params &p, int a, int w, int d, int r, unsigned round_id, bool enq,
                                         LStats &ls) {
  atomicSub(p.res + a, d);
  atomicAdd(p.res + __ldg(p.par + a), d);
  long long old = push_excess(p, w, d, ls);
  ls.pushes++;
  if (enq && !is_term(p, w) && old + d > 0) enqueue(p, r, round_id, w);
}

// Arcs a lane handles together in a tile discharge.
constexpr int kPushBatch = 4;


// Queues the heads x[k] marked in `cand` for round r+1 (each at most once per
// round, by its stamp): all stamp exchanges in flight together, then all degree
// reads, then one reservation for the non-hub heads (hubs go to the chunk queue).
template <int K>
__device__ __forceinline__ void enqueue_batch(const Params &p, const int (&x)[K], unsigned cand, int r,
                                              unsigned round_id) {
  unsigned keep = 0;
#pragma unroll
  for (int k = 0; k < K; k++)
    if ((cand >> k) & 1)
      if (atomicExch(p.stamp + x[k], (int)round_id) != (int)round_id) keep |= 1u << k;
  if (!keep) return;
  int dg[K];
#pragma unroll
  for (int k = 0; k < K; k++) dg[k] = ((keep >> k) & 1) ? deg_of(p, x[k]) : 0;
  int cnt = 0;
  unsigned small = 0;
#pragma unroll
  for (int k = 0; k < K; k++)
    if ((keep >> k) & 1) {
      if (dg[k] > p.hub_deg) {
        append_hub(p, p.wh[r & 1], &p.ctrl->whtail[r % 3], x[k]);
      } else {
        small |= 1u << k;
        cnt++;
      }
    }
  if (!cnt) return;
  int pos = reserve(&p.ctrl->wtail[r % 3], cnt);
  int *q = p.wq[r & 1];
#pragma unroll
  for (int k = 0; k < K; k++)
    if ((small >> k) & 1) q[pos++] = x[k];
}

// Pushes d[k] > 0 units over arcs a[k] into heads w[k] (one lane's batch): the
// residual and excess atomics of all arcs are in flight together, then the
// partner residuals; heads whose excess became positive are queued (enq).
template <int K>
__device__ __forceinline__ void push_batch(const Params &p, const int (&a)[K], const int (&w)[K], const int (&d)[K],
                                           int r, unsigned round_id, bool enq, LStats &ls) {
  int pk[K];  // partner arcs, loaded while the atomics below are in flight
#pragma unroll
  for (int k = 0; k < K; k++) pk[k] = d[k] > 0 ? __ldg(p.par + a[k]) : 0;
  long long old[K];
#pragma unroll
  for (int k = 0; k < K; k++)
    if (d[k] > 0) {
      atomicSub(p.res + a[k], d[k]);
      old[k] = push_excess(p, w[k], d[k], ls);
    }
  unsigned cand = 0;
#pragma unroll
  for (int k = 0; k < K; k++)
    if (d[k] > 0) {
      atomicAdd(p.res + pk[k], d[k]);
      ls.pushes++;
      if (enq && !is_term(p, w[k]) && old[k] + d[k] > 0) cand |= 1u << k;
    }
  if (cand) enqueue_batch<K>(p, w, cand, r, round_id);
}

// Adjacency bound of the register-resident thread discharge below.
constexpr int kSmallMax = 8;

// Discharge of a vertex of degree <= kSmallMax by one thread, with the same
// push/relabel rule as discharge() but laid out for latency: per cycle the
// residuals and head heights of all arcs are loaded together, the pushes are
// decided in registers (excess spread over the admissible arcs in arc order),
// and every atomic of the cycle is in flight before any result is used; the
// heads that became active are deduplicated by their stamps together and
// appended with one reservation.  A head height may be one load old when it is
// used (a concurrent relabel only raises it), which can leave a label above
// the exact distance for a while; labels only steer the pushes -- dead
// vertices and termination are decided by the exact BFS of each relabel.
__device__ __forceinline__ void discharge_small(const Params &p, int v, int beg, int deg, long long ex0, int h, int r,
                                unsigned round_id, bool enq, LStats &ls) {
  int rr[kSmallMax], w[kSmallMax], hw[kSmallMax];
#pragma unroll
  for (int k = 0; k < kSmallMax; k++) {
    rr[k] = k < deg ? __ldcg(p.res + beg + k) : 0;
    w[k] = k < deg ? __ldg(p.adj + beg + k) : 0;
  }
  unsigned cand = 0;  // bit k: head k may have become active; bit kSmallMax: v itself
  long long ex = ex0;
  for (int cyc = 0; cyc < p.cycles && ex > 0 && h < p.n; cyc++) {
    if (cyc > 0) {
#pragma unroll
      for (int k = 0; k < kSmallMax; k++)
        if (k < deg) rr[k] = __ldcg(p.res + beg + k);
    }
#pragma unroll
    for (int k = 0; k < kSmallMax; k++) hw[k] = k < deg ? __ldcg(p.height + w[k]) : INT_MAX;
    ls.arcs += deg;
    int dd[kSmallMax];
    long long left = ex;
#pragma unroll
    for (int k = 0; k < kSmallMax; k++) {
      dd[k] = 0;
      if (rr[k] > 0 && hw[k] < h && left > 0) {
        dd[k] = (int)(rr[k] < left ? rr[k] : left);
        left -= dd[k];
      }
    }
    int pk[kSmallMax];  // partner arcs, loaded while the atomics below are in flight
#pragma unroll
    for (int k = 0; k < kSmallMax; k++) pk[k] = dd[k] > 0 ? __ldg(p.par + beg + k) : 0;
    long long old[kSmallMax];
#pragma unroll
    for (int k = 0; k < kSmallMax; k++)
      if (dd[k] > 0) {
        atomicSub(p.res + beg + k, dd[k]);
        old[k] = push_excess(p, w[k], dd[k], ls);
      }
#pragma unroll
    for (int k = 0; k < kSmallMax; k++)
      if (dd[k] > 0) {
        atomicAdd(p.res + pk[k], dd[k]);
        rr[k] -= dd[k];
        ls.pushes++;
        if (enq && !is_term(p, w[k]) && old[k] + dd[k] > 0) cand |= 1u << k;
      }
    ex = left;
    if (ex > 0) {  // every admissible arc is saturated: relabel
      int mh = INT_MAX;
#pragma unroll
      for (int k = 0; k < kSmallMax; k++)
        if (rr[k] > 0) mh = min(mh, hw[k]);
      h = mh >= p.n ? p.n : mh + 1;
      p.height[v] = h;
      ls.relabels++;
    }
  }
  if (ex0 != ex) atomic_add_ll(p.excess + v, ex - ex0);
  if (enq && ex > 0 && h < p.n) cand |= 1u << kSmallMax;
  if (!cand) return;
  int x[kSmallMax + 1];
#pragma unroll
  for (int k = 0; k < kSmallMax; k++) x[k] = w[k];
  x[kSmallMax] = v;
  enqueue_batch<kSmallMax + 1>(p, x, cand, r, round_id);
}

// Discharge of a non-hub v by a lane or a tile: up to `cycles` rounds of
// push-then-relabel, the push/relabel of staticMaxFlow_kernel_14
// (code/dyn_data.h:89-131) with every admissible arc (head below h) used per
// round instead of only the lowest one.
//  * adjacency within the group width: one load per lane, the excess is split
//    over the admissible arcs in arc order by a group prefix sum;
//  * longer adjacency: pass 1 has every lane sum the admissible residual and the
//    minimum non-admissible height over its strided arcs (independent loads); a
//    group prefix sum turns the sums into per-lane budgets; pass 2 pushes each
//    lane's budget greedily.
// When every admissible arc was saturated and excess is left, h becomes
// 1 + the minimum height over the arcs still residual.  Concurrent relabels only
// raise heights, so a pass-2 arc that lost admissibility is skipped and the
// round is retried instead of relabelled.
template <class G>
__device__ __forceinline__ void discharge(G &g, const Params &p, int v, int r, unsigned round_id, bool enq, LStats &ls,
                          int *seen) {
  long long ex0;
  int h;
  // one read, broadcast: concurrent pushes may change excess[v] meanwhile
  if constexpr (G::size() == 1) {
    ex0 = __ldcg(p.excess + v);
    h = __ldcg(p.height + v);
  } else {
    long long e = 0;
    int hh = 0;
    if (g.rank() == 0) {
      e = __ldcg(p.excess + v);
      hh = __ldcg(p.height + v);
    }
    ex0 = g.g.shfl(e, 0);
    h = g.g.shfl(hh, 0);
  }
  if (!(ex0 > 0 && h < p.n) || is_term(p, v)) return;
  if (g.rank() == 0) {
    ls.visits++;
    if (seen) (*seen)++;
  }
  long long ex = ex0;
  const int beg = __ldg(p.off + v), end = __ldg(p.off + v + 1);
  constexpr int S = G::size();
  if constexpr (S == 1) {
    if (end - beg <= kSmallMax) {
      discharge_small(p, v, beg, end - beg, ex0, h, r, round_id, enq, ls);
      return;
    }
  }
  for (int cyc = 0; cyc < p.cycles && ex > 0 && h < p.n; cyc++) {
    if (end - beg <= S) {
      const int a = beg + g.rank();
      int rr = 0, w = -1, hw = INT_MAX;
      if (a < end) {
        rr = __ldcg(p.res + a);
        if (rr > 0) {
          w = __ldg(p.adj + a);
          hw = __ldcg(p.height + w);
        }
        ls.arcs++;
      }
      const bool adm = rr > 0 && hw < h;
      long long tot;
      const long long pre = g.scan(adm ? (long long)rr : 0ll, tot);
      int d = 0;
      if (adm) {
        long long left = ex - pre;
        d = left <= 0 ? 0 : (left < rr ? (int)left : rr);
      }
      if (d > 0) push_arc(p, a, w, d, r, round_id, enq, ls);
      ex -= (tot < ex ? tot : ex);
      if (ex > 0) {
        const int mh = g.min_all(rr > 0 && !(adm && d == rr) ? hw : INT_MAX);
        h = mh >= p.n ? p.n : mh + 1;
        if (g.rank() == 0) {
          p.height[v] = h;
          ls.relabels++;
        }
      }
      continue;
    }
    // pass 1 (batches of kPushBatch arcs a lane: heads and residuals, then head
    // heights, each batch's loads in flight together)
    long long tsum = 0;
    int tmin = INT_MAX;
    for (int a0 = beg + g.rank(); a0 < end; a0 += kPushBatch * S) {
      int rr[kPushBatch], w[kPushBatch];
#pragma unroll
      for (int k = 0; k < kPushBatch; k++) {
        const int a = a0 + k * S;
        rr[k] = a < end ? __ldcg(p.res + a) : 0;
        w[k] = a < end ? __ldg(p.adj + a) : 0;
      }
#pragma unroll
      for (int k = 0; k < kPushBatch; k++)
        if (rr[k] > 0) {
          const int hw = __ldcg(p.height + w[k]);
          if (hw < h) tsum += rr[k];
          else tmin = min(tmin, hw);
        }
    }
    ls.arcs += (unsigned long long)((end - beg - g.rank() + S - 1) / S);
    long long tot;
    const long long pre = g.scan(tsum, tot);
    // pass 2: heights reread (a concurrent relabel may have made an arc
    // inadmissible), the lane's budget spread greedily, each batch's pushes in
    // flight together
    long long budget = ex - pre;
    budget = budget < 0 ? 0 : (budget > tsum ? tsum : budget);
    long long done = 0;
    for (int a0 = beg + g.rank(); a0 < end && budget > 0; a0 += kPushBatch * S) {
      int aa[kPushBatch], rr[kPushBatch], w[kPushBatch], dd[kPushBatch];
#pragma unroll
      for (int k = 0; k < kPushBatch; k++) {
        aa[k] = a0 + k * S;
        rr[k] = aa[k] < end ? __ldcg(p.res + aa[k]) : 0;
        w[k] = aa[k] < end ? __ldg(p.adj + aa[k]) : 0;
      }
      int hw[kPushBatch];
#pragma unroll
      for (int k = 0; k < kPushBatch; k++) hw[k] = rr[k] > 0 ? __ldcg(p.height + w[k]) : INT_MAX;
#pragma unroll
      for (int k = 0; k < kPushBatch; k++) {
        dd[k] = 0;
        if (hw[k] < h && budget > 0) {
          dd[k] = (int)(rr[k] < budget ? rr[k] : budget);
          budget -= dd[k];
          done += dd[k];
        }
      }
      push_batch<kPushBatch>(p, aa, w, dd, r, round_id, enq, ls);
    }
    const long long moved = g.sum_all(done);
    ex -= moved;
    if (ex > 0 && moved == tot) {  // all admissible arcs saturated: relabel
      const int mh = g.min_all(tmin);
      h = mh >= p.n ? p.n : mh + 1;
      if (g.rank() == 0) {
        p.height[v] = h;
        ls.relabels++;
      }
    }
  }
  if (g.rank() == 0) {
    if (ex0 != ex) atomic_add_ll(p.excess + v, ex - ex0);
    if (enq && ex > 0 && h < p.n) enqueue(p, r, round_id, v);
  }
}

// Inputs of push round r: non-hub vertices and hub chunks.
struct RoundIn {
  const int *nlist;
  int nn;
  const int2 *hlist;
  int nh;
};

// dph: a round of the local repair inside the dead set (always worklist-driven:
// a topology sweep would discharge live vertices too).
__device__ __forceinline__ RoundIn round_inputs(const Params &p, const Ctrl *c, int r, bool dph) {
  RoundIn in;
  if (p.variant == DMF_VARIANT_TOPO && !dph) {
    in.nlist = nullptr;
    in.nn = p.n;
    in.hlist = p.hch;
    in.nh = p.nhch;
  } else if (r == 0) {
    in.nlist = p.aq;
    in.nn = ld_vol(&c->act_q);
    in.hlist = p.ah;
    in.nh = ld_vol(&c->act_hq);
  } else {
    in.nlist = p.wq[(r - 1) & 1];
    in.nn = ld_vol(&c->wtail[(r - 1) % 3]);
    in.hlist = p.wh[(r - 1) & 1];
    in.nh = ld_vol(&c->whtail[(r - 1) % 3]);
  }
  return in;
}

// Push round, phase 1: non-hub vertices are discharged completely; every hub
// chunk sums its admissible residual, adds its minimum non-admissible head
// height to the hub's, and pushes its share of the hub's excess.
template <int TILE, int BLOCK>
__device__ __forceinline__ void ph_push1(const Params &p, const RoundIn &in, int r, unsigned round_id, unsigned gepoch, LStats &ls,
                         typename BlockGroup<BLOCK>::Temp &btmp, int *bci, long long *bcl, bool dph) {
  Ctrl *c = p.ctrl;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const bool topo = p.variant == DMF_VARIANT_TOPO && !dph;
  if (gt == 0) {
    if (r == 0) {  // read during the BFS just finished; cleared for the next one
      c->pos_count = 0;
      c->unexplored = 0;
    }
    c->wtail[(r + 1) % 3] = c->whtail[(r + 1) % 3] = c->seen[(r + 1) % 3] = 0;
  }
  {
    // Hub chunks: scan, then claim a share of the hub's excess and push it from
    // the scan's registers, in one phase.  A hub's excess only grows during the
    // phase (its own pushes leave it in phase 2), so each chunk's read of it at
    // the start of its item is at most the hub's excess at the end of the
    // phase, and the shares claimed in arc-chunk order by the atomic on the
    // hub's allocation never add up to more than that.
    TileGroup<32> wg;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = spread_group<32>(); i < in.nh; i += nwarps) {
      const int2 it = __ldcg(in.hlist + i);
      const int v = it.x;
      ItemTimer tmr(p);
      int hh = 0;
      long long ex_start = 0;  // the hub's excess as the phase found it
      if (wg.rank() == 0) {
        hh = __ldcg(p.height + v);
        ex_start = __ldcg(p.excess + v);
      }
      const int h = wg.g.shfl(hh, 0);
      const bool has_ex = wg.g.shfl(ex_start, 0) > 0;
      const int hid = __ldg(p.hub_base + v), cidx = hid + it.y;
      const unsigned long long key = ((unsigned long long)gepoch << 32) | (unsigned)h;
      unsigned long long mk = 0;
      if (wg.rank() == 0) mk = __ldcg(p.chunk_mark + cidx);
      mk = wg.g.shfl(mk, 0);
      // A hub without excess (topology rounds sweep every hub) needs nothing.
      // Every chunk that does look counts itself: the hub is relabelled only
      // when all its chunks contributed to the minimum head height.
      if (!has_ex || h >= p.n || is_term(p, v) || !inst_on(p, v)) {
      } else if (mk == key) {  // exhausted at this height: only its minimum head height matters
        if (wg.rank() == 0) {
          const int tm = __ldcg(p.chunk_tmin + cidx);
          if (tm != INT_MAX) atomicMin(p.hc_min + hid, tm);
          atomicAdd(p.hc_done + hid, 1);
        }
      } else {
        int beg, end;
        chunk_range(p, it, beg, end);
        int aa[kBatch], rr[kBatch], w[kBatch], hw[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; k++) {
          aa[k] = beg + wg.rank() + 32 * k;
          rr[k] = aa[k] < end ? __ldcg(p.res + aa[k]) : 0;
          w[k] = aa[k] < end ? __ldg(p.adj + aa[k]) : 0;
        }
#pragma unroll
        for (int k = 0; k < kBatch; k++) hw[k] = rr[k] > 0 ? __ldcg(p.height + w[k]) : INT_MAX;
        long long tsum = 0;
        int tmin = INT_MAX;
#pragma unroll
        for (int k = 0; k < kBatch; k++) {
          if (rr[k] > 0) {
            if (hw[k] < h) tsum += rr[k];
            else tmin = min(tmin, hw[k]);
          }
        }
        ls.arcs += kBatch;
        long long ts;
        const long long pre = wg.scan(tsum, ts);
        const int tm = wg.min_all(tmin);
        long long cb = 0;  // this chunk's share of the hub's excess
        if (wg.rank() == 0) {
          if (tm != INT_MAX) atomicMin(p.hc_min + hid, tm);
          atomicAdd(p.hc_done + hid, 1);
          if (ts > 0) {
            const long long old = atomic_add_ll(p.hc_alloc + hid, ts);
            cb = ex_start - old;
            cb = cb < 0 ? 0 : (cb > ts ? ts : cb);
          }
        }
        cb = wg.g.shfl(cb, 0);
        long long moved = 0;
        if (cb > 0) {  // warp-uniform
          long long budget = cb - pre;
          budget = budget < 0 ? 0 : (budget > tsum ? tsum : budget);
          long long done = 0;
          int dd[kBatch];
#pragma unroll
          for (int k = 0; k < kBatch; k++) {
            dd[k] = 0;
            if (rr[k] > 0 && hw[k] < h && budget > 0) {
              dd[k] = (int)(rr[k] < budget ? rr[k] : budget);
              budget -= dd[k];
              done += dd[k];
            }
          }
          push_batch<kBatch>(p, aa, w, dd, r, round_id, !topo, ls);
          moved = wg.sum_all(done);
          if (wg.rank() == 0 && moved) atomic_add_ll(p.hc_moved + hid, moved);
        }
        // no admissible arc left in the chunk at this height: skip it until the
        // hub's height or the relabel epoch changes
        if (wg.rank() == 0 && moved == ts) {
          p.chunk_mark[cidx] = key;
          p.chunk_tmin[cidx] = tm;
        }
      }
      tmr.done(ls, v);
    }
  }
  int seen = 0;
  // topology rounds sweep every vertex: only those with excess need a look
  for_tiered<TILE>(
      p, ls, in.nlist, in.nn,
      [&](auto &g, int v) { discharge(g, p, v, r, round_id, !topo, ls, topo ? &seen : nullptr); },
      [&](int v) { return !topo || (__ldcg(p.excess + v) > 0 && inst_on(p, v)); });
  if (topo) agg_add_int(&c->seen[r % 3], seen);
  sink_flush(p, ls);
}

// Push round, phase 2 (hubs): per hub (its first chunk), the moved total leaves
// its excess; when all of the hub's admissible residual was pushed and excess is
// left, the hub is relabelled to 1 + the minimum non-admissible height; a hub
// with excess left is queued for the next round.  The hub's totals are reset.
__device__ __forceinline__ void ph_push3(const Params &p, const RoundIn &in, int r, unsigned round_id, LStats &ls,
                                         bool dph) {
  const int nt = gridDim.x * blockDim.x;
  const bool topo = p.variant == DMF_VARIANT_TOPO && !dph;
  int seen = 0;
  for (int i = spread_thread(); i < in.nh; i += nt) {
    const int2 it = __ldcg(in.hlist + i);
    if (it.y != 0) continue;
    const int v = it.x;
    const int hid = __ldg(p.hub_base + v);
    const long long tot = __ldcg(p.hc_alloc + hid), moved = __ldcg(p.hc_moved + hid);
    const int mh = __ldcg(p.hc_min + hid), looked = __ldcg(p.hc_done + hid);
    const long long ex0 = __ldcg(p.excess + v);
    int h = __ldcg(p.height + v);
    const bool complete = looked == nchunks(deg_of(p, v));  // every chunk gave its minimum
    // clean for the next round
    p.hc_alloc[hid] = 0;
    p.hc_moved[hid] = 0;
    p.hc_min[hid] = INT_MAX;
    p.hc_done[hid] = 0;
    if (!(ex0 > 0 && h < p.n) || is_term(p, v) || !inst_on(p, v)) continue;
    seen++;
    ls.visits++;
    const long long ex = ex0 - moved;
    if (moved) atomic_add_ll(p.excess + v, -moved);
    if (ex > 0 && moved == tot && complete) {  // every admissible arc saturated: relabel
      h = mh >= p.n ? p.n : mh + 1;
      p.height[v] = h;
      ls.relabels++;
    }
    if (!topo && ex > 0 && h < p.n) enqueue(p, r, round_id, v);
  }
  if (topo) agg_add_int(&p.ctrl->seen[r % 3], seen);
}

// recalculate_max_flow_kernel_39 (code/dyn_data.h:208-215) as a reduction:
// flow = excess(t) + sum of negative excess over v != s, t (per instance in
// batched mode).
template <int BLOCK>
// Dead vertices are skipped: a sink or a deficit is a seed of every global
// relabel, so it is never proven dead.
__device__ __forceinline__ void ph_flow(const Params &p, typename BlockGroup<BLOCK>::Temp &btmp) {
  long long acc = 0;
  for_live_vertices<8>(p, [&](int v) {
    const long long ex = __ldcg(p.excess + v);
    long long c = 0;
    if (is_snk(p, v)) c = ex;
    else if (!is_src(p, v) && ex < 0) c = ex;
    if (p.inst) {
      if (c) atomic_add_ll(p.inst_flow + __ldg(p.inst + v), c);
    } else {
      acc += c;
    }
  });
  if (p.inst) return;
  __syncthreads();
  long long tot = typename BlockGroup<BLOCK>::RedL(btmp.redl).Sum(acc);
  if (threadIdx.x == 0 && tot) atomic_add_ll(&p.ctrl->flow, tot);
}

__device__ __forceinline__ void clear_slot(Slot *s) {
  s->q = 0;
  s->hq = 0;
  s->arcs = 0;
  s->cnt = 0;
}

// ---- push-pull, phase 1 (code/dyn_pp_bench.cu:6-88, part_pp) --------------------
// The cut kept from the previous solve splits the vertices into the sink side B
// (side = 1) and the source side A (side = 0).  Phase 1 works inside each side:
// B pushes its excess towards t and B's deficits (heights: residual distance to
// them within B, pp_bfs code/dyn_pp.h:99-120), A pulls its deficits from A's
// excess (heights: residual distance from an excess vertex within A; pull_kernel
// code/dyn_pp.h:237-280), both in the same rounds.  Arcs between the sides are
// not touched.  Phase 2, the general solve, then finishes exactly.

__device__ __forceinline__ bool pp_active(const Params &p, int v, long long ex) {
  if (is_term(p, v)) return false;
  return p.side[v] ? ex > 0 : ex < 0;
}

// Seeds (pp_bfs_init, code/dyn_pp.h:76-83): t, B's deficits and A's excess.
__device__ __forceinline__ void ph_pp_init(const Params &p, Slot *out) {
  const int nt = gridDim.x * blockDim.x, gt = blockIdx.x * blockDim.x + threadIdx.x;
  Ctrl *c = p.ctrl;
  if (gt == 0) {
    c->act_q = 0;
    c->act_hq = 0;
    c->wtail[0] = c->whtail[0] = c->seen[0] = 0;
  }
  int pos = 0;
  for (int v = gt; v < p.n; v += nt) {
    if (!inst_on(p, v)) continue;
    const long long ex = __ldcg(p.excess + v);
    const int sd = p.side[v];
    const bool seed = is_snk(p, v) || (!is_src(p, v) && (sd ? ex < 0 : ex > 0));
    if (seed) {
      p.height[v] = 0;
      if (deg_of(p, v) > p.hub_deg) append_hub(p, p.fh[0], &out->hq, v);
      else append(p.fq[0], &out->q, v);
    } else {
      p.height[v] = UNV;
    }
    if (pp_active(p, v, ex)) pos++;
  }
  agg_add_int(&c->pos_count, pos);
}

// One level over the frontier: a B vertex x labels B neighbours w with residual
// w->x, an A vertex x labels A neighbours w with residual x->w; s and t are
// never labelled.  All phase-1 actives go to the non-hub active list.
__device__ __forceinline__ void pp_td_range(const Params &p, Slot *out, int nxt, int x, int first, int end,
                                            int stride, int L, LStats &ls, VisitAcc &acc) {
  const int sx = p.side[x];
  for (int a = first; a < end; a += stride) {
    const int w = __ldg(p.adj + a);
    ls.arcs++;
    if (is_term(p, w) || p.side[w] != sx) continue;
    if (__ldcg(p.height + w) != UNV) continue;
    const int r = sx ? __ldcg(p.res + __ldg(p.par + a)) : __ldcg(p.res + a);
    if (r <= 0 || atomicCAS(p.height + w, UNV, L + 1) != UNV) continue;
    const int d = deg_of(p, w);
    if (d > p.hub_deg) append_hub(p, p.fh[nxt], &out->hq, w);
    else append(p.fq[nxt], &out->q, w);
    if (pp_active(p, w, __ldcg(p.excess + w))) {
      append(p.aq, &p.ctrl->act_q, w);
      acc.reached++;
    }
  }
}

template <int TILE>
__device__ __forceinline__ void ph_pp_bfs(const Params &p, const Slot *in, Slot *out, int L, LStats &ls) {
  const int cur = L & 1, nxt = cur ^ 1;
  const int nn = ld_vol(&in->q), nh = ld_vol(&in->hq);
  VisitAcc acc;
  const int lane = threadIdx.x & 31, nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = spread_group<32>(); i < nh; i += nwarps) {
    const int2 it = __ldcg(p.fh[cur] + i);
    int beg, end;
    chunk_range(p, it, beg, end);
    pp_td_range(p, out, nxt, it.x, beg + lane, end, 32, L, ls, acc);
  }
  for_tiered<TILE>(p, ls, p.fq[cur], nn, [&](auto &g, int x) {
    const int beg = __ldg(p.off + x), end = __ldg(p.off + x + 1);
    pp_td_range(p, out, nxt, x, beg + g.rank(), end, g.size(), L, ls, acc);
  });
  flush_visits(p, out, acc);
}

// Unlabelled vertices cannot reach a target within their side: inactive for
// phase 1 (not dead: the general solve decides that).
__device__ __forceinline__ void ph_pp_finalize(const Params &p) {
  const int nt = gridDim.x * blockDim.x, gt = blockIdx.x * blockDim.x + threadIdx.x;
  if (gt == 0) p.ctrl->pos_count = 0;  // read by every block before this phase
  for (int v = gt; v < p.n; v += nt)
    if (__ldcg(p.height + v) == UNV && inst_on(p, v)) p.height[v] = p.n;
}

__device__ __forceinline__ void pp_enqueue(const Params &p, int r, unsigned round_id, int v) {
  if (atomicExch(p.stamp + v, (int)round_id) == (int)round_id) return;
  append(p.wq[r & 1], &p.ctrl->wtail[r % 3], v);
}

// Push (B vertex, to B neighbours) or pull (A vertex, from A neighbours) of one
// vertex by a group, two passes per cycle as in discharge: pass 1 sums the
// admissible residual (head / tail labelled below h) and the minimum label over
// the other residual arcs; a group prefix sum gives lane budgets; pass 2 moves
// them.  A pull of d from w along w->v lowers res(w->v) and excess(w).
template <class G>
__device__ __forceinline__ void pp_discharge(G &g, const Params &p, int v, int r, unsigned round_id, LStats &ls) {
  long long e0 = 0;
  int hh = 0;
  if (g.rank() == 0) {
    e0 = __ldcg(p.excess + v);
    hh = __ldcg(p.height + v);
  }
  long long ex0;
  int h;
  if constexpr (G::size() == 1) {
    ex0 = e0;
    h = hh;
  } else {
    ex0 = g.g.shfl(e0, 0);
    h = g.g.shfl(hh, 0);
  }
  const bool pull = p.side[v] == 0;
  if (!pp_active(p, v, ex0) || h >= p.n) return;
  if (g.rank() == 0) ls.visits++;
  long long need = pull ? -ex0 : ex0;
  const long long need0 = need;
  const int beg = __ldg(p.off + v), end = __ldg(p.off + v + 1);
  constexpr int S = G::size();
  for (int cyc = 0; cyc < p.cycles && need > 0 && h < p.n; cyc++) {
    long long tsum = 0;
    int tmin = INT_MAX;
    for (int a = beg + g.rank(); a < end; a += S) {
      const int w = __ldg(p.adj + a);
      ls.arcs++;
      // B pushes to B (t included); A pulls from A (s excluded: its arcs are saturated)
      if (is_src(p, w) || p.side[w] != (pull ? 0 : 1)) continue;
      const int rr = pull ? __ldcg(p.res + __ldg(p.par + a)) : __ldcg(p.res + a);
      if (rr <= 0) continue;
      const int hw = __ldcg(p.height + w);
      if (hw < h) tsum += rr;
      else tmin = min(tmin, hw);
    }
    long long tot;
    const long long pre = g.scan(tsum, tot);
    long long budget = need - pre;
    budget = budget < 0 ? 0 : (budget > tsum ? tsum : budget);
    long long done = 0;
    for (int a = beg + g.rank(); a < end && budget > 0; a += S) {
      const int w = __ldg(p.adj + a);
      if (is_src(p, w) || p.side[w] != (pull ? 0 : 1)) continue;
      const int pa = __ldg(p.par + a);
      const int rr = pull ? __ldcg(p.res + pa) : __ldcg(p.res + a);
      if (rr <= 0 || __ldcg(p.height + w) >= h) continue;
      const int d = (int)(rr < budget ? rr : budget);
      if (pull) {
        atomicSub(p.res + pa, d);
        atomicAdd(p.res + a, d);
        const long long old = atomic_add_ll(p.excess + w, -(long long)d);
        if (old - d < 0 && old >= 0) pp_enqueue(p, r, round_id, w);  // w now has a deficit
      } else {
        atomicSub(p.res + a, d);
        atomicAdd(p.res + pa, d);
        const long long old = atomic_add_ll(p.excess + w, (long long)d);
        if (old + d > 0 && old <= 0) pp_enqueue(p, r, round_id, w);  // w now has excess
      }
      ls.pushes++;
      budget -= d;
      done += d;
    }
    const long long moved = g.sum_all(done);
    need -= moved;
    if (need > 0 && moved == tot) {
      const int mh = g.min_all(tmin);
      h = mh >= p.n ? p.n : mh + 1;
      if (g.rank() == 0) {
        p.height[v] = h;
        ls.relabels++;
      }
    }
  }
  if (g.rank() == 0) {
    const long long moved_total = need0 - need;
    if (moved_total) atomic_add_ll(p.excess + v, pull ? moved_total : -moved_total);
    if (need > 0 && h < p.n) pp_enqueue(p, r, round_id, v);
  }
}

template <int TILE>
__device__ __forceinline__ void ph_pp_round(const Params &p, const Ctrl *sc, int r, unsigned round_id, LStats &ls) {
  Ctrl *c = p.ctrl;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  if (gt == 0) c->wtail[(r + 1) % 3] = c->whtail[(r + 1) % 3] = c->seen[(r + 1) % 3] = 0;
  const int *list = r == 0 ? p.aq : p.wq[(r - 1) & 1];
  const int nn = r == 0 ? sc->act_q : sc->wtail[(r - 1) % 3];
  // small vertices by a lane, medium ones by a tile; hubs wait for phase 2
  const int nt = gridDim.x * blockDim.x;
  for (int i = spread_thread(rot_threads()); i < nn; i += nt) {
    const int v = __ldcg(list + i);
    if (deg_of(p, v) > p.small_deg) continue;
    ThreadGroup th;
    pp_discharge(th, p, v, r, round_id, ls);
  }
  TileGroup<TILE> tg;
  for (int i = spread_group<TILE>(rot_tiles()); i < nn; i += nt / TILE) {
    int v = 0, d = 0;
    if (tg.rank() == 0) {
      v = __ldcg(list + i);
      d = deg_of(p, v);
    }
    v = tg.g.shfl(v, 0);
    d = tg.g.shfl(d, 0);
    if (d <= p.small_deg || d > p.hub_deg) continue;  // hubs are left to the general solve
    pp_discharge(tg, p, v, r, round_id, ls);
  }
}

template <int TILE, int BLOCK>
__device__ __forceinline__ void run(const Params &p, LStats &ls, typename BlockGroup<BLOCK>::Temp &btmp, int *bci,
                    long long *bcl, Ctrl *sc) {
  // c: the control block in global memory (atomics, writes by the lead);
  // sc: this block's copy taken at the last barrier, for every read of a count
  // the previous phase produced
  Ctrl *c = p.ctrl;
  const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
  int ph = 0;
  int kind = 0;  // phase kind, recorded in the optional timeline
  long long items = 0, hubitems = 0;  // work of the phase, recorded with it
  auto slot_out = [&]() { return &c->slot[ph % 3]; };
  auto slot_in = [&]() { return &sc->slot[(ph + 2) % 3]; };
  auto record = [&]() {
    if (lead && p.trace && ph < p.trace_cap) {
      p.trace[4 * ph] = (unsigned long long)kind | ((unsigned long long)(items & 0xffffffffll) << 8) |
                        ((unsigned long long)(hubitems & 0xffffff) << 40);
      p.trace[4 * ph + 1] = globaltimer();
      p.trace[4 * ph + 2] = ph > 0 ? ld_vol((const long long *)&c->probe[(ph + 1) & 1]) : 0;
      p.trace[4 * ph + 3] = ph > 0 ? ld_vol((const long long *)&c->blk[(ph + 1) & 1]) : 0;
      c->probe[(ph + 1) & 1] = 0;
      c->blk[(ph + 1) & 1] = 0;
    }
  };
  auto next = [&]() -> bool {
    if (p.probe) {  // longest item of the phase that is ending
      cg::thread_block_tile<32> w = cg::tiled_partition<32>(cg::this_thread_block());
      const unsigned long long mx = cg::reduce(w, ls.probe, cg::greater<unsigned long long>());
      if (w.thread_rank() == 0 && mx) atomicMax(&c->probe[ph & 1], mx);
      ls.probe = 0;
      __syncthreads();  // the block's work of this phase is done
      if (threadIdx.x == 0 && ls.t_phase) atomicMax(&c->blk[ph & 1], globaltimer() - ls.t_phase);
    }
    if (!grid_barrier(c, sc, p.barrier_ns)) return false;
    if (p.probe && threadIdx.x == 0) ls.t_phase = globaltimer();
    ph++;
    record();
    if (lead) clear_slot(&c->slot[(ph + 1) % 3]);
    return true;
  };
  if ((int)blockIdx.x == p.absent_block) return;  // test hook: the others time out
  record();
  if (lead) clear_slot(&c->slot[1]);

  // ---- prologue --------------------------------------------------------------
  if (p.mode == MODE_STATIC) {
    kind = TR_INIT_RES;
    ph_init_res(p);
    if (!next()) return;
    kind = TR_SATURATE;
    ph_saturate(p);
    if (!next()) return;
  } else if (p.mode == MODE_DYNAMIC || p.mode == MODE_RECOMPUTE) {
    const bool dyn = p.mode == MODE_DYNAMIC;
    kind = TR_LOOKUP;
    ph_lookup(p);
    if (!next()) return;
    kind = TR_APPLY;
    ph_claim_apply(p, dyn);
    if (!next()) return;
    if (sc->dup_at) {  // every claim is done: undo them, reject the batch
      ph_unclaim(p, dyn);
      if (lead) set_err(c, ERR_DUP_ARC, sc->dup_at - 1);
      return;
    }
    if (dyn) {
      kind = TR_REPAIR;
      ph_repair(p, sc);
      if (!next()) return;
      if (p.variant == DMF_VARIANT_PP && !p.keep_dead) {  // with the dead set kept, ph_reopen does it
        kind = TR_CUT_SATURATE;
        ph_cut_saturate(p);
        if (!next()) return;
      }
      // source saturation and reopening touch disjoint arcs (a reopened arc's
      // tail is dead, so neither it nor its partner is a source arc): one phase
      kind = TR_SATURATE;
      ph_saturate(p);
      if (p.keep_dead) ph_reopen(p, sc);
      if (!next()) return;
    } else {
      kind = TR_INIT_RES;
      ph_init_res(p);
      if (!next()) return;
      kind = TR_SATURATE;
      ph_saturate(p);
      if (!next()) return;
    }
  }

  unsigned round_id = p.round_base;

  // ---- local repair inside the kept dead set ------------------------------------
  bool revive = true;  // the first global relabel revives every vertex
  if (p.mode == MODE_DYNAMIC && p.keep_dead) {
    revive = false;
    kind = TR_DEAD_SEED;
    items = sc->dcand;
    hubitems = 0;
    ph_dead_seed(p, sc, slot_out());
    if (!next()) return;
    if (lead) c->st_dseeds = (unsigned long long)sc->dseeds;
    if (sc->dseeds > 0) {
      const int nwarps = (gridDim.x * blockDim.x) >> 5;
      for (int r = 0; r < kDeadRounds; r++) {
        const Slot *in = slot_in();
        if (in->q == 0) break;
        kind = TR_DEAD_PULL;
        items = in->q;
        hubitems = 0;
        if (in->q <= kPullTail) {  // the remaining rounds in one block
          if (blockIdx.x == 0) pull_tail_rounds(p, r, in->q, round_id, ls);
          round_id += (unsigned)(kDeadRounds - r);
          if (!next()) return;
          if (lead) c->rounds_used = round_id - p.round_base;
          break;
        }
        round_id++;
        ph_dead_pull(p, p.fq[r & 1], in->q, p.fq[(r + 1) & 1], &slot_out()->q, spread_group<32>(), nwarps, round_id,
                     ls);
        if (!next()) return;
        if (lead) c->rounds_used = round_id - p.round_base;
      }
      kind = TR_DEAD_CHECK;
      items = sc->dcand;
      hubitems = 0;
      ph_dead_check(p, sc, slot_out());
      if (!next()) return;
      if (sc->dleft > 0) {
        // deficits left: revive what can reach them (partial), unless that
        // grows past a budget of arcs, then every vertex
        const long long budget = (long long)p.m / 16;
        long long scanned = 0;
        for (int L = 0;; L++) {
          const Slot *in = slot_in();
          if (L > 0) scanned += in->arcs;
          if (in->q + in->hq == 0) break;
          if (scanned > budget) {
            revive = true;
            break;
          }
          kind = TR_DEAD_REVIVE;
          items = in->q;
          hubitems = in->hq;
          ph_dead_revive<TILE>(p, in, slot_out(), L, ls);
          if (!next()) return;
        }
      }
    }
    if (lead) c->dkept = revive ? 0 : 1;
  }

  // ---- push-pull phase 1 (dynamic batches of the push-pull variant) ----------------
  // With the dead set kept, the batch is already split along the kept cut (the
  // dead side handled its deficits itself); phase 1 runs when it was revived.
  if (p.variant == DMF_VARIANT_PP && p.mode == MODE_DYNAMIC && revive) {
    for (int it1 = 0; it1 < kPPIters; it1++) {
      kind = TR_PP_INIT;
      items = hubitems = 0;
      ph_pp_init(p, slot_out());
      if (!next()) return;
      const int P = sc->pos_count;
      int reached = 0;
      for (int L = 0;; L++) {
        const Slot *in = slot_in();
        const int F = in->q + in->hq;
        reached += in->cnt;
        if (F == 0 || P == 0 || reached == P) break;
        kind = TR_PP_BFS;
        items = in->q;
        hubitems = in->hq;
        ph_pp_bfs<TILE>(p, in, slot_out(), L, ls);
        if (!next()) return;
      }
      kind = TR_PP_FINALIZE;
      items = hubitems = 0;
      ph_pp_finalize(p);
      if (!next()) return;
      const int A = sc->act_q;
      if (A == 0) break;
      for (int r = 0; r < p.interval; r++) {
        round_id++;
        kind = TR_PP_ROUND;
        items = r == 0 ? A : sc->wtail[(r - 1) % 3];
        hubitems = 0;
        ph_pp_round<TILE>(p, sc, r, round_id, ls);
        if (!next()) return;
        if (lead) c->rounds_used = round_id - p.round_base;
        if (sc->wtail[r % 3] == 0) break;
      }
    }
  }

  // ---- global relabel / push rounds ---------------------------------------------
  const bool cut_only = p.mode == MODE_CUT;
  const bool topo = p.variant == DMF_VARIANT_TOPO;
  for (int it = 0;; it++) {
    if (it >= p.max_iters) {
      if (lead) set_err(c, ERR_NO_CONV, it);
      return;
    }
    kind = TR_BFS_INIT;
    items = hubitems = 0;
    ph_bfs_init(p, slot_out(), it == 0 && revive, it == 0 && !revive);
    if (!next()) return;
    if (lead) c->st_outer++;
    const int P = sc->pos_count;
    const bool want_cut = p.need_cut || cut_only;
    if (P == 0 && !want_cut) break;
    long long m_u = sc->unexplored;
    bool bu = false, full = true;
    int L = 0, reached = 0;
    for (;; L++) {
      const Slot *in = slot_in();
      const int F = in->q + in->hq;
      const long long m_f = in->arcs;
      reached += in->cnt;
      if (F == 0) break;  // complete
      if (!cut_only && P > 0 && reached == P) {
        full = false;  // every active vertex has its exact distance
        break;
      }
      if (L > 0) m_u -= m_f;
      // a bottom-up level reads the arcs of the unvisited vertices and sweeps
      // every vertex's label (about n/16 arc reads' worth): with a kept dead set
      // the live part can be small next to that sweep
      if (!bu && p.bu_alpha > 0 && m_f * p.bu_alpha > m_u + p.n / 16) bu = true;
      else if (bu && (long long)F * 24 < p.n) bu = false;
      kind = bu ? TR_BFS_BU : TR_BFS_TD;
      items = in->q;
      hubitems = in->hq;
      if (bu) ph_bfs_bu<TILE>(p, slot_out(), L, ls);
      else ph_bfs_td<TILE>(p, in, slot_out(), L, ls);
      if (!next()) return;
      if (lead) c->st_levels++;
    }
    kind = TR_BFS_FINALIZE;
    items = hubitems = 0;
    ph_bfs_finalize(p, full, L + 1, full && want_cut);
    if (!next()) return;
    const int A = sc->act_q + sc->act_hq;
    if (A == 0 || cut_only) break;
    // a global relabel costs about one phase per BFS level and a push round moves
    // excess about one hop: on deep graphs (grids) allow as many rounds as the
    // relabel had levels before relabelling again (the loop ends early when the
    // worklist empties)
    const int rounds = (p.interval > L || !p.adaptive) ? p.interval : L;
    for (int r = 0; r < rounds; r++) {
      round_id++;
      const RoundIn in = round_inputs(p, sc, r, false);
      kind = TR_PUSH;
      items = in.nn;
      hubitems = in.nh;
      ph_push1<TILE, BLOCK>(p, in, r, round_id, p.relabel_base + it, ls, btmp, bci, bcl, false);
      if (!next()) return;
      if (in.nh > 0) {
        kind = TR_PUSH_HUB_FINISH;
        ph_push3(p, in, r, round_id, ls, false);
        if (!next()) return;
      }
      if (lead) {
        c->st_rounds++;
        c->rounds_used = round_id - p.round_base;
      }
      const int W = topo ? sc->seen[r % 3] : sc->wtail[r % 3] + sc->whtail[r % 3];
      if (W == 0) break;
    }
  }
  kind = TR_FLOW;
  items = hubitems = 0;
  ph_flow<BLOCK>(p, btmp);
  if (lead) c->rounds_used = round_id - p.round_base;
  // the flow phase ends without a barrier; its end is the kernel's end
  if (lead && p.trace && ph + 1 < p.trace_cap) c->trace_len = ph + 1;
}

template <int TILE, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_solve(Params p) {
  __shared__ typename BlockGroup<BLOCK>::Temp btmp;
  __shared__ int bci;
  __shared__ long long bcl;
  __shared__ Ctrl snap;
  LStats ls;
  run<TILE, BLOCK>(p, ls, btmp, &bci, &bcl, &snap);
  // statistics: one atomic per block and counter
  __syncthreads();
  typedef cub::BlockReduce<unsigned long long, BLOCK> R;
  __shared__ typename R::TempStorage rt;
  unsigned long long v[5] = {ls.pushes, ls.relabels, ls.arcs + ls.barcs, ls.visits, ls.barcs};
  unsigned long long *dst[5] = {&p.ctrl->st_pushes, &p.ctrl->st_relabels, &p.ctrl->st_arcs, &p.ctrl->st_visits,
                                &p.ctrl->st_barcs};
  for (int i = 0; i < 5; i++) {
    unsigned long long s = R(rt).Sum(v[i]);
    if (threadIdx.x == 0 && s) atomicAdd(dst[i], s);
    __syncthreads();
  }
}


using KernelFn = void (*)(Params);

// The kernel instantiations of tile width T (dmf_kernel_tT.cu); minb = resident
// blocks per SM the register budget is sized for (1: up to 128 registers a
// thread, 2: up to 64).
KernelFn solve_kernel_t4(int minb);
KernelFn solve_kernel_t8(int minb);
KernelFn solve_kernel_t16(int minb);
KernelFn solve_kernel_t32(int minb);

}  // namespace dmfk
