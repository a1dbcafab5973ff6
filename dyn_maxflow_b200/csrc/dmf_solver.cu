// dmf_solver.cu -- device half of libdmf.so: the persistent push-relabel
// solver for sm_100a and the solver entry points of the C ABI.
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
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "dmf_device.cuh"
#include "dmf_internal.h"
#include "dmf_sched_internal.h"

using namespace dmfd;

namespace {

constexpr int kBlock = 512;
constexpr int kChunk = 256;  // arcs per hub chunk: one warp item, 8 arcs per lane
constexpr int kPPIters = 1;  // push-pull phase-1 relabel rounds before the general solve

enum Mode : int { MODE_STATIC = 0, MODE_DYNAMIC = 1, MODE_RECOMPUTE = 2, MODE_CUT = 3 };

// Phase kinds of the optional timeline (dmf_trace_get); values are part of the ABI.
enum TraceKind : int {
  TR_START = 0, TR_INIT_RES = 1, TR_SATURATE = 2, TR_LOOKUP = 3, TR_APPLY = 4, TR_REPAIR = 5,
  TR_CUT_SATURATE = 6, TR_BFS_INIT = 7, TR_BFS_TD = 8, TR_BFS_BU = 9, TR_BFS_FINALIZE = 10, TR_PUSH = 11,
  TR_FLOW = 12, TR_PUSH_HUB = 13, TR_PUSH_HUB_FINISH = 14, TR_PP_INIT = 15, TR_PP_BFS = 16, TR_PP_FINALIZE = 17,
  TR_PP_ROUND = 18
};

// Largest capacity an update may set: keeps cap(e) + cap(partner) < 2^31 when
// both arcs of a pair change in one batch.
constexpr int kMaxUpdateCap = (1 << 30) - 1;

struct Params {
  int n, m, s, t;
  const int *__restrict__ off;
  const int *__restrict__ adj;
  const int *__restrict__ par;
  const int *__restrict__ sidx;
  int *cap, *res, *height, *stamp, *astamp, *uarc;
  long long *excess;
  unsigned char *dead, *side;
  int *fq[2], *wq[2], *aq;     // non-hub vertex queues
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
  int bu_alpha;  // bottom-up when frontier arcs * bu_alpha > unexplored arcs (0: never)
  int adaptive;  // push rounds per relabel at least the depth of the last relabel BFS
  unsigned round_base;
  int epoch;
  unsigned long long *trace;  // optional phase timeline: 4 words per entry
  int trace_cap;
  int probe;                  // time work items (DMF_FLAG_PROBE)
};

struct LStats {
  unsigned long long pushes = 0, relabels = 0, arcs = 0, visits = 0;
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

__device__ __forceinline__ void set_err(Ctrl *c, int bit, int info) {
  if (atomicOr(&c->err, bit) == 0) c->err_info = info;
}

// ---- prologue phases ----------------------------------------------------------

// staticMaxFlow_kernel_1 (code/dyn_data.h:25-35): residual = capacity, excess 0.
__device__ __forceinline__ void ph_init_res(const Params &p) {
  const int nt = gridDim.x * blockDim.x, gt = blockIdx.x * blockDim.x + threadIdx.x;
  for (int e = gt; e < p.m; e += nt) p.res[e] = __ldcg(p.cap + e);
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
      const int s = __ldg(p.srcs + i);
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

// Arc lookup of OnAdd_kernel (code/dyn_data.h:196-201) by binary search over the
// per-vertex head-sorted index; also validates the batch.
// Arc u->v by binary search over u's head-sorted arc index (the last arc among
// equal heads, as OnAdd_kernel's linear scan keeps the last match), or -1.
__device__ __forceinline__ int find_arc_dev(const int *__restrict__ off, const int *__restrict__ adj,
                                            const int *__restrict__ sidx, int u, int v) {
  const int first = __ldg(off + u);
  int lo = first, hi = __ldg(off + u + 1);
  while (lo < hi) {  // last position with head <= v
    const int mid = (lo + hi) >> 1;
    if (__ldg(adj + __ldg(sidx + mid)) <= v) lo = mid + 1;
    else hi = mid;
  }
  if (lo > first) {
    const int cand = __ldg(sidx + lo - 1);
    if (__ldg(adj + cand) == v) return cand;
  }
  return -1;
}

__device__ __forceinline__ void ph_lookup(const Params &p) {
  const int nt = gridDim.x * blockDim.x, gt = spread_thread();
  for (int i = gt; i < p.k; i += nt) {
    int u = __ldg(p.usrc + i), v = __ldg(p.udst + i), w = __ldg(p.uw + i);
    p.uarc[i] = -1;
    if (u < 0 || u >= p.n || v < 0 || v >= p.n || w < 0 || w > kMaxUpdateCap) {
      set_err(p.ctrl, ERR_BAD_UPDATE, i);
      continue;
    }
    if (u == v) continue;  // ignored, as OnAdd_kernel does (code/dyn_data.h:194)
    const int e = find_arc_dev(p.off, p.adj, p.sidx, u, v);
    if (e < 0) {
      set_err(p.ctrl, ERR_UNKNOWN_ARC, i);
      continue;
    }
    if (atomicExch(p.astamp + e, p.epoch) == p.epoch) {
      set_err(p.ctrl, ERR_DUP_ARC, i);
      continue;
    }
    if ((long long)w + __ldcg(p.cap + __ldg(p.par + e)) > INT_MAX) {
      set_err(p.ctrl, ERR_BAD_UPDATE, i);
      continue;
    }
    p.uarc[i] = e;
  }
}

// Capacity apply of OnAdd_kernel (code/dyn_data.h:202-205); in recompute mode
// only the capacity is set (update_kernel, code/dyn_data_bench.cu:300-322).
__device__ __forceinline__ void ph_apply(const Params &p, bool residual) {
  const int nt = gridDim.x * blockDim.x, gt = spread_thread();
  for (int i = gt; i < p.k; i += nt) {
    int e = __ldcg(p.uarc + i);
    if (e < 0) continue;
    int w = __ldg(p.uw + i);
    int delta = w - __ldcg(p.cap + e);
    p.cap[e] = w;
    if (residual && delta) atomicAdd(p.res + e, delta);
  }
}

// Over-capacity repair driven by the batch: replaces the O(m) sweeps
// incremental_kernel_20 / _22 (code/dyn_data.h:157-183).  An arc whose residual
// went negative carries more flow than its new capacity; the excess is returned
// to its tail and taken from its head.  At most one arc of a pair can be
// negative because res(e) + res(partner) = cap(e) + cap(partner) >= 0.
__device__ __forceinline__ void ph_repair(const Params &p) {
  const int nt = gridDim.x * blockDim.x, gt = spread_thread();
  for (int i = gt; i < p.k; i += nt) {
    int e = __ldcg(p.uarc + i);
    if (e < 0) continue;
    int r = __ldcg(p.res + e);
    if (r < 0) {
      p.res[e] = 0;
      atomicAdd(p.res + __ldg(p.par + e), r);
      atomic_add_ll(p.excess + __ldg(p.usrc + i), -(long long)r);
      atomic_add_ll(p.excess + __ldg(p.adj + e), (long long)r);
    }
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
    int u = __ldg(p.usrc + i), v = __ldg(p.adj + e);
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

// Seeds (my_init_1, code/dyn_data.h:60-67): t and every deficit vertex other
// than s get height 0; all other live vertices become unvisited.
__device__ __forceinline__ void ph_bfs_init(const Params &p, Slot *out, bool reset_dead) {
  const int nt = gridDim.x * blockDim.x, gt = blockIdx.x * blockDim.x + threadIdx.x;
  Ctrl *c = p.ctrl;
  if (gt == 0) {
    c->act_q = 0;
    c->act_hq = 0;
    c->wtail[0] = c->whtail[0] = c->seen[0] = 0;  // written by push round 0
  }
  int pos = 0;
  long long unexpl = 0, seed_arcs = 0;
  for (int v = gt; v < p.n; v += nt) {
    if (p.inst_active && !p.inst_active[__ldg(p.inst + v)]) {
      if (reset_dead) {
        p.dead[v] = 1;
        p.height[v] = p.n;
      }
      continue;
    }
    if (reset_dead) {
      if (__ldcg(p.dead + v)) p.dead[v] = 0;
    } else if (__ldcg(p.dead + v)) {
      continue;
    }
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
  }
  block_add_int(&c->pos_count, pos);
  block_add_ll(&c->unexplored, unexpl);
  block_add_ll(&out->arcs, seed_arcs);
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
      if (w[k] >= 0) ls.arcs++;
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
    if (w[k] >= 0) ls.arcs++;
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
__device__ __forceinline__ void ph_bfs_finalize(const Params &p, bool full, int floor_h, bool write_side) {
  const int nt = gridDim.x * blockDim.x, gt = blockIdx.x * blockDim.x + threadIdx.x;
  int nd = 0;
  for (int v = gt; v < p.n; v += nt) {
    int h = __ldcg(p.height + v);
    if (h == UNV) {
      if (full) {
        p.dead[v] = 1;
        p.height[v] = p.n;
        nd++;
      } else {
        p.height[v] = floor_h;
      }
    }
    if (write_side && (!p.inst_active || p.inst_active[__ldg(p.inst + v)])) p.side[v] = h < p.n ? 1 : 0;
  }
  block_add_ll((long long *)&p.ctrl->st_dead, nd);
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

__device__ __forceinline__ RoundIn round_inputs(const Params &p, const Ctrl *c, int r) {
  RoundIn in;
  if (p.variant == DMF_VARIANT_TOPO) {
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
                         typename BlockGroup<BLOCK>::Temp &btmp, int *bci, long long *bcl) {
  Ctrl *c = p.ctrl;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const bool topo = p.variant == DMF_VARIANT_TOPO;
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
      if (!has_ex || h >= p.n || is_term(p, v)) {
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
      [&](int v) { return !topo || __ldcg(p.excess + v) > 0; });
  if (topo) agg_add_int(&c->seen[r % 3], seen);
  sink_flush(p, ls);
}

// Push round, phase 2 (hubs): per hub (its first chunk), the moved total leaves
// its excess; when all of the hub's admissible residual was pushed and excess is
// left, the hub is relabelled to 1 + the minimum non-admissible height; a hub
// with excess left is queued for the next round.  The hub's totals are reset.
__device__ __forceinline__ void ph_push3(const Params &p, const RoundIn &in, int r, unsigned round_id, LStats &ls) {
  const int nt = gridDim.x * blockDim.x;
  const bool topo = p.variant == DMF_VARIANT_TOPO;
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
    if (!(ex0 > 0 && h < p.n) || is_term(p, v)) continue;
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
__device__ __forceinline__ void ph_flow(const Params &p, typename BlockGroup<BLOCK>::Temp &btmp) {
  const int nt = gridDim.x * blockDim.x, gt = blockIdx.x * blockDim.x + threadIdx.x;
  long long acc = 0;
  for (int v = gt; v < p.n; v += nt) {
    const long long ex = __ldcg(p.excess + v);
    long long c = 0;
    if (is_snk(p, v)) c = ex;
    else if (!is_src(p, v) && ex < 0) c = ex;
    if (p.inst) {
      if (c && (!p.inst_active || p.inst_active[__ldg(p.inst + v)])) atomic_add_ll(p.inst_flow + __ldg(p.inst + v), c);
    } else {
      acc += c;
    }
  }
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
    if (__ldcg(p.height + v) == UNV) p.height[v] = p.n;
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
    if (!grid_barrier(c, sc)) return false;
    if (p.probe && threadIdx.x == 0) ls.t_phase = globaltimer();
    ph++;
    record();
    if (lead) clear_slot(&c->slot[(ph + 1) % 3]);
    return true;
  };
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
  } else if (p.mode == MODE_DYNAMIC) {
    kind = TR_LOOKUP;
    ph_lookup(p);
    if (!next()) return;
    kind = TR_APPLY;
    ph_apply(p, true);
    if (!next()) return;
    kind = TR_REPAIR;
    ph_repair(p);
    if (!next()) return;
    if (p.variant == DMF_VARIANT_PP) {
      kind = TR_CUT_SATURATE;
      ph_cut_saturate(p);
      if (!next()) return;
    }
    kind = TR_SATURATE;
    ph_saturate(p);
    if (!next()) return;
  } else if (p.mode == MODE_RECOMPUTE) {
    kind = TR_LOOKUP;
    ph_lookup(p);
    if (!next()) return;
    kind = TR_APPLY;
    ph_apply(p, false);
    if (!next()) return;
    kind = TR_INIT_RES;
    ph_init_res(p);
    if (!next()) return;
    kind = TR_SATURATE;
    ph_saturate(p);
    if (!next()) return;
  }

  unsigned round_id = p.round_base;

  // ---- push-pull phase 1 (dynamic batches of the push-pull variant) ----------------
  if (p.variant == DMF_VARIANT_PP && p.mode == MODE_DYNAMIC) {
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
    ph_bfs_init(p, slot_out(), it == 0);
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
      if (!bu && p.bu_alpha > 0 && m_f * p.bu_alpha > m_u) bu = true;
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
      const RoundIn in = round_inputs(p, sc, r);
      kind = TR_PUSH;
      items = in.nn;
      hubitems = in.nh;
      ph_push1<TILE, BLOCK>(p, in, r, round_id, p.relabel_base + it, ls, btmp, bci, bcl);
      if (!next()) return;
      if (in.nh > 0) {
        kind = TR_PUSH_HUB_FINISH;
        ph_push3(p, in, r, round_id, ls);
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
  unsigned long long v[4] = {ls.pushes, ls.relabels, ls.arcs, ls.visits};
  unsigned long long *dst[4] = {&p.ctrl->st_pushes, &p.ctrl->st_relabels, &p.ctrl->st_arcs, &p.ctrl->st_visits};
  for (int i = 0; i < 4; i++) {
    unsigned long long s = R(rt).Sum(v[i]);
    if (threadIdx.x == 0 && s) atomicAdd(dst[i], s);
    __syncthreads();
  }
}

// Raw feature sums of an update batch against the current residual state, for
// the schedule picker (nothing is modified).  Updates the solver would reject
// (bad ids, unknown arcs) are skipped here; the solve reports them.
__global__ void __launch_bounds__(256) k_features(const int *__restrict__ off, const int *__restrict__ adj,
                                                  const int *__restrict__ sidx, const int *cap, const int *res, int n,
                                                  int k, const int *usrc, const int *udst, const int *uw,
                                                  dmfs::FeatAcc *acc) {
  unsigned long long valid = 0, dec = 0, satdec = 0, incsat = 0, ins = 0, del = 0, sdeg = 0, mdeg = 0;
  long long exc = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
    const int u = __ldg(usrc + i), v = __ldg(udst + i), w = __ldg(uw + i);
    if (u < 0 || u >= n || v < 0 || v >= n || u == v) continue;
    const int e = find_arc_dev(off, adj, sidx, u, v);
    if (e < 0) continue;
    valid++;
    const int c0 = __ldcg(cap + e), r = __ldcg(res + e);
    const long long flow = (long long)c0 - r;  // negative: the partner carries flow
    const unsigned long long d = (unsigned long long)(__ldg(off + u + 1) - __ldg(off + u));
    sdeg += d;
    mdeg = d > mdeg ? d : mdeg;
    if (w < c0) {
      dec++;
      if (flow > w) {
        satdec++;
        exc += flow - w;
      }
    } else if (w > c0 && r == 0) {
      incsat++;
    }
    if (c0 == 0 && w > 0) ins++;
    if (c0 > 0 && w == 0) del++;
  }
  cg::thread_block_tile<32> wp = cg::tiled_partition<32>(cg::this_thread_block());
  valid = cg::reduce(wp, valid, cg::plus<unsigned long long>());
  dec = cg::reduce(wp, dec, cg::plus<unsigned long long>());
  satdec = cg::reduce(wp, satdec, cg::plus<unsigned long long>());
  incsat = cg::reduce(wp, incsat, cg::plus<unsigned long long>());
  ins = cg::reduce(wp, ins, cg::plus<unsigned long long>());
  del = cg::reduce(wp, del, cg::plus<unsigned long long>());
  sdeg = cg::reduce(wp, sdeg, cg::plus<unsigned long long>());
  mdeg = cg::reduce(wp, mdeg, cg::greater<unsigned long long>());
  exc = cg::reduce(wp, exc, cg::plus<long long>());
  if (wp.thread_rank() == 0 && valid) {
    atomicAdd(&acc->valid, valid);
    atomicAdd(&acc->dec, dec);
    atomicAdd(&acc->satdec, satdec);
    atomicAdd(&acc->incsat, incsat);
    atomicAdd(&acc->ins, ins);
    atomicAdd(&acc->del, del);
    atomicAdd(&acc->sum_deg, sdeg);
    atomicMax(&acc->max_deg, mdeg);
    atomic_add_ll(&acc->excess_created, exc);
  }
}

using KernelFn = void (*)(Params);

// minb = resident blocks per SM the register budget is sized for (1: up to 128
// registers a thread, 2: up to 64).
KernelFn pick_kernel(int tile, int minb) {
  if (minb == 1) {
    switch (tile) {
      case 4: return k_solve<4, kBlock, 1>;
      case 8: return k_solve<8, kBlock, 1>;
      case 16: return k_solve<16, kBlock, 1>;
      default: return k_solve<32, kBlock, 1>;
    }
  }
  switch (tile) {
    case 4: return k_solve<4, kBlock, 2>;
    case 8: return k_solve<8, kBlock, 2>;
    case 16: return k_solve<16, kBlock, 2>;
    default: return k_solve<32, kBlock, 2>;
  }
}

}  // namespace

// ============================================================================
// host side
// ============================================================================
using dmf::fail;
using dmf::ok;
using dmf::guarded;

struct dmf_solver {
  int dev = 0;
  cudaStream_t stream = nullptr;
  int n = 0, m = 0, s = 0, t = 0;
  dmf_opts opts{};
  int tile = 32, grid = 0, block = kBlock, hub_deg = 256, small_deg = 8, minb = 2, bu_alpha = 2;
  int *off = nullptr, *adj = nullptr, *par = nullptr, *sidx = nullptr, *cap = nullptr, *res = nullptr;
  int *height = nullptr, *stamp = nullptr, *astamp = nullptr, *uarc = nullptr;
  long long *excess = nullptr;
  unsigned char *dead = nullptr, *side = nullptr;
  int *qbuf = nullptr;    // 5 vertex queues (frontier x2, worklist x2, active)
  int2 *hqbuf = nullptr;  // 5 hub-chunk queues, same roles
  int2 *hch = nullptr;    // every hub's chunks
  int nchunk = 0;         // total hub chunks = capacity of each hub-chunk queue
  long long *hc_moved = nullptr, *hc_alloc = nullptr;  // per hub, push-round totals
  int *hc_min = nullptr, *hc_done = nullptr;
  int *hub_base = nullptr;
  unsigned long long *chunk_mark = nullptr;
  int *chunk_tmin = nullptr;
  unsigned relabel_base = 1;
  bool thresholds_set = false;
  // batched instances (dmf_multi_*): roles, instance ids, sources, per-instance flows
  int ninst = 1;
  unsigned char *role = nullptr;
  int *inst = nullptr;
  int *srcs = nullptr;
  int *src_off = nullptr;  // prefix sums of the sources' degrees
  int nsrc = 1;
  long long *inst_flow = nullptr;
  long long *h_inst_flow = nullptr;  // pinned
  std::vector<int> vbase;            // first vertex of each instance in the union
  std::vector<int64_t> flows;        // last per-instance flows
  cudaStream_t own_stream = nullptr; // for graph capture when the user stream is the legacy one
  unsigned char *inst_active = nullptr;     // device mask for the next launch (batched mode)
  unsigned char *h_inst_active = nullptr;   // pinned staging
  bool use_active = false;
  int *ubuf = nullptr;  // device update staging: src | dst | w
  int kcap = 0;
  int *h_ubuf = nullptr;  // pinned host staging
  int h_kcap = 0;
  Ctrl *ctrl = nullptr;
  Ctrl *h_ctrl = nullptr;  // pinned
  unsigned long long *trace = nullptr;  // device timeline (opts.flags & DMF_FLAG_TRACE)
  int trace_cap = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  unsigned round_base = 1;
  int epoch = 0;
  bool solved = false, side_valid = false;
  dmf_stats st{};
  // schedule picker: feature sums of the batch being scheduled, per-batch log
  dmfs::FeatAcc *facc = nullptr;
  struct SchedRecord {
    float feat[DMF_SCHED_FEATURES];
    int action;
    float ms;
    int64_t flow;
  };
  std::vector<SchedRecord> records;
  std::vector<void *> allocs;
};

namespace {

int cuda_fail(cudaError_t e, const char *what) {
  return fail(e == cudaErrorMemoryAllocation ? DMF_ERR_OOM : DMF_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call, what)                                  \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, what);  \
  } while (0)

template <class T>
int dalloc(dmf_solver *sv, T **p, size_t count) {
  void *q = nullptr;
  sv->allocs.reserve(sv->allocs.size() + 1);  // may throw; the push below then cannot
  cudaError_t e = cudaMalloc(&q, sizeof(T) * std::max<size_t>(count, 1));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  sv->allocs.push_back(q);
  *p = (T *)q;
  return DMF_OK;
}

void free_all(dmf_solver *sv) {
  if (sv->dev >= 0) cudaSetDevice(sv->dev);
  if (sv->stream) cudaStreamSynchronize(sv->stream);
  for (void *q : sv->allocs) cudaFree(q);
  sv->allocs.clear();
  if (sv->h_ubuf) cudaFreeHost(sv->h_ubuf);
  if (sv->h_ctrl) cudaFreeHost(sv->h_ctrl);
  if (sv->h_inst_flow) cudaFreeHost(sv->h_inst_flow);
  sv->h_inst_flow = nullptr;
  if (sv->h_inst_active) cudaFreeHost(sv->h_inst_active);
  sv->h_inst_active = nullptr;
  if (sv->own_stream) cudaStreamDestroy(sv->own_stream);
  sv->own_stream = nullptr;
  if (sv->ev0) cudaEventDestroy(sv->ev0);
  if (sv->ev1) cudaEventDestroy(sv->ev1);
  sv->h_ubuf = nullptr;
  sv->h_ctrl = nullptr;
  sv->ev0 = sv->ev1 = nullptr;
}

int choose_tile(const dmf_opts &o, int n, int m) {
  if (o.tile == 1 || o.tile == 2 || o.tile == 4) return 4;
  if (o.tile == 8 || o.tile == 16 || o.tile == 32) return o.tile;
  double avg = n > 0 ? (double)m / n : 0;
  if (avg <= 6) return 4;
  if (avg <= 12) return 8;
  if (avg <= 24) return 16;
  return 32;
}

int configure(dmf_solver *sv) {
  sv->tile = choose_tile(sv->opts, sv->n, sv->m);
  if (!sv->thresholds_set) {  // fixed for the solver's life: they size the hub-chunk queues
    sv->hub_deg = 8 * sv->tile;
    sv->small_deg = 8;
    // tuning overrides (thread-per-vertex and chunked-hub degree bounds)
    if (const char *e = std::getenv("DMF_SMALL_DEG")) sv->small_deg = std::max(0, std::atoi(e));
    if (const char *e = std::getenv("DMF_HUB_DEG")) sv->hub_deg = std::max(32, std::atoi(e));
    if (const char *e = std::getenv("DMF_BU_ALPHA")) sv->bu_alpha = std::max(0, std::atoi(e));
    sv->thresholds_set = true;
  }
  sv->minb = 2;
  if (const char *e = std::getenv("DMF_MINB")) sv->minb = std::atoi(e) == 1 ? 1 : 2;
  KernelFn fn = pick_kernel(sv->tile, sv->minb);
  int per_sm = 0, sms = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)fn, kBlock, 0), "occupancy");
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, sv->dev), "sm count");
  int coop = 0;
  CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, sv->dev), "coop attr");
  if (!coop || per_sm < 1) return fail(DMF_ERR_CUDA, "device does not support cooperative launch of the solver");
  sv->grid = per_sm * sms;
  if (sv->opts.grid_blocks > 0) sv->grid = std::min(sv->grid, sv->opts.grid_blocks);
  if (sv->opts.small_deg > 0) sv->small_deg = sv->opts.small_deg;
  else if (sv->opts.small_deg < 0) sv->small_deg = 0;  // no thread tier
  sv->block = kBlock;
  return DMF_OK;
}

int ensure_ubuf(dmf_solver *sv, int k) {
  if (k <= sv->kcap) return DMF_OK;
  int want = std::max(k, 1024);
  int *nb = nullptr;
  CK(cudaMalloc(&nb, sizeof(int) * 4 * (size_t)want), "cudaMalloc updates");
  // uarc lives in the 4th quarter
  if (sv->ubuf) {
    cudaStreamSynchronize(sv->stream);
    cudaFree(sv->ubuf);
  }
  sv->ubuf = nb;
  sv->kcap = want;
  return DMF_OK;
}

int ensure_host_ubuf(dmf_solver *sv, int k) {
  if (k <= sv->h_kcap) return DMF_OK;
  int want = std::max(k, 1024);
  int *nb = nullptr;
  CK(cudaMallocHost(&nb, sizeof(int) * 3 * (size_t)want), "cudaMallocHost");
  if (sv->h_ubuf) {
    cudaStreamSynchronize(sv->stream);
    cudaFreeHost(sv->h_ubuf);
  }
  sv->h_ubuf = nb;
  sv->h_kcap = want;
  return DMF_OK;
}

Params make_params(dmf_solver *sv, int mode, int k, const int *d_src, const int *d_dst, const int *d_w) {
  Params p{};
  p.n = sv->n;
  p.m = sv->m;
  p.s = sv->s;
  p.t = sv->t;
  p.off = sv->off;
  p.adj = sv->adj;
  p.par = sv->par;
  p.sidx = sv->sidx;
  p.cap = sv->cap;
  p.res = sv->res;
  p.height = sv->height;
  p.stamp = sv->stamp;
  p.astamp = sv->astamp;
  p.uarc = sv->ubuf ? sv->ubuf + 3 * (size_t)sv->kcap : nullptr;
  p.excess = sv->excess;
  p.dead = sv->dead;
  p.side = sv->side;
  const size_t N = (size_t)sv->n + 1;
  const size_t NC = (size_t)std::max(sv->nchunk, 1);
  for (int i = 0; i < 2; i++) {
    p.fq[i] = sv->qbuf + (0 + i) * N;
    p.wq[i] = sv->qbuf + (2 + i) * N;
    p.fh[i] = sv->hqbuf + (0 + i) * NC;
    p.wh[i] = sv->hqbuf + (2 + i) * NC;
  }
  p.aq = sv->qbuf + 4 * N;
  p.ah = sv->hqbuf + 4 * NC;
  p.hch = sv->hch;
  p.nhch = sv->nchunk;
  p.hc_moved = sv->hc_moved;
  p.hc_alloc = sv->hc_alloc;
  p.hc_min = sv->hc_min;
  p.hc_done = sv->hc_done;
  p.hub_base = sv->hub_base;
  p.role = sv->role;
  p.inst = sv->inst;
  p.inst_flow = sv->inst_flow;
  p.srcs = sv->srcs;
  p.src_off = sv->src_off;
  p.nsrc = sv->nsrc;
  p.inst_active = sv->use_active ? sv->inst_active : nullptr;
  p.chunk_mark = sv->chunk_mark;
  p.chunk_tmin = sv->chunk_tmin;
  p.relabel_base = sv->relabel_base;
  p.usrc = d_src;
  p.udst = d_dst;
  p.uw = d_w;
  p.k = k;
  p.ctrl = sv->ctrl;
  p.mode = mode;
  p.variant = sv->opts.variant;
  const int avg = sv->n > 0 ? std::max(1, sv->m / sv->n) : 1;
  (void)avg;
  p.cycles = sv->opts.kernel_cycles > 0 ? sv->opts.kernel_cycles : 2;
  p.interval = sv->opts.relabel_interval > 0 ? sv->opts.relabel_interval : 6;
  p.max_iters = sv->opts.max_iters > 0 ? sv->opts.max_iters : 100000;
  p.hub_deg = sv->hub_deg;
  p.small_deg = sv->small_deg;
  p.bu_alpha = sv->bu_alpha;
  p.adaptive = (sv->opts.flags & DMF_FLAG_FIXED_INTERVAL) ? 0 : 1;
  p.need_cut = sv->opts.variant == DMF_VARIANT_PP ? 1 : 0;
  p.round_base = sv->round_base;
  p.trace = (sv->opts.flags & DMF_FLAG_TRACE) ? sv->trace : nullptr;
  p.probe = (sv->opts.flags & DMF_FLAG_PROBE) && p.trace ? 1 : 0;
  p.trace_cap = sv->trace_cap;
  p.epoch = ++sv->epoch;
  if (sv->epoch == INT_MAX) sv->epoch = 0;
  return p;
}

int launch(dmf_solver *sv, int mode, int k, const int *d_src, const int *d_dst, const int *d_w) {
  Params p = make_params(sv, mode, k, d_src, d_dst, d_w);
  CK(cudaMemsetAsync(sv->ctrl, 0, sizeof(Ctrl), sv->stream), "memset ctrl");
  if (sv->inst_flow) CK(cudaMemsetAsync(sv->inst_flow, 0, 8 * (size_t)sv->ninst, sv->stream), "memset flows");
  void *args[] = {&p};
  CK(cudaLaunchCooperativeKernel((const void *)pick_kernel(sv->tile, sv->minb), dim3(sv->grid), dim3(sv->block), args, 0,
                                 sv->stream),
     "cooperative launch");
  CK(cudaMemcpyAsync(sv->h_ctrl, sv->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, sv->stream), "D2H ctrl");
  if (sv->inst_flow)
    CK(cudaMemcpyAsync(sv->h_inst_flow, sv->inst_flow, 8 * (size_t)sv->ninst, cudaMemcpyDeviceToHost, sv->stream),
       "D2H flows");
  return DMF_OK;
}

// Waits for the launch sequence, records timing and maps device errors.
int finish(dmf_solver *sv, int64_t *flow, bool need_cut_valid) {
  CK(cudaEventRecord(sv->ev1, sv->stream), "event record");
  CK(cudaEventSynchronize(sv->ev1), "solve");
  float ms = 0;
  cudaEventElapsedTime(&ms, sv->ev0, sv->ev1);
  const Ctrl &c = *sv->h_ctrl;
  sv->st.last_ms = ms;
  sv->st.outer_iters = (int64_t)c.st_outer;
  sv->st.bfs_levels = (int64_t)c.st_levels;
  sv->st.push_rounds = (int64_t)c.st_rounds;
  sv->st.pushes = (int64_t)c.st_pushes;
  sv->st.relabels = (int64_t)c.st_relabels;
  sv->st.arcs_scanned = (int64_t)c.st_arcs;
  sv->st.vertices_visited = (int64_t)c.st_visits;
  sv->st.dead_vertices = (int64_t)c.st_dead;
  sv->st.grid_blocks = sv->grid;
  sv->st.block_threads = sv->block;
  sv->st.tile = sv->tile;
  sv->round_base += c.rounds_used + 2;
  sv->relabel_base += (unsigned)c.st_outer + 2;
  if (c.err) {
    sv->solved = false;
    sv->side_valid = false;
    if (c.err & ERR_TIMEOUT) return fail(DMF_ERR_TIMEOUT, "a grid-barrier wait timed out");
    if (c.err & ERR_UNKNOWN_ARC) {
      // nothing was applied: lookup errors stop the launch before any change
      sv->solved = true;
      return fail(DMF_ERR_UNKNOWN_ARC, "update %d names an arc that is not in the graph", c.err_info);
    }
    if (c.err & ERR_DUP_ARC) {
      sv->solved = true;
      return fail(DMF_ERR_DUP_ARC, "update %d repeats an arc already in this batch", c.err_info);
    }
    if (c.err & ERR_BAD_UPDATE) {
      sv->solved = true;
      return fail(DMF_ERR_INVALID_ARG,
                  "update %d: vertex out of range, capacity outside [0, 2^30-1], or capacity + partner "
                  "capacity exceeds int32",
                  c.err_info);
    }
    if (c.err & ERR_NO_CONV) return fail(DMF_ERR_NO_CONVERGENCE, "no convergence after %d global relabels", c.err_info);
    return fail(DMF_ERR_CUDA, "device error flags 0x%x", c.err);
  }
  sv->solved = true;
  sv->side_valid = need_cut_valid;
  if (sv->inst_flow) {
    if (sv->use_active && (int)sv->flows.size() == sv->ninst) {
      for (int i = 0; i < sv->ninst; i++)
        if (sv->h_inst_active[i]) sv->flows[i] = sv->h_inst_flow[i];
    } else {
      sv->flows.assign(sv->h_inst_flow, sv->h_inst_flow + sv->ninst);
    }
    int64_t tot = 0;
    for (int64_t f : sv->flows) tot += f;
    sv->st.flow = tot;
  } else {
    sv->st.flow = c.flow;
    sv->flows.assign(1, c.flow);
  }
  if (flow) *flow = sv->st.flow;
  return ok();
}

int run_mode(dmf_solver *sv, int mode, int k, const int *d_src, const int *d_dst, const int *d_w, int64_t *flow,
             bool started) {
  if (!started) CK(cudaEventRecord(sv->ev0, sv->stream), "event record");
  int st = launch(sv, mode, k, d_src, d_dst, d_w);
  if (st) return st;
  return finish(sv, flow, sv->opts.variant == DMF_VARIANT_PP || mode == MODE_CUT);
}

int check_updates_args(dmf_solver *sv, int32_t k, const void *a, const void *b, const void *c) {
  if (!sv) return fail(DMF_ERR_INVALID_ARG, "null solver");
  if (k < 0 || (k > 0 && (!a || !b || !c))) return fail(DMF_ERR_INVALID_ARG, "bad update arrays");
  return DMF_OK;
}

// Host copy into pinned staging: pieces of 64 KiB over up to 8 threads for a
// large array (a single thread copies well below the DRAM bandwidth).
void stage_copy(int32_t *to, const int32_t *from, size_t count) {
  constexpr size_t kPiece = 16384;  // int32 elements
  const long pieces = (long)((count + kPiece - 1) / kPiece);
  if (pieces < 4) {
    std::memcpy(to, from, 4 * count);
    return;
  }
#pragma omp parallel for num_threads(8) schedule(static)
  for (long i = 0; i < pieces; i++) {
    const size_t b = (size_t)i * kPiece, e = std::min(count, b + kPiece);
    std::memcpy(to + b, from + b, 4 * (e - b));
  }
}

// Copies a host batch into the device staging buffers through pinned memory;
// each array's H2D starts while the next one is copied.  The solve's start
// event is recorded before the first H2D (the copies are part of its time).
int stage_batch(dmf_solver *sv, int32_t k, const int32_t *src, const int32_t *dst, const int32_t *w) {
  int st;
  CK(cudaSetDevice(sv->dev), "cudaSetDevice");
  if ((st = ensure_ubuf(sv, k)) || (st = ensure_host_ubuf(sv, k))) return st;
  const size_t K = (size_t)sv->kcap, HK = (size_t)sv->h_kcap;
  const int32_t *from[3] = {src, dst, w};
  for (int a = 0; a < 3; a++) {
    if (k > 0) stage_copy(sv->h_ubuf + a * HK, from[a], (size_t)k);
    if (a == 0) CK(cudaEventRecord(sv->ev0, sv->stream), "event record");
    if (k > 0)
      CK(cudaMemcpyAsync(sv->ubuf + a * K, sv->h_ubuf + a * HK, 4 * (size_t)k, cudaMemcpyHostToDevice, sv->stream),
         "H2D batch");
  }
  return DMF_OK;
}

int host_updates(dmf_solver *sv, int mode, int32_t k, const int32_t *src, const int32_t *dst, const int32_t *w,
                 int64_t *flow) {
  int st = check_updates_args(sv, k, src, dst, w);
  if (st) return st;
  if (mode == MODE_DYNAMIC && !sv->solved) return fail(DMF_ERR_NOT_SOLVED, "apply_updates before a solve");
  if ((st = stage_batch(sv, k, src, dst, w))) return st;
  const size_t K = (size_t)sv->kcap;
  return run_mode(sv, mode, k, sv->ubuf, sv->ubuf + K, sv->ubuf + 2 * K, flow, true);
}

// Feature sums of the staged batch, then the picker's decision (sched = null:
// features only, action 0).
int batch_features(dmf_solver *sv, dmf_sched *sched, int k, float *feat, int *action) {
  CK(cudaMemsetAsync(sv->facc, 0, sizeof(dmfs::FeatAcc), sv->stream), "memset features");
  if (k > 0) {
    const size_t K = (size_t)sv->kcap;
    const int blocks = std::min((k + 255) / 256, 4 * 148);
    k_features<<<blocks, 256, 0, sv->stream>>>(sv->off, sv->adj, sv->sidx, sv->cap, sv->res, sv->n, k, sv->ubuf,
                                               sv->ubuf + K, sv->ubuf + 2 * K, sv->facc);
    CK(cudaGetLastError(), "feature launch");
  }
  dmfs::FeatScalars sc;
  sc.k = (float)k;
  sc.m = (float)sv->m;
  sc.n = (float)sv->n;
  sc.last_flow = (float)sv->st.flow;
  sc.last_levels = (float)sv->st.bfs_levels;
  sc.last_outer = (float)sv->st.outer_iters;
  return dmf_sched_decide(sched, sv->facc, sc, sv->stream, sv->dev, feat, nullptr, action);
}

// Runs the staged batch under one of the DMF_ACTION_* schedules; the solver's
// own options are restored afterwards.
int apply_action(dmf_solver *sv, int action, int k, int64_t *flow) {
  const dmf_opts saved = sv->opts;
  const int saved_small = sv->small_deg;
  int mode = MODE_DYNAMIC;
  switch (action) {
    case DMF_ACTION_SHORT:
      sv->opts.relabel_interval = 2;
      sv->opts.flags |= DMF_FLAG_FIXED_INTERVAL;
      break;
    case DMF_ACTION_WARP:
      sv->opts.relabel_interval = 12;
      sv->opts.flags |= DMF_FLAG_FIXED_INTERVAL;
      sv->small_deg = 0;
      break;
    case DMF_ACTION_RECOMPUTE:
      mode = MODE_RECOMPUTE;
      break;
    default:
      break;
  }
  const size_t K = (size_t)sv->kcap;
  const int st = run_mode(sv, mode, k, sv->ubuf, sv->ubuf + K, sv->ubuf + 2 * K, flow, true);
  sv->opts = saved;
  sv->small_deg = saved_small;
  return st;
}

// Shared body of dmf_apply_updates_action / _scheduled (action < 0: ask sched).
int scheduled_updates(dmf_solver *sv, dmf_sched *sched, int action, int32_t k, const int32_t *src,
                      const int32_t *dst, const int32_t *w, int64_t *flow, int32_t *chosen) {
  int st = check_updates_args(sv, k, src, dst, w);
  if (st) return st;
  if (!sv->solved) return fail(DMF_ERR_NOT_SOLVED, "apply_updates before a solve");
  if (action >= DMF_SCHED_ACTIONS) return fail(DMF_ERR_INVALID_ARG, "unknown action %d", action);
  if ((st = stage_batch(sv, k, src, dst, w))) return st;
  dmf_solver::SchedRecord rec{};
  int picked = 0;
  if ((st = batch_features(sv, action < 0 ? sched : nullptr, k, rec.feat, &picked))) return st;
  if (action >= 0) picked = action;
  int64_t f = 0;
  if ((st = apply_action(sv, picked, k, &f))) return st;
  rec.action = picked;
  rec.ms = (float)sv->st.last_ms;
  rec.flow = f;
  if (sv->records.size() < (1u << 20)) sv->records.push_back(rec);
  if (flow) *flow = f;
  if (chosen) *chosen = picked;
  return ok();
}

int device_updates(dmf_solver *sv, int mode, int32_t k, const int32_t *src, const int32_t *dst, const int32_t *w,
                   int64_t *flow) {
  int st = check_updates_args(sv, k, src, dst, w);
  if (st) return st;
  if (mode == MODE_DYNAMIC && !sv->solved) return fail(DMF_ERR_NOT_SOLVED, "apply_updates before a solve");
  CK(cudaSetDevice(sv->dev), "cudaSetDevice");
  if ((st = ensure_ubuf(sv, k))) return st;  // for the per-update arc scratch
  return run_mode(sv, mode, k, src, dst, w, flow, false);
}

// ---- allocation-free static solve ------------------------------------------------
// Some callers cannot allocate device memory while they run: code inside a
// pre-sized memory pool or arena, a host that forbids cudaMalloc after start-up,
// or a deployment that must never grow its footprint mid-flight.  For them
// dmf_static_maxflow_noalloc keeps all solver scratch (control block, labels,
// excess, stamps, dead/side marks, vertex queues) in the file-scope array below
// instead of memory the library allocates; the caller supplies the graph and
// the residual output in its own device memory.  The array is sized for
// kNoAllocMaxVertices vertices (about 10 MiB); every GPU that loads the library
// holds it until the process exits.
constexpr int kNoAllocMaxVertices = 1 << 18;
constexpr size_t kNoAllocAlign = 256;
constexpr size_t na_round(size_t b) { return (b + kNoAllocAlign - 1) / kNoAllocAlign * kNoAllocAlign; }
constexpr size_t kNoAllocV = (size_t)kNoAllocMaxVertices + 1;
constexpr size_t kNoAllocBytes = na_round(sizeof(Ctrl)) + na_round(4 * kNoAllocV) /* height */ +
                                 na_round(4 * kNoAllocV) /* stamp */ + na_round(8 * kNoAllocV) /* excess */ +
                                 na_round(kNoAllocV) /* dead */ + na_round(kNoAllocV) /* side */ +
                                 5 * na_round(4 * kNoAllocV) /* queues */ + 4 * kNoAllocAlign /* unused hub slots */ +
                                 kNoAllocAlign /* source list */;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch, looked up once per device (the name is
// only a host-side stand-in for the array; a kernel must be given this address).
std::mutex g_noalloc_mu;
void *g_noalloc_addr[128] = {};

int noalloc_scratch(int dev, unsigned char **out) {
  if (dev < 0 || dev >= 128) return fail(DMF_ERR_CUDA, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) return cuda_fail(e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress");
    g_noalloc_addr[dev] = ptr;
  }
  *out = (unsigned char *)g_noalloc_addr[dev];
  return DMF_OK;
}

}  // namespace

extern "C" {

int dmf_static_maxflow_noalloc(int32_t n, int32_t m, const int32_t *d_index, const int32_t *d_adj,
                               const int32_t *d_cap, const int32_t *d_par, int32_t s, int32_t t, int32_t *d_res,
                               int64_t *flow, void *stream) {
  if (n < 2 || m < 0 || !d_index || !flow || (m > 0 && (!d_adj || !d_cap || !d_par || !d_res)))
    return fail(DMF_ERR_INVALID_ARG, "bad arguments");
  if (n > kNoAllocMaxVertices)
    return fail(DMF_ERR_INVALID_ARG, "n=%d exceeds the %d vertices the allocation-free scratch holds", n,
                kNoAllocMaxVertices);
  if (s < 0 || t < 0 || s >= n || t >= n || s == t)
    return fail(DMF_ERR_INVALID_ARG, "need distinct s, t in [0, n): s=%d t=%d", s, t);
  int dev = 0;
  CK(cudaGetDevice(&dev), "cudaGetDevice");
  unsigned char *base = nullptr;
  int st = noalloc_scratch(dev, &base);
  if (st) return st;
  const int tile = n > 0 && (double)m / n <= 6 ? 4 : (double)m / n <= 12 ? 8 : (double)m / n <= 24 ? 16 : 32;
  KernelFn fn = pick_kernel(tile, 2);
  int per_sm = 0, sms = 0, coop = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)fn, kBlock, 0), "occupancy");
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "sm count");
  CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev), "coop attr");
  if (!coop || per_sm < 1) return fail(DMF_ERR_CUDA, "device does not support cooperative launch of the solver");
  // carve the scratch
  size_t off = 0;
  auto carve = [&](size_t bytes) {
    unsigned char *q = base + off;
    off += na_round(bytes);
    return q;
  };
  const size_t N = (size_t)n + 1;
  Ctrl *ctrl = (Ctrl *)carve(sizeof(Ctrl));
  Params p{};
  p.height = (int *)carve(4 * N);
  p.stamp = (int *)carve(4 * N);
  p.excess = (long long *)carve(8 * N);
  p.dead = carve(N);
  p.side = carve(N);
  p.fq[0] = (int *)carve(4 * N);
  p.fq[1] = (int *)carve(4 * N);
  p.wq[0] = (int *)carve(4 * N);
  p.wq[1] = (int *)carve(4 * N);
  p.aq = (int *)carve(4 * N);
  // no hubs in this mode (hub_deg = INT_MAX): the hub structures are never read
  int2 *hub_dummy = (int2 *)carve(kNoAllocAlign);
  long long *ll_dummy = (long long *)carve(kNoAllocAlign);
  int *int_dummy = (int *)carve(kNoAllocAlign);
  unsigned long long *mark_dummy = (unsigned long long *)carve(kNoAllocAlign);
  int *src_list = (int *)carve(kNoAllocAlign);
  if (off > kNoAllocBytes) return fail(DMF_ERR_CUDA, "internal: scratch layout exceeds the array");
  p.srcs = src_list;  // one source; filled below by a plain copy (no allocation)
  p.nsrc = 1;
  p.role = nullptr;
  p.inst = nullptr;
  p.inst_flow = nullptr;
  p.fh[0] = p.fh[1] = p.wh[0] = p.wh[1] = p.ah = hub_dummy;
  p.hch = hub_dummy;
  p.nhch = 0;
  p.hc_moved = p.hc_alloc = ll_dummy;
  p.hc_min = p.hc_done = int_dummy;
  p.hub_base = int_dummy;
  p.chunk_mark = mark_dummy;
  p.chunk_tmin = int_dummy;
  p.n = n;
  p.m = m;
  p.s = s;
  p.t = t;
  p.off = d_index;
  p.adj = d_adj;
  p.par = d_par;
  p.sidx = nullptr;
  p.cap = const_cast<int *>(d_cap);  // read only in static mode
  p.res = d_res;
  p.astamp = nullptr;
  p.uarc = nullptr;
  p.ctrl = ctrl;
  p.mode = MODE_STATIC;
  p.variant = DMF_VARIANT_DATA;
  p.cycles = 2;
  p.interval = 6;
  p.max_iters = 100000;
  p.hub_deg = INT_MAX;
  p.small_deg = 8;
  p.bu_alpha = 2;
  p.need_cut = 0;
  p.round_base = 1;
  p.relabel_base = 1;
  p.epoch = 1;
  p.trace = nullptr;
  p.trace_cap = 0;
  p.probe = 0;
  cudaStream_t S = (cudaStream_t)stream;
  // the array keeps the previous call's contents: the control block and the
  // worklist stamps must start at zero (everything else is written before use)
  CK(cudaMemsetAsync(ctrl, 0, sizeof(Ctrl), S), "memset control");
  CK(cudaMemsetAsync(p.stamp, 0, 4 * N, S), "memset stamps");
  const int32_t src_host = s;
  CK(cudaMemcpyAsync(src_list, &src_host, sizeof(src_host), cudaMemcpyHostToDevice, S), "H2D source");
  void *args[] = {&p};
  CK(cudaLaunchCooperativeKernel((const void *)fn, dim3(per_sm * sms), dim3(kBlock), args, 0, S),
     "cooperative launch");
  Ctrl hc;
  CK(cudaMemcpyAsync(&hc, ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, S), "D2H control");
  CK(cudaStreamSynchronize(S), "solve");
  if (hc.err & ERR_TIMEOUT) return fail(DMF_ERR_TIMEOUT, "a grid-barrier wait timed out");
  if (hc.err & ERR_NO_CONV) return fail(DMF_ERR_NO_CONVERGENCE, "no convergence");
  if (hc.err) return fail(DMF_ERR_CUDA, "device error flags 0x%x", hc.err);
  *flow = hc.flow;
  return ok();
}

int dmf_device_count(void) {
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return c;
}

}  // extern "C"

namespace {

struct MultiSpec {
  int count = 0;
  std::vector<int> vbase, srcs;
  std::vector<unsigned char> role;
  std::vector<int> inst;
};

int setup_solver(dmf_solver *sv, const dmf_graph *g, int32_t s, int32_t t, const dmf_opts *opts, void *stream,
                 const MultiSpec *ms);

int create_impl(const dmf_graph *g, int32_t s, int32_t t, const dmf_opts *opts, void *stream, const MultiSpec *ms,
                dmf_solver **out) {
  if (!g || !out) return fail(DMF_ERR_INVALID_ARG, "null argument");
  if (g->n < 2 || s < 0 || t < 0 || s >= g->n || t >= g->n || s == t)
    return fail(DMF_ERR_INVALID_ARG, "need n >= 2 and distinct s, t in [0, n): n=%d s=%d t=%d", g->n, s, t);
  if ((int64_t)g->sidx.size() != g->m) return fail(DMF_ERR_INVALID_ARG, "graph has no arc index");
  int ndev = dmf_device_count();
  if (ndev == 0) return fail(DMF_ERR_CUDA, "no CUDA device is visible; the solver runs only on the GPU");
  if (opts && (opts->variant < 0 || opts->variant > 2))
    return fail(DMF_ERR_INVALID_ARG, "unknown variant %d", opts->variant);
  dmf_solver *sv = nullptr;
  const int st = guarded([&]() -> int {
    sv = new dmf_solver();
    return setup_solver(sv, g, s, t, opts, stream, ms);
  });
  if (st) {
    if (sv) {
      char msg[1024];
      std::snprintf(msg, sizeof msg, "%s", dmf_last_error());
      free_all(sv);
      delete sv;
      fail(st, "%s", msg);
    }
    return st;
  }
  *out = sv;
  return ok();
}

// Fills a new solver: device arrays, hub chunks, sources.  On failure the
// caller frees what was allocated (free_all).
int setup_solver(dmf_solver *sv, const dmf_graph *g, int32_t s, int32_t t, const dmf_opts *opts, void *stream,
                 const MultiSpec *ms) {
  if (opts) sv->opts = *opts;
  else dmf_opts_default(&sv->opts);
  sv->n = g->n;
  sv->m = g->m;
  sv->s = s;
  sv->t = t;
  sv->stream = (cudaStream_t)stream;
  int st = DMF_OK;
  if (sv->opts.device >= 0) sv->dev = sv->opts.device;
  else if (cudaGetDevice(&sv->dev) != cudaSuccess) return cuda_fail(cudaGetLastError(), "cudaGetDevice");
  if (cudaSetDevice(sv->dev) != cudaSuccess) return cuda_fail(cudaGetLastError(), "cudaSetDevice");
  if ((st = configure(sv))) return st;
  const size_t N = (size_t)g->n + 1, M = (size_t)g->m;
  if ((st = dalloc(sv, &sv->off, N)) || (st = dalloc(sv, &sv->adj, M)) || (st = dalloc(sv, &sv->par, M)) ||
      (st = dalloc(sv, &sv->sidx, M)) || (st = dalloc(sv, &sv->cap, M)) || (st = dalloc(sv, &sv->res, M)) ||
      (st = dalloc(sv, &sv->astamp, M)) || (st = dalloc(sv, &sv->height, N)) || (st = dalloc(sv, &sv->stamp, N)) ||
      (st = dalloc(sv, &sv->excess, N)) || (st = dalloc(sv, &sv->dead, N)) || (st = dalloc(sv, &sv->side, N)) ||
      (st = dalloc(sv, &sv->qbuf, 5 * N)) || (st = dalloc(sv, &sv->ctrl, 1)))
    return st;
  std::vector<int2> hub_chunks;
  std::vector<int> hub_base(g->n, -1);
  for (int v = 0; v < g->n; v++) {
    const int d = g->off[v + 1] - g->off[v];
    if (d > sv->hub_deg) {
      hub_base[v] = (int)hub_chunks.size();
      for (int c = 0; c * kChunk < d; c++) hub_chunks.push_back(make_int2(v, c));
    }
  }
  sv->nchunk = (int)hub_chunks.size();
  const size_t NC = (size_t)std::max(sv->nchunk, 1);
  if ((st = dalloc(sv, &sv->hqbuf, 5 * NC)) || (st = dalloc(sv, &sv->hch, NC)) ||
      (st = dalloc(sv, &sv->hc_moved, NC)) || (st = dalloc(sv, &sv->hc_alloc, NC)) ||
      (st = dalloc(sv, &sv->hc_min, NC)) || (st = dalloc(sv, &sv->hc_done, NC)) ||
      (st = dalloc(sv, &sv->hub_base, N)) || (st = dalloc(sv, &sv->chunk_mark, NC)) ||
      (st = dalloc(sv, &sv->chunk_tmin, NC)))
    return st;
  cudaStream_t S = sv->stream;
  cudaError_t e = cudaSuccess;
  auto up = [&](void *d, const void *h, size_t bytes) {
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, S);
  };
  up(sv->off, g->off.data(), 4 * N);
  up(sv->adj, g->adj.data(), 4 * M);
  up(sv->par, g->par.data(), 4 * M);
  up(sv->sidx, g->sidx.data(), 4 * M);
  up(sv->cap, g->w.data(), 4 * M);
  up(sv->hch, hub_chunks.data(), sizeof(int2) * hub_chunks.size());
  up(sv->hub_base, hub_base.data(), 4 * (size_t)g->n);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->chunk_mark, 0, 8 * NC, S);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->astamp, 0, 4 * M, S);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->hc_done, 0, 4 * NC, S);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->hc_alloc, 0, 8 * NC, S);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->hc_moved, 0, 8 * NC, S);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->stamp, 0, 4 * N, S);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->dead, 0, N, S);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->side, 0, N, S);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->excess, 0, 8 * N, S);
  if (e == cudaSuccess) e = cudaMallocHost(&sv->h_ctrl, sizeof(Ctrl));
  if (e == cudaSuccess) e = cudaEventCreate(&sv->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&sv->ev1);
  if (e == cudaSuccess) e = cudaStreamSynchronize(S);
  if (e != cudaSuccess) return cuda_fail(e, "solver upload");
  if ((st = ensure_ubuf(sv, 1024))) return st;
  // sources (and, for batched instances, roles, instance ids, per-instance flows)
  {
    const std::vector<int> one(1, s);
    const std::vector<int> &sl = ms ? ms->srcs : one;
    sv->nsrc = (int)sl.size();
    sv->ninst = ms ? ms->count : 1;
    std::vector<int> so(sl.size() + 1, 0);
    for (size_t i = 0; i < sl.size(); i++) {
      const long long nx = (long long)so[i] + g->off[sl[i] + 1] - g->off[sl[i]];
      if (nx > INT_MAX) return fail(DMF_ERR_INVALID_ARG, "sources have more than 2^31 arcs in total");
      so[i + 1] = (int)nx;
    }
    if ((st = dalloc(sv, &sv->srcs, sl.size())) || (st = dalloc(sv, &sv->src_off, so.size()))) return st;
    if (cudaMemcpy(sv->srcs, sl.data(), 4 * sl.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(sv->src_off, so.data(), 4 * so.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return cuda_fail(cudaGetLastError(), "H2D sources");
    if (ms) {
      sv->vbase = ms->vbase;
      if ((st = dalloc(sv, &sv->role, N)) || (st = dalloc(sv, &sv->inst, N)) ||
          (st = dalloc(sv, &sv->inst_flow, (size_t)ms->count)) ||
          (st = dalloc(sv, &sv->inst_active, (size_t)ms->count)))
        return st;
      if (cudaMallocHost(&sv->h_inst_active, (size_t)ms->count) != cudaSuccess)
        return cuda_fail(cudaGetLastError(), "pinned mask");
      if (cudaMemcpy(sv->role, ms->role.data(), ms->role.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(sv->inst, ms->inst.data(), 4 * ms->inst.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMallocHost(&sv->h_inst_flow, 8 * (size_t)ms->count) != cudaSuccess)
        return cuda_fail(cudaGetLastError(), "batched-instance upload");
    }
  }
  sv->trace_cap = 1 << 16;
  if ((st = dalloc(sv, &sv->trace, 4 * (size_t)sv->trace_cap))) return st;
  if ((st = dalloc(sv, &sv->facc, 1))) return st;
  return ok();
}

}  // namespace

extern "C" {

int dmf_solver_create(const dmf_graph *g, int32_t s, int32_t t, const dmf_opts *opts, void *stream,
                      dmf_solver **out) {
  return create_impl(g, s, t, opts, stream, nullptr, out);
}

int dmf_multi_create(int32_t count, const dmf_graph *const *graphs, const int32_t *s, const int32_t *t,
                     const dmf_opts *opts, void *stream, dmf_solver **out) {
  if (count < 1 || !graphs || !s || !t || !out) return fail(DMF_ERR_INVALID_ARG, "bad arguments");
  int64_t N = 0, M = 0;
  for (int i = 0; i < count; i++) {
    const dmf_graph *g = graphs[i];
    if (!g || g->n < 2 || s[i] < 0 || t[i] < 0 || s[i] >= g->n || t[i] >= g->n || s[i] == t[i])
      return fail(DMF_ERR_INVALID_ARG, "instance %d: need a graph with n >= 2 and distinct s, t in [0, n)", i);
    if ((int64_t)g->sidx.size() != g->m) return fail(DMF_ERR_INVALID_ARG, "instance %d has no arc index", i);
    N += g->n;
    M += g->m;
  }
  if (N >= INT32_MAX || M >= INT32_MAX) return fail(DMF_ERR_INVALID_ARG, "union too large for int32 ids");
  return guarded([&]() -> int {
    dmf_graph U;
    U.n = (int32_t)N;
    U.m = (int32_t)M;
    U.off.resize((size_t)N + 1);
    U.adj.resize((size_t)M);
    U.w.resize((size_t)M);
    U.par.resize((size_t)M);
    U.sidx.resize((size_t)M);
    MultiSpec ms;
    ms.count = count;
    ms.vbase.resize((size_t)count + 1);
    ms.srcs.resize(count);
    ms.role.assign((size_t)N + 1, 0);
    ms.inst.resize((size_t)N + 1);
    std::vector<int64_t> abase((size_t)count + 1, 0);
    int64_t vb = 0;
    for (int i = 0; i < count; i++) {
      ms.vbase[i] = (int)vb;
      abase[i + 1] = abase[i] + graphs[i]->m;
      vb += graphs[i]->n;
    }
    ms.vbase[count] = (int)vb;
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < count; i++) {
      const dmf_graph &g = *graphs[i];
      const int vb_i = ms.vbase[i];
      const int ab = (int)abase[i];
      for (int v = 0; v < g.n; v++) {
        U.off[vb_i + v] = ab + g.off[v];
        ms.inst[vb_i + v] = i;
      }
      for (int e = 0; e < g.m; e++) {
        U.adj[ab + e] = vb_i + g.adj[e];
        U.w[ab + e] = g.w[e];
        U.par[ab + e] = ab + g.par[e];
        U.sidx[ab + e] = ab + g.sidx[e];
      }
    }
    U.off[N] = (int32_t)M;
    for (int i = 0; i < count; i++) {
      ms.srcs[i] = ms.vbase[i] + s[i];
      ms.role[ms.vbase[i] + s[i]] |= 1;
      ms.role[ms.vbase[i] + t[i]] |= 2;
    }
    return create_impl(&U, ms.srcs[0], ms.vbase[0] + t[0], opts, stream, &ms, out);
  });
}

int dmf_multi_info(const dmf_solver *sv, int32_t *count, int32_t *vertex_base) {
  if (!sv || !count) return fail(DMF_ERR_INVALID_ARG, "null argument");
  *count = sv->ninst;
  if (vertex_base) {
    if (sv->vbase.empty()) vertex_base[0] = 0;
    else for (int i = 0; i < sv->ninst; i++) vertex_base[i] = sv->vbase[i];
  }
  return ok();
}

int dmf_multi_static_maxflow(dmf_solver *sv, int64_t *flows) {
  if (!sv || !flows) return fail(DMF_ERR_INVALID_ARG, "null argument");
  int st = dmf_static_maxflow(sv, nullptr);
  if (st) return st;
  for (int i = 0; i < sv->ninst; i++) flows[i] = sv->flows[i];
  return ok();
}

int dmf_multi_apply_updates(dmf_solver *sv, int32_t k, const int32_t *inst, const int32_t *src, const int32_t *dst,
                            const int32_t *w, int64_t *flows) {
  return guarded([&]() -> int {
    if (!sv || !flows || k < 0 || (k > 0 && (!inst || !src || !dst || !w)))
      return fail(DMF_ERR_INVALID_ARG, "bad arguments");
    std::vector<int32_t> gs(k), gd(k);
    for (int32_t i = 0; i < k; i++) {
      const int in = inst[i];
      if (in < 0 || in >= sv->ninst) return fail(DMF_ERR_INVALID_ARG, "update %d: instance %d out of range", i, in);
      const int b = sv->vbase.empty() ? 0 : sv->vbase[in];
      const int nloc = sv->vbase.empty() ? sv->n : sv->vbase[in + 1] - b;
      if (src[i] < 0 || dst[i] < 0 || src[i] >= nloc || dst[i] >= nloc)
        return fail(DMF_ERR_INVALID_ARG, "update %d: vertex out of range for instance %d", i, in);
      gs[i] = b + src[i];
      gd[i] = b + dst[i];
    }
    // only the instances this batch touches are relabelled, pushed and read out
    if (sv->inst_active && (int)sv->flows.size() == sv->ninst && sv->solved) {
      std::memset(sv->h_inst_active, 0, (size_t)sv->ninst);
      for (int32_t i = 0; i < k; i++) sv->h_inst_active[inst[i]] = 1;
      CK(cudaMemcpyAsync(sv->inst_active, sv->h_inst_active, (size_t)sv->ninst, cudaMemcpyHostToDevice, sv->stream),
         "H2D mask");
      sv->use_active = true;
    }
    int st = host_updates(sv, MODE_DYNAMIC, k, gs.data(), gd.data(), w, nullptr);
    sv->use_active = false;
    if (st) return st;
    for (int i = 0; i < sv->ninst; i++) flows[i] = sv->flows[i];
    return ok();
  });
}

int dmf_multi_run_batches(dmf_solver *sv, int32_t steps, const int64_t *ofs, const int32_t *d_src,
                          const int32_t *d_dst, const int32_t *d_w, int32_t use_graph, int64_t *flows, double *ms) {
  return guarded([&]() -> int {
    if (!sv || steps < 1 || !ofs || !flows || !d_src || !d_dst || !d_w) return fail(DMF_ERR_INVALID_ARG, "bad arguments");
    if (!sv->solved) return fail(DMF_ERR_NOT_SOLVED, "run_batches before a solve");
    CK(cudaSetDevice(sv->dev), "cudaSetDevice");
    int64_t kmax = 0;
    for (int b = 0; b < steps; b++) {
      if (ofs[b + 1] < ofs[b]) return fail(DMF_ERR_INVALID_ARG, "offsets decrease at step %d", b);
      kmax = std::max(kmax, ofs[b + 1] - ofs[b]);
    }
    if (kmax > INT32_MAX) return fail(DMF_ERR_INVALID_ARG, "batch too large");
    int st = ensure_ubuf(sv, (int)kmax);
    if (st) return st;
    cudaStream_t S = sv->stream;
    if (use_graph && !S) {  // the legacy default stream cannot be captured
      if (!sv->own_stream) CK(cudaStreamCreateWithFlags(&sv->own_stream, cudaStreamNonBlocking), "stream create");
      CK(cudaStreamSynchronize(nullptr), "sync");
      S = sv->own_stream;
    }
    const int cnt = sv->ninst;
    Ctrl *h_ctrl = nullptr;
    long long *h_fl = nullptr;
    CK(cudaMallocHost(&h_ctrl, sizeof(Ctrl) * (size_t)steps), "pinned control");
    if (cudaMallocHost(&h_fl, 8 * (size_t)steps * cnt) != cudaSuccess) {
      cudaFreeHost(h_ctrl);
      return fail(DMF_ERR_OOM, "pinned flows");
    }
    // step b uses its own range of round ids, relabel epochs and batch stamp
    constexpr unsigned kRoundStride = 1u << 20, kRelabelStride = 1u << 18;
    KernelFn fn = pick_kernel(sv->tile, sv->minb);
    auto enqueue_steps = [&]() -> cudaError_t {
      for (int b = 0; b < steps; b++) {
        Params p = make_params(sv, MODE_DYNAMIC, (int)(ofs[b + 1] - ofs[b]), d_src + ofs[b], d_dst + ofs[b],
                               d_w + ofs[b]);
        p.round_base = sv->round_base + (unsigned)b * kRoundStride;
        p.relabel_base = sv->relabel_base + (unsigned)b * kRelabelStride;
        p.trace = nullptr;
        p.probe = 0;
        cudaError_t e = cudaMemsetAsync(sv->ctrl, 0, sizeof(Ctrl), S);
        if (e == cudaSuccess && sv->inst_flow) e = cudaMemsetAsync(sv->inst_flow, 0, 8 * (size_t)cnt, S);
        if (e != cudaSuccess) return e;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(sv->grid);
        cfg.blockDim = dim3(sv->block);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = S;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelEx(&cfg, fn, p);
        if (e != cudaSuccess) return e;
        e = cudaMemcpyAsync(h_ctrl + b, sv->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, S);
        if (e == cudaSuccess) {
          if (sv->inst_flow)
            e = cudaMemcpyAsync(h_fl + (size_t)b * cnt, sv->inst_flow, 8 * (size_t)cnt, cudaMemcpyDeviceToHost, S);
          else
            e = cudaMemcpyAsync(h_fl + b, &sv->ctrl->flow, 8, cudaMemcpyDeviceToHost, S);
        }
        if (e != cudaSuccess) return e;
      }
      return cudaSuccess;
    };
    cudaError_t e = cudaSuccess;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (use_graph) {
      e = cudaStreamBeginCapture(S, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        cudaError_t e2 = enqueue_steps();
        e = cudaStreamEndCapture(S, &graph);
        if (e2 != cudaSuccess) e = e2;
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    }
    if (e == cudaSuccess) e = cudaEventRecord(sv->ev0, S);
    if (e == cudaSuccess) e = use_graph ? cudaGraphLaunch(exec, S) : enqueue_steps();
    if (e == cudaSuccess) e = cudaEventRecord(sv->ev1, S);
    if (e == cudaSuccess) e = cudaEventSynchronize(sv->ev1);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      cudaFreeHost(h_ctrl);
      cudaFreeHost(h_fl);
      return cuda_fail(e, use_graph ? "graph-captured batch loop" : "batch loop");
    }
    float t_ms = 0;
    cudaEventElapsedTime(&t_ms, sv->ev0, sv->ev1);
    if (ms) *ms = t_ms;
    int rc = DMF_OK;
    unsigned outer = 0;
    for (int b = 0; b < steps && !rc; b++) {
      const Ctrl &c = h_ctrl[b];
      outer += (unsigned)c.st_outer;
      if (c.err) rc = fail(c.err & ERR_TIMEOUT ? DMF_ERR_TIMEOUT
                           : c.err & ERR_NO_CONV ? DMF_ERR_NO_CONVERGENCE
                           : c.err & (ERR_UNKNOWN_ARC | ERR_DUP_ARC | ERR_BAD_UPDATE) ? DMF_ERR_INVALID_ARG
                                                                                      : DMF_ERR_CUDA,
                           "step %d: device error flags 0x%x (update %d)", b, c.err, c.err_info);
    }
    for (size_t i = 0; i < (size_t)steps * cnt; i++) flows[i] = h_fl[i];
    sv->round_base += (unsigned)steps * kRoundStride;
    sv->relabel_base += (unsigned)steps * kRelabelStride;
    if (!rc) {
      sv->flows.assign(h_fl + (size_t)(steps - 1) * cnt, h_fl + (size_t)steps * cnt);
      int64_t tot = 0;
      for (int64_t f : sv->flows) tot += f;
      sv->st.flow = tot;
      sv->st.last_ms = t_ms;
      sv->st.outer_iters = outer;
      sv->side_valid = false;
    } else {
      sv->solved = false;
    }
    cudaFreeHost(h_ctrl);
    cudaFreeHost(h_fl);
    return rc ? rc : ok();
  });
}

int dmf_autotune(dmf_solver *sv, int32_t repeats, dmf_opts *chosen) {
  return guarded([&]() -> int {
    if (!sv) return fail(DMF_ERR_INVALID_ARG, "null solver");
    if (repeats < 1) repeats = 1;
    dmf_opts best = sv->opts;
    auto cost = [&](const dmf_opts &o, double *out) -> int {
      sv->opts = o;
      int st = configure(sv);
      if (st) return st;
      double b = 1e30;
      for (int r = 0; r < repeats; r++) {
        st = host_updates(sv, MODE_RECOMPUTE, 0, nullptr, nullptr, nullptr, nullptr);
        if (st) return st;
        b = std::min(b, sv->st.last_ms);
      }
      *out = b;
      return DMF_OK;
    };
    double best_ms = 0;
    int st = cost(best, &best_ms);
    if (st) return st;
    auto try_dim = [&](int32_t dmf_opts::*field, std::initializer_list<int32_t> vals) -> int {
      for (int32_t v : vals) {
        dmf_opts o = best;
        if (o.*field == v) continue;
        o.*field = v;
        double ms = 0;
        int s2 = cost(o, &ms);
        if (s2) return s2;
        if (ms < best_ms) {
          best_ms = ms;
          best = o;
        }
      }
      return DMF_OK;
    };
    if ((st = try_dim(&dmf_opts::tile, {4, 8, 16, 32})) || (st = try_dim(&dmf_opts::small_deg, {-1, 4, 8, 16, 32})) ||
        (st = try_dim(&dmf_opts::relabel_interval, {2, 3, 6, 12})) || (st = try_dim(&dmf_opts::kernel_cycles, {1, 2, 4})))
      return st;
    sv->opts = best;
    if ((st = configure(sv))) return st;
    st = host_updates(sv, MODE_RECOMPUTE, 0, nullptr, nullptr, nullptr, nullptr);  // leave a solved state
    if (st) return st;
    if (chosen) *chosen = best;
    return ok();
  });
}

int dmf_solver_set_opts(dmf_solver *sv, const dmf_opts *opts) {
  return guarded([&]() -> int {
    if (!sv || !opts) return fail(DMF_ERR_INVALID_ARG, "null argument");
    if (opts->variant < 0 || opts->variant > 2) return fail(DMF_ERR_INVALID_ARG, "unknown variant");
    bool variant_changed = opts->variant != sv->opts.variant;
    sv->opts = *opts;
    if (cudaSetDevice(sv->dev) != cudaSuccess) return cuda_fail(cudaGetLastError(), "cudaSetDevice");
    int st = configure(sv);
    if (st) return st;
    if (variant_changed) sv->side_valid = false;
    return ok();
  });
}

int dmf_static_maxflow(dmf_solver *sv, int64_t *flow) {
  return guarded([&]() -> int {
    if (!sv) return fail(DMF_ERR_INVALID_ARG, "null solver");
    CK(cudaSetDevice(sv->dev), "cudaSetDevice");
    return run_mode(sv, MODE_STATIC, 0, nullptr, nullptr, nullptr, flow, false);
  });
}

int dmf_apply_updates(dmf_solver *sv, int32_t k, const int32_t *src, const int32_t *dst, const int32_t *w,
                      int64_t *flow) {
  return guarded([&]() -> int {
    return host_updates(sv, MODE_DYNAMIC, k, src, dst, w, flow);
  });
}

int dmf_apply_updates_device(dmf_solver *sv, int32_t k, const int32_t *d_src, const int32_t *d_dst,
                             const int32_t *d_w, int64_t *flow) {
  return guarded([&]() -> int {
    return device_updates(sv, MODE_DYNAMIC, k, d_src, d_dst, d_w, flow);
  });
}

int dmf_recompute(dmf_solver *sv, int32_t k, const int32_t *src, const int32_t *dst, const int32_t *w,
                  int64_t *flow) {
  return guarded([&]() -> int {
    return host_updates(sv, MODE_RECOMPUTE, k, src, dst, w, flow);
  });
}

int dmf_recompute_device(dmf_solver *sv, int32_t k, const int32_t *d_src, const int32_t *d_dst,
                         const int32_t *d_w, int64_t *flow) {
  return guarded([&]() -> int {
    return device_updates(sv, MODE_RECOMPUTE, k, d_src, d_dst, d_w, flow);
  });
}

int dmf_flow_value(const dmf_solver *sv, int64_t *flow) {
  if (!sv || !flow) return fail(DMF_ERR_INVALID_ARG, "null argument");
  if (!sv->solved) return fail(DMF_ERR_NOT_SOLVED, "no solve yet");
  *flow = sv->st.flow;
  return ok();
}

int dmf_get_cut(dmf_solver *sv, uint8_t *sink_side) {
  return guarded([&]() -> int {
    if (!sv || !sink_side) return fail(DMF_ERR_INVALID_ARG, "null argument");
    if (!sv->solved) return fail(DMF_ERR_NOT_SOLVED, "no solve yet");
    CK(cudaSetDevice(sv->dev), "cudaSetDevice");
    if (!sv->side_valid) {
      int64_t f = sv->st.flow;
      dmf_stats keep = sv->st;
      int st = run_mode(sv, MODE_CUT, 0, nullptr, nullptr, nullptr, nullptr, false);
      if (st) return st;
      sv->st = keep;
      sv->st.flow = f;
      sv->side_valid = true;
    }
    CK(cudaMemcpyAsync(sink_side, sv->side, (size_t)sv->n, cudaMemcpyDeviceToHost, sv->stream), "D2H cut");
    CK(cudaStreamSynchronize(sv->stream), "cut");
    return ok();
  });
}

int dmf_get_state(dmf_solver *sv, int32_t *cap, int32_t *res, int64_t *excess, int32_t *height) {
  if (!sv) return fail(DMF_ERR_INVALID_ARG, "null solver");
  CK(cudaSetDevice(sv->dev), "cudaSetDevice");
  const size_t M = (size_t)sv->m, N = (size_t)sv->n;
  if (cap) CK(cudaMemcpyAsync(cap, sv->cap, 4 * M, cudaMemcpyDeviceToHost, sv->stream), "D2H cap");
  if (res) CK(cudaMemcpyAsync(res, sv->res, 4 * M, cudaMemcpyDeviceToHost, sv->stream), "D2H res");
  if (excess) CK(cudaMemcpyAsync(excess, sv->excess, 8 * N, cudaMemcpyDeviceToHost, sv->stream), "D2H excess");
  if (height) CK(cudaMemcpyAsync(height, sv->height, 4 * N, cudaMemcpyDeviceToHost, sv->stream), "D2H height");
  CK(cudaStreamSynchronize(sv->stream), "state");
  return ok();
}

int dmf_trace_items(dmf_solver *sv, int32_t cap, int64_t *items, int64_t *hubs, int64_t *slow_ns,
                    int64_t *slow_v) {
  return guarded([&]() -> int {
    if (!sv || cap < 0 || (cap > 0 && (!items || !hubs))) return fail(DMF_ERR_INVALID_ARG, "bad arguments");
    const int len = std::min(std::min(sv->h_ctrl ? sv->h_ctrl->trace_len : 0, sv->trace_cap), cap);
    if (len <= 0) return ok();
    std::vector<unsigned long long> h(4 * (size_t)len);
    CK(cudaSetDevice(sv->dev), "cudaSetDevice");
    CK(cudaMemcpyAsync(h.data(), sv->trace, 32 * (size_t)len, cudaMemcpyDeviceToHost, sv->stream), "D2H trace");
    CK(cudaStreamSynchronize(sv->stream), "trace");
    for (int i = 0; i < len; i++) {
      items[i] = (int64_t)((h[4 * i] >> 8) & 0xffffffffull);
      hubs[i] = (int64_t)(h[4 * i] >> 40);
      if (slow_ns) slow_ns[i] = (int64_t)(h[4 * i + 2] >> 32);
      if (slow_v) slow_v[i] = (int64_t)(h[4 * i + 2] & 0xffffffffull);
    }
    return ok();
  });
}

int dmf_trace_blocks(dmf_solver *sv, int32_t cap, int64_t *block_ns) {
  return guarded([&]() -> int {
    if (!sv || cap < 0 || (cap > 0 && !block_ns)) return fail(DMF_ERR_INVALID_ARG, "bad arguments");
    const int len = std::min(std::min(sv->h_ctrl ? sv->h_ctrl->trace_len : 0, sv->trace_cap), cap);
    if (len <= 0) return ok();
    std::vector<unsigned long long> h(4 * (size_t)len);
    CK(cudaSetDevice(sv->dev), "cudaSetDevice");
    CK(cudaMemcpyAsync(h.data(), sv->trace, 32 * (size_t)len, cudaMemcpyDeviceToHost, sv->stream), "D2H trace");
    CK(cudaStreamSynchronize(sv->stream), "trace");
    for (int i = 0; i < len; i++) block_ns[i] = (int64_t)h[4 * i + 3];
    return ok();
  });
}

int dmf_trace_get(dmf_solver *sv, int32_t cap, int32_t *kinds, double *t_us, int32_t *count) {
  return guarded([&]() -> int {
    if (!sv || !count || cap < 0 || (cap > 0 && (!kinds || !t_us))) return fail(DMF_ERR_INVALID_ARG, "bad arguments");
    const int len = std::min(sv->h_ctrl ? sv->h_ctrl->trace_len : 0, sv->trace_cap);
    *count = len;
    if (len == 0 || cap == 0) return ok();
    std::vector<unsigned long long> h(4 * (size_t)len);
    CK(cudaSetDevice(sv->dev), "cudaSetDevice");
    CK(cudaMemcpyAsync(h.data(), sv->trace, 32 * (size_t)len, cudaMemcpyDeviceToHost, sv->stream), "D2H trace");
    CK(cudaStreamSynchronize(sv->stream), "trace");
    for (int i = 0; i < std::min(len, cap); i++) {
      kinds[i] = (int32_t)(h[4 * i] & 0xff);
      t_us[i] = (double)(h[4 * i + 1] - h[1]) * 1e-3;
    }
    return ok();
  });
}

int dmf_stats_get(const dmf_solver *sv, dmf_stats *st) {
  if (!sv || !st) return fail(DMF_ERR_INVALID_ARG, "null argument");
  *st = sv->st;
  return ok();
}

int dmf_solver_features(dmf_solver *sv, int32_t k, const int32_t *src, const int32_t *dst, const int32_t *w,
                        float *feat) {
  return guarded([&]() -> int {
    int st = check_updates_args(sv, k, src, dst, w);
    if (st) return st;
    if (!feat) return fail(DMF_ERR_INVALID_ARG, "null feature output");
    if ((st = stage_batch(sv, k, src, dst, w))) return st;
    int action = 0;
    if ((st = batch_features(sv, nullptr, k, feat, &action))) return st;
    return ok();
  });
}

int dmf_apply_updates_action(dmf_solver *sv, int32_t action, int32_t k, const int32_t *src, const int32_t *dst,
                             const int32_t *w, int64_t *flow) {
  return guarded([&]() -> int {
    if (action < 0) return fail(DMF_ERR_INVALID_ARG, "unknown action %d", action);
    return scheduled_updates(sv, nullptr, action, k, src, dst, w, flow, nullptr);
  });
}

int dmf_apply_updates_scheduled(dmf_solver *sv, dmf_sched *sched, int32_t k, const int32_t *src, const int32_t *dst,
                                const int32_t *w, int64_t *flow, int32_t *action) {
  return guarded([&]() -> int {
    return scheduled_updates(sv, sched, -1, k, src, dst, w, flow, action);
  });
}

int dmf_sched_records(dmf_solver *sv, int32_t cap, float *feat, int32_t *action, float *ms, int64_t *flow,
                      int32_t *count) {
  if (!sv || cap < 0 || !count) return fail(DMF_ERR_INVALID_ARG, "bad arguments");
  const int n = (int)std::min<size_t>((size_t)cap, sv->records.size());
  for (int i = 0; i < n; i++) {
    const auto &r = sv->records[i];
    if (feat) std::memcpy(feat + (size_t)i * DMF_SCHED_FEATURES, r.feat, sizeof(r.feat));
    if (action) action[i] = r.action;
    if (ms) ms[i] = r.ms;
    if (flow) flow[i] = r.flow;
  }
  sv->records.erase(sv->records.begin(), sv->records.begin() + n);
  *count = n;
  return ok();
}

int dmf_solver_copy_state(dmf_solver *dst, const dmf_solver *src) {
  return guarded([&]() -> int {
    if (!dst || !src) return fail(DMF_ERR_INVALID_ARG, "null solver");
    if (dst == src) return ok();
    if (dst->n != src->n || dst->m != src->m || dst->hub_deg != src->hub_deg || dst->nchunk != src->nchunk ||
        dst->ninst != 1 || src->ninst != 1 || dst->dev != src->dev)
      return fail(DMF_ERR_INVALID_ARG, "copy_state needs two single-instance solvers of the same graph, hub "
                                       "threshold and device");
    CK(cudaSetDevice(dst->dev), "cudaSetDevice");
    CK(cudaStreamSynchronize(src->stream), "source solver");
    const size_t N = (size_t)src->n + 1, M = (size_t)src->m, NC = (size_t)std::max(src->nchunk, 1);
    cudaStream_t S = dst->stream;
    CK(cudaMemcpyAsync(dst->cap, src->cap, 4 * M, cudaMemcpyDeviceToDevice, S), "D2D cap");
    CK(cudaMemcpyAsync(dst->res, src->res, 4 * M, cudaMemcpyDeviceToDevice, S), "D2D res");
    CK(cudaMemcpyAsync(dst->astamp, src->astamp, 4 * M, cudaMemcpyDeviceToDevice, S), "D2D astamp");
    CK(cudaMemcpyAsync(dst->excess, src->excess, 8 * N, cudaMemcpyDeviceToDevice, S), "D2D excess");
    CK(cudaMemcpyAsync(dst->height, src->height, 4 * N, cudaMemcpyDeviceToDevice, S), "D2D height");
    CK(cudaMemcpyAsync(dst->stamp, src->stamp, 4 * N, cudaMemcpyDeviceToDevice, S), "D2D stamp");
    CK(cudaMemcpyAsync(dst->dead, src->dead, N, cudaMemcpyDeviceToDevice, S), "D2D dead");
    CK(cudaMemcpyAsync(dst->side, src->side, N, cudaMemcpyDeviceToDevice, S), "D2D side");
    CK(cudaMemcpyAsync(dst->chunk_mark, src->chunk_mark, 8 * NC, cudaMemcpyDeviceToDevice, S), "D2D marks");
    CK(cudaMemcpyAsync(dst->chunk_tmin, src->chunk_tmin, 4 * NC, cudaMemcpyDeviceToDevice, S), "D2D marks");
    CK(cudaStreamSynchronize(S), "copy state");
    dst->round_base = src->round_base;
    dst->relabel_base = src->relabel_base;
    dst->epoch = src->epoch;
    dst->solved = src->solved;
    dst->side_valid = src->side_valid;
    dst->st = src->st;
    dst->flows = src->flows;
    return ok();
  });
}

int dmf_solver_destroy(dmf_solver *sv) {
  if (!sv) return ok();
  if (sv->ubuf) {
    cudaSetDevice(sv->dev);
    if (sv->stream) cudaStreamSynchronize(sv->stream);
    cudaFree(sv->ubuf);
    sv->ubuf = nullptr;
  }
  free_all(sv);
  delete sv;
  return ok();
}

}  // extern "C"
