// dmf_solver.cu -- host side of the solver in libdmf.so: device state, launch
// of the persistent sm_100a kernel (dmf_kernel.cuh), the batch feature kernel
// of the schedule picker, and the solver entry points of the C ABI.
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "dmf_kernel.cuh"
#include "dmf_internal.h"
#include "dmf_sched_internal.h"

using namespace dmfd;
using namespace dmfk;

namespace {

// Raw feature sums of an update batch against the current residual state, for
// the schedule picker (nothing is modified).  Updates the solver would reject
// (bad ids, unknown arcs) are skipped here; the solve reports them.
__global__ void __launch_bounds__(256) k_features(const int *__restrict__ off, const ArcSlot *atab,
                                                  long long nslots, const unsigned long long *capx, const int *res,
                                                  int n,
                                                  int k, const int *usrc, const int *udst, const int *uw,
                                                  dmfs::FeatAcc *acc) {
  unsigned long long valid = 0, dec = 0, satdec = 0, incsat = 0, ins = 0, del = 0, sdeg = 0, mdeg = 0;
  long long exc = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
    const int u = __ldg(usrc + i), v = __ldg(udst + i), w = __ldg(uw + i);
    if (u < 0 || u >= n || v < 0 || v >= n || u == v) continue;
    const int e = find_arc_table(atab, nslots, u, v);
    if (e < 0) continue;
    valid++;
    const int c0 = (int)(unsigned)__ldcg(capx + e), r = __ldcg(res + e);
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

// minb = resident blocks per SM the register budget is sized for (1: up to 128
// registers a thread, 2: up to 64).
KernelFn pick_kernel(int tile, int minb) {
  switch (tile) {
    case 4: return solve_kernel_t4(minb);
    case 8: return solve_kernel_t8(minb);
    case 16: return solve_kernel_t16(minb);
    default: return solve_kernel_t32(minb);
  }
}

}  // namespace

// ============================================================================
// host side
// ============================================================================
using dmf::fail;
using dmf::ok;
using dmf::guarded;

// Fills the arc table: a warp per tail vertex of degree <= hub_deg (a lane per
// arc), and a warp per hub chunk (kChunk arcs of a longer row), so that one
// warp never walks a hub's whole row.  Equal (tail, head) pairs keep the
// largest arc index.  Every insert ends: the table has more slots than arcs,
// so an empty slot or the key is always found.
__device__ __forceinline__ void table_insert(ArcSlot *tab, long long nslots, int u, int v, int a) {
  const unsigned long long key = arc_key(u, v);
  long long sl = arc_slot0(u, v, nslots);
  for (long long probe = 0; probe < nslots; probe++) {
    const unsigned long long old = atomicCAS(reinterpret_cast<unsigned long long *>(tab + sl), ~0ull, key);
    if (old == ~0ull || old == key) {
      atomicMax(&tab[sl].arc, a);
      return;
    }
    sl = sl + 1 == nslots ? 0 : sl + 1;
  }
}

__global__ void __launch_bounds__(256) k_arc_table_build(const int *__restrict__ off, const int *__restrict__ adj,
                                                         int n, int hub_deg, const int2 *__restrict__ hch,
                                                         int nchunk, ArcSlot *tab, long long nslots) {
  const int lane = threadIdx.x & 31;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long u = warp; u < n; u += nwarps) {
    const int b = __ldg(off + u), e = __ldg(off + u + 1);
    if (e - b > hub_deg) continue;  // by chunks below
    for (int a = b + lane; a < e; a += 32) table_insert(tab, nslots, (int)u, __ldg(adj + a), a);
  }
  for (long long c = warp; c < nchunk; c += nwarps) {
    const int2 it = __ldg(hch + c);
    const int b = __ldg(off + it.x) + it.y * kChunk, e = min(__ldg(off + it.x + 1), b + kChunk);
    for (int a = b + lane; a < e; a += 32) table_insert(tab, nslots, it.x, __ldg(adj + a), a);
  }
}

// Capacity words from the uploaded int32 capacities (epoch 0: set by no batch).
__global__ void __launch_bounds__(256) k_cap_widen(const int *__restrict__ w, unsigned long long *capx, long long m) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (long long)gridDim.x * blockDim.x)
    capx[e] = (unsigned long long)(unsigned)__ldg(w + e);
}

// The capacities of a range of capacity words.
__global__ void __launch_bounds__(256) k_cap_low(const unsigned long long *__restrict__ capx, int *out, long long m) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (long long)gridDim.x * blockDim.x)
    out[e] = (int)(unsigned)__ldg(capx + e);
}

struct dmf_solver {
  int dev = 0;
  cudaStream_t stream = nullptr;
  int n = 0, m = 0, s = 0, t = 0;
  dmf_opts opts{};
  int tile = 32, grid = 0, block = kBlock, hub_deg = 256, small_deg = 8, minb = 2, bu_alpha = 2;
  int *off = nullptr, *adj = nullptr, *par = nullptr, *res = nullptr;
  unsigned long long *capx = nullptr;  // (epoch of the batch that set it << 32) | capacity
  ArcSlot *atab = nullptr;  // (tail, head) -> arc, with the per-arc batch stamps
  long long nslots = 0;
  int *height = nullptr, *stamp = nullptr, *uarc = nullptr;
  long long *excess = nullptr;
  unsigned char *dead = nullptr, *side = nullptr;
  int *dlab = nullptr;    // dead-set repair labels, tagged with the launch epoch
  int *pcur = nullptr;    // per vertex: pull scan cursor in its row
  bool caps_bounded = false;  // every capacity <= 2^30 - 1 (updates keep it so)
  int *qbuf = nullptr;    // 6 vertex queues (frontier x2, worklist x2, active, dead-set candidates)
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
  CK(cudaMalloc(&nb, sizeof(int) * 5 * (size_t)want), "cudaMalloc updates");
  // src, dst, w (staged host batches), then the per-update arc and claimed capacity
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
  p.atab = sv->atab;
  p.nslots = sv->nslots;
  p.cap = nullptr;
  p.capx = sv->capx;
  p.res = sv->res;
  p.height = sv->height;
  p.stamp = sv->stamp;
  p.uarc = sv->ubuf ? sv->ubuf + 3 * (size_t)sv->kcap : nullptr;
  p.uold = sv->ubuf ? sv->ubuf + 4 * (size_t)sv->kcap : nullptr;
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
  p.dq = sv->qbuf + 5 * N;
  p.dlab = sv->dlab;
  p.pcur = sv->pcur;
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
  p.keep_dead = mode == MODE_DYNAMIC && !(sv->opts.flags & DMF_FLAG_REVIVE_DEAD) ? 1 : 0;
  p.caps_bounded = sv->caps_bounded ? 1 : 0;
  const bool hook = (sv->opts.flags & DMF_FLAG_TEST_BARRIER_TIMEOUT) != 0;
  p.barrier_ns = hook ? kTestBarrierTimeoutNs : kBarrierTimeoutNs;
  p.absent_block = hook && sv->grid > 1 ? sv->grid - 1 : -1;
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
  sv->st.bfs_arcs = (int64_t)c.st_barcs;
  sv->st.dead_deficits = (int64_t)c.st_dseeds;
  sv->st.dead_revived = (int64_t)c.st_revived;
  sv->st.dead_kept = c.dkept;
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

// Host batch -> pinned staging -> device, pipelined: the three arrays are cut
// into pieces of kStagePiece updates; copier threads fill the pinned buffer
// piece by piece (piece i by thread i mod kStageCopiers, so early pieces finish
// first) while one issuer thread starts the H2D of each piece as soon as it is
// in, so the copy engine works while later pieces are still being copied.  A
// batch of fewer than four pieces is copied and sent whole.
constexpr size_t kStagePiece = 1 << 18;  // updates (1 MiB of int32)
constexpr int kStageCopiers = 8;

int stage_batch(dmf_solver *sv, int32_t k, const int32_t *src, const int32_t *dst, const int32_t *w) {
  int st;
  CK(cudaSetDevice(sv->dev), "cudaSetDevice");
  if ((st = ensure_ubuf(sv, k)) || (st = ensure_host_ubuf(sv, k))) return st;
  const size_t K = (size_t)sv->kcap, HK = (size_t)sv->h_kcap, n = (size_t)k;
  const int32_t *from[3] = {src, dst, w};
  const size_t per = (n + kStagePiece - 1) / kStagePiece, total = 3 * per;
  if (total < 4) {
    for (int a = 0; a < 3 && n > 0; a++) {
      std::memcpy(sv->h_ubuf + a * HK, from[a], 4 * n);
      CK(cudaMemcpyAsync(sv->ubuf + a * K, sv->h_ubuf + a * HK, 4 * n, cudaMemcpyHostToDevice, sv->stream),
         "H2D batch");
    }
  } else {
    std::vector<std::atomic<int>> ready(total);
    for (auto &r : ready) r.store(0, std::memory_order_relaxed);
    cudaError_t err = cudaSuccess;
    auto piece = [&](size_t i, size_t &a, size_t &b, size_t &e) {
      a = i / per;
      b = (i % per) * kStagePiece;
      e = std::min(n, b + kStagePiece);
    };
#pragma omp parallel num_threads(kStageCopiers + 1)
    {
      const int tid = omp_get_thread_num(), nthr = omp_get_num_threads();
      if (tid == 0) {  // the issuer (with no other thread it copies too)
        for (size_t i = 0; i < total; i++) {
          size_t a, b, e;
          piece(i, a, b, e);
          if (nthr == 1) std::memcpy(sv->h_ubuf + a * HK + b, from[a] + b, 4 * (e - b));
          else
            while (!ready[i].load(std::memory_order_acquire)) std::this_thread::yield();
          if (err == cudaSuccess)
            err = cudaMemcpyAsync(sv->ubuf + a * K + b, sv->h_ubuf + a * HK + b, 4 * (e - b),
                                  cudaMemcpyHostToDevice, sv->stream);
        }
      } else {
        for (size_t i = (size_t)(tid - 1); i < total; i += (size_t)(nthr - 1)) {
          size_t a, b, e;
          piece(i, a, b, e);
          std::memcpy(sv->h_ubuf + a * HK + b, from[a] + b, 4 * (e - b));
          ready[i].store(1, std::memory_order_release);
        }
      }
    }
    if (err != cudaSuccess) return cuda_fail(err, "H2D batch");
  }
  CK(cudaEventRecord(sv->ev0, sv->stream), "event record");
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
    k_features<<<blocks, 256, 0, sv->stream>>>(sv->off, sv->atab, sv->nslots, sv->capx, sv->res, sv->n, k,
                                               sv->ubuf, sv->ubuf + K, sv->ubuf + 2 * K, sv->facc);
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
  int mode = MODE_DYNAMIC;
  switch (action) {
    case DMF_ACTION_SHORT:
      sv->opts.relabel_interval = 2;
      sv->opts.flags |= DMF_FLAG_FIXED_INTERVAL;
      break;
    case DMF_ACTION_REVIVE:
      sv->opts.flags |= DMF_FLAG_REVIVE_DEAD;
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
                                 5 * na_round(4 * kNoAllocV) /* queues */ + 4 * kNoAllocAlign /* unused hub slots */;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch on the current device (the name is only a
// host-side stand-in for the array; a kernel must be given this address).  It
// is looked up on every call: the lookup allocates nothing, and a context that
// was reset and re-created may have loaded the array at another address.
int noalloc_scratch(unsigned char **out) {
  void *ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if (e != cudaSuccess || !ptr) return cuda_fail(e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress");
  *out = (unsigned char *)ptr;
  return DMF_OK;
}

}  // namespace

extern "C" {

int dmf_static_maxflow_noalloc(int32_t n, int32_t m, const int32_t *d_index, const int32_t *d_adj,
                               const int32_t *d_cap, const int32_t *d_par, int32_t s, int32_t t, int32_t *d_res,
                               int64_t *flow, void *stream) {
  return guarded([&]() -> int {
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
    int st = noalloc_scratch(&base);
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
    p.dq = nullptr;  // static solves never keep a dead set
    p.dlab = nullptr;
    p.pcur = nullptr;
    // no hubs in this mode (hub_deg = INT_MAX): the hub structures are never read
    int2 *hub_dummy = (int2 *)carve(kNoAllocAlign);
    long long *ll_dummy = (long long *)carve(kNoAllocAlign);
    int *int_dummy = (int *)carve(kNoAllocAlign);
    unsigned long long *mark_dummy = (unsigned long long *)carve(kNoAllocAlign);
    if (off > kNoAllocBytes) return fail(DMF_ERR_CUDA, "internal: scratch layout exceeds the array");
    p.srcs = nullptr;  // one source: the kernel takes it from p.s
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
    p.atab = nullptr;
    p.nslots = 0;
    p.cap = const_cast<int *>(d_cap);  // read only in static mode
    p.capx = nullptr;
    p.res = d_res;
    p.uarc = nullptr;
    p.uold = nullptr;
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
    p.keep_dead = 0;
    p.caps_bounded = 0;
    p.barrier_ns = kBarrierTimeoutNs;
    p.absent_block = -1;
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
  });
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
      (st = dalloc(sv, &sv->atab, (size_t)arc_table_slots((long long)M))) || (st = dalloc(sv, &sv->capx, M)) ||
      (st = dalloc(sv, &sv->res, M)) || (st = dalloc(sv, &sv->height, N)) || (st = dalloc(sv, &sv->stamp, N)) ||
      (st = dalloc(sv, &sv->excess, N)) || (st = dalloc(sv, &sv->dead, N)) || (st = dalloc(sv, &sv->side, N)) ||
      (st = dalloc(sv, &sv->qbuf, 6 * N)) || (st = dalloc(sv, &sv->dlab, N)) || (st = dalloc(sv, &sv->pcur, N)) || (st = dalloc(sv, &sv->ctrl, 1)))
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
  sv->nslots = arc_table_slots((long long)M);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->atab, 0xFF, sizeof(ArcSlot) * (size_t)sv->nslots, S);
  up(sv->res, g->w.data(), 4 * M);  // staged in res, widened into capx (epoch 0)
  if (e == cudaSuccess && M > 0) {
    k_cap_widen<<<(int)std::min<size_t>((M + 255) / 256, 8 * 148), 256, 0, S>>>(sv->res, sv->capx, (long long)M);
    e = cudaGetLastError();
  }
  {
    int32_t mx = 0;
#pragma omp parallel for schedule(static) reduction(max : mx)
    for (int64_t i = 0; i < (int64_t)M; i++) mx = std::max(mx, g->w[i]);
    sv->caps_bounded = mx <= kMaxUpdateCap;
  }
  up(sv->hch, hub_chunks.data(), sizeof(int2) * hub_chunks.size());
  up(sv->hub_base, hub_base.data(), 4 * (size_t)g->n);
  if (e == cudaSuccess && g->n > 0) {
    const int warps = 8, blocks = (int)std::min<long long>(((long long)g->n + warps - 1) / warps, 16LL * 148);
    k_arc_table_build<<<blocks, 32 * warps, 0, S>>>(sv->off, sv->adj, g->n, sv->hub_deg, sv->hch, sv->nchunk,
                                                    sv->atab, sv->nslots);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->chunk_mark, 0, 8 * NC, S);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->hc_done, 0, 4 * NC, S);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->hc_alloc, 0, 8 * NC, S);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->hc_moved, 0, 8 * NC, S);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->stamp, 0, 4 * N, S);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->dead, 0, N, S);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->dlab, 0, 4 * N, S);
  if (e == cudaSuccess) e = cudaMemsetAsync(sv->pcur, 0, 4 * N, S);
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

int64_t dmf::solver_footprint(int64_t n, int64_t m) {
  // adj, par, res, capacity words; the arc table; off, labels, stamps,
  // excess, marks, repair labels, hub bases and six vertex queues (rounded up)
  return 20 * m + (int64_t)sizeof(ArcSlot) * arc_table_slots(m) + 64 * n;
}

int dmf::reserve_updates(dmf_solver *sv, int32_t k) {
  CK(cudaSetDevice(sv->dev), "cudaSetDevice");
  int st = ensure_ubuf(sv, k);
  if (!st) st = ensure_host_ubuf(sv, k);
  return st;
}

int dmf::resident_solve_blocks(int32_t *blocks) {
  int dev = 0, per_sm = 0, sms = 0;
  CK(cudaGetDevice(&dev), "cudaGetDevice");
  // every instantiation has the same launch bounds (kBlock threads, 2 blocks per SM)
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)pick_kernel(32, 2), kBlock, 0), "occupancy");
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "sm count");
  *blocks = per_sm * sms;
  return DMF_OK;
}

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
    if (best.tile <= 0) best.tile = sv->tile;  // the result names the tile the defaults resolved to
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
  if (cap && M > 0) {  // the low halves of the capacity words, through a device buffer in pieces
    const size_t piece = std::min<size_t>(M, (size_t)1 << 26);
    int *tmp = nullptr;
    CK(cudaMalloc(&tmp, 4 * piece), "cudaMalloc capacity readout");
    cudaError_t e = cudaSuccess;
    for (size_t b = 0; b < M && e == cudaSuccess; b += piece) {
      const size_t len = std::min(piece, M - b);
      k_cap_low<<<(int)std::min<size_t>((len + 255) / 256, 8 * 148), 256, 0, sv->stream>>>(sv->capx + b, tmp,
                                                                                          (long long)len);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaMemcpyAsync(cap + b, tmp, 4 * len, cudaMemcpyDeviceToHost, sv->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(sv->stream);
    }
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_fail(e, "D2H cap");
  }
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
    CK(cudaMemcpyAsync(dst->capx, src->capx, 8 * M, cudaMemcpyDeviceToDevice, S), "D2D cap");
    CK(cudaMemcpyAsync(dst->res, src->res, 4 * M, cudaMemcpyDeviceToDevice, S), "D2D res");
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
    // later than every epoch either solver used: no stale batch stamp or
    // repair-label tag in dst's own arrays can equal a future launch's epoch
    dst->epoch = std::max(dst->epoch, src->epoch);
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
