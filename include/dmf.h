/*
 * dmf.h -- C ABI of libdmf.so, the B200 dynamic s-t max-flow engine.
 *
 * The library is a drop-in for the hot path of ShruthiKannappan/dyn_maxflow:
 * it reads the same CSR graph and update .bin formats and computes, after every
 * capacity-update batch, the exact maximum s-t flow with push-relabel kernels
 * written for sm_100a.  The reference has no library API; each entry point below
 * names the reference function or kernel sequence it replaces (file:line in that
 * project).
 *
 * Conventions
 *   - Every function returns a dmf_status (0 = DMF_OK).  dmf_last_error()
 *     returns a message for the last failure on the calling thread.  The
 *     library never calls exit(), and no C++ exception leaves an entry point:
 *     a failed host allocation returns DMF_ERR_OOM, any other host runtime
 *     failure DMF_ERR_HOST.
 *   - Host arrays passed in are copied during the call; the caller keeps them.
 *     Arrays returned through out-pointers are owned by the library and freed
 *     with dmf_free() / dmf_graph_free().
 *   - A dmf_solver owns all of its device memory, lives on one CUDA device and
 *     one stream, and is not re-entrant.  Different solvers may be used
 *     concurrently from different host threads.
 *   - Capacities are int32 and must be >= 0; cap(e) + cap(partner(e)) must fit
 *     in int32.  Flow values and excesses are int64.
 *   - An update is (src, dst, w): the arc src->dst, which must already exist in
 *     the CSR (reserved zero-capacity slots serve as insert targets), gets the
 *     absolute new capacity w.  Updates with src == dst are ignored, as in the
 *     reference.  An arc may appear at most once per batch.
 */
#ifndef DMF_H
#define DMF_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  DMF_OK = 0,
  DMF_ERR_INVALID_ARG = 1,   /* bad size, vertex id, s == t, negative capacity */
  DMF_ERR_BAD_FILE = 2,      /* missing, truncated or inconsistent .bin */
  DMF_ERR_UNKNOWN_ARC = 3,   /* update names an arc absent from the CSR */
  DMF_ERR_DUP_ARC = 4,       /* an arc appears twice in one batch */
  DMF_ERR_OOM = 5,           /* device or host allocation failed */
  DMF_ERR_NO_CONVERGENCE = 6,/* outer-iteration bound reached */
  DMF_ERR_CUDA = 7,          /* CUDA runtime error, or no usable device */
  DMF_ERR_TIMEOUT = 8,       /* a bounded device-side wait gave up */
  DMF_ERR_OVERFLOW = 9,      /* cap(e) + cap(partner) exceeds int32 */
  DMF_ERR_NOT_SOLVED = 10,   /* update or query before the first solve */
  DMF_ERR_HOST = 11          /* host runtime failure other than allocation (thread, lock) */
} dmf_status;

/* Algorithm variants: the three reference entry points. */
typedef enum {
  DMF_VARIANT_DATA = 0, /* dyn_data: worklist-driven push-relabel (code/dyn_data.h) */
  DMF_VARIANT_TOPO = 1, /* dyn_topo: topology-driven sweeps (code/dyn_topo.h) */
  DMF_VARIANT_PP = 2    /* dyn_pp: push-pull on the kept min-cut partition (code/dyn_pp.h) */
} dmf_variant;

/* dmf_opts.flags bits */
#define DMF_FLAG_TRACE 1 /* record a per-phase device timeline (dmf_trace_get) */
#define DMF_FLAG_PROBE 2 /* with TRACE: also time every work item (dmf_trace_items) */
#define DMF_FLAG_REVIVE_DEAD 8 /* batches revive every vertex at their first global relabel
                                  instead of keeping the dead set of the last solve */
#define DMF_FLAG_TEST_BARRIER_TIMEOUT 16 /* failure-injection hook for tests: one block of
                                  the persistent grid leaves at once and never arrives
                                  at a grid barrier, and the barrier wait limit drops
                                  from 4 s to 20 ms, so the call returns
                                  DMF_ERR_TIMEOUT (every wait stays bounded; the
                                  next call without the flag solves normally) */
#define DMF_FLAG_FIXED_INTERVAL 4 /* exactly relabel_interval push rounds per global relabel
                                     (default: at least the depth of the last relabel BFS) */

typedef struct dmf_graph dmf_graph;   /* host CSR, owned by the library */
typedef struct dmf_solver dmf_solver; /* device-resident residual state */

typedef struct {
  int32_t variant;          /* dmf_variant */
  int32_t kernel_cycles;    /* push/relabel cycles per vertex visit; 0 = avg degree
                               (the reference runs avg_deg-1, avg_deg, avg_deg+1,
                               code/dyn_data_bench.cu:529-562) */
  int32_t relabel_interval; /* push rounds between global relabels; 0 = adaptive */
  int32_t tile;             /* lanes per vertex (1,2,4,8,16,32); 0 = chosen from degree */
  int32_t max_iters;        /* bound on global-relabel iterations per solve; 0 = default */
  int32_t device;           /* CUDA device ordinal; -1 = current device */
  int32_t block_threads;    /* threads per block of the persistent kernel; 0 = 512 */
  int32_t flags;            /* DMF_FLAG_* bits */
  int32_t small_deg;        /* vertices of degree <= small_deg are handled one per
                               thread, larger ones one per tile (thread-vs-warp
                               per vertex); 0 = 8, -1 = no per-thread tier */
  int32_t grid_blocks;      /* cap on the persistent grid (0 = every SM); a smaller
                               grid lets several solvers run side by side */
} dmf_opts;

typedef struct {
  int64_t flow;             /* last flow value */
  int64_t outer_iters;      /* global relabels in the last solve */
  int64_t bfs_levels;       /* BFS levels expanded in the last solve */
  int64_t push_rounds;      /* worklist rounds in the last solve */
  int64_t pushes;           /* non-zero pushes in the last solve */
  int64_t relabels;         /* local relabels in the last solve */
  int64_t arcs_scanned;     /* adjacency entries read in the last solve */
  int64_t vertices_visited; /* vertex visits (BFS + push) in the last solve */
  int64_t dead_vertices;    /* vertices proven unable to reach t or a deficit */
  double last_ms;           /* device time of the last solve call (CUDA events), from
                               the batch on the device to the result (host-array
                               calls: the H2D of the batch is not included) */
  int32_t grid_blocks;      /* persistent-kernel grid */
  int32_t block_threads;
  int32_t tile;
  int32_t pad;
  int64_t bfs_arcs;         /* adjacency entries read by global-relabel BFS levels
                               (included in arcs_scanned) */
  int64_t dead_deficits;    /* deficits a batch left inside the kept dead set */
  int64_t dead_revived;     /* dead vertices revived because they reach a deficit the
                               local repair left (partial revival) */
  int32_t dead_kept;        /* 1: the batch kept the dead set of the last solve
                               (all of it but the partially revived vertices) */
  int32_t pad2;
} dmf_stats;

/* ---- errors and options ------------------------------------------------- */
const char *dmf_last_error(void);
const char *dmf_status_string(int status);
void dmf_opts_default(dmf_opts *opts);
void dmf_free(void *p);

/* ---- graphs (host only; no GPU needed) ---------------------------------- */
/* Replaces graph::loadGraph, code/graph.hpp:202-223 (no magic: int32 n, m,
 * index[n+1], adj[m], w[m], par[m]).  Validates sizes, offsets, ids and the
 * partner involution. */
int dmf_graph_load(const char *path, dmf_graph **out);
/* Builds from CSR arrays with the same validation as dmf_graph_load. */
int dmf_graph_from_csr(int32_t n, int32_t m, const int32_t *index,
                       const int32_t *adj, const int32_t *w, const int32_t *par,
                       dmf_graph **out);
/* Replaces input_create/create_bin.cpp:67-124 in O(k log k): self-loops
 * dropped, duplicate arcs summed, a zero-capacity partner for every arc,
 * adjacency in first-touch order (byte-identical .bin). */
int dmf_graph_from_edges(int64_t k, const int32_t *u, const int32_t *v,
                         const int32_t *w, dmf_graph **out);
/* Writes the .bin, input_create/create_bin.cpp:18-64 (writeCSR). */
int dmf_graph_save(const dmf_graph *g, const char *path);
int dmf_graph_info(const dmf_graph *g, int32_t *n, int32_t *m);
/* Borrowed pointers into the graph (valid until dmf_graph_free). */
int dmf_graph_arrays(const dmf_graph *g, const int32_t **index,
                     const int32_t **adj, const int32_t **w, const int32_t **par);
/* Arc index of src->dst (last match, as OnAdd_kernel code/dyn_data.h:196-201),
 * or -1. */
int64_t dmf_graph_find_arc(const dmf_graph *g, int32_t src, int32_t dst);
/* Sets the capacity of existing arcs on the host copy (the reference's
 * update_kernel, code/dyn_data_bench.cu:300-322). */
int dmf_graph_set_caps(dmf_graph *g, int32_t k, const int32_t *src,
                       const int32_t *dst, const int32_t *w);
void dmf_graph_free(dmf_graph *g);

/* ---- update files (host only) ------------------------------------------- */
/* Replaces loadUpdateFile, code/update.hpp:52-88 (int32 k, src[k], dst[k],
 * w[k]); returns exactly k records (no zero-typed padding). */
int dmf_updates_load(const char *path, int32_t *k, int32_t **src,
                     int32_t **dst, int32_t **w);
/* Writes the update .bin, input_create/create_update_bin.cpp:41-49. */
int dmf_updates_save(const char *path, int32_t k, const int32_t *src,
                     const int32_t *dst, const int32_t *w);

/* ---- seeded generators (host only) -------------------------------------- */
/* Directed 4-neighbour rows x cols grid, both directions, caps uniform
 * [cap_lo, cap_hi] from `seed`; source = vertex (0,0) joined to every column-0
 * vertex, sink = (rows-1, cols-1) fed by every last-column vertex, both with
 * capacity st_cap (coinciding arcs summed, as create_bin does). */
int dmf_gen_grid(int32_t rows, int32_t cols, uint64_t seed, int32_t cap_lo,
                 int32_t cap_hi, int32_t st_cap, dmf_graph **out, int32_t *s,
                 int32_t *t);
/* R-MAT: 2^scale vertices, `narcs` directed samples with probabilities
 * (a, b, c, 1-a-b-c); self-loops and duplicates dropped; caps uniform
 * [cap_lo, cap_hi]; `reserve` extra distinct non-arcs added with capacity 0
 * as insert slots.  s = max out-degree vertex, t = max in-degree vertex != s. */
int dmf_gen_rmat(int32_t scale, int64_t narcs, double a, double b, double c,
                 uint64_t seed, int32_t cap_lo, int32_t cap_hi, int64_t reserve,
                 dmf_graph **out, int32_t *s, int32_t *t);
/* Successive mixed batches over the graph's current capacities (the graph is
 * not modified).  Each batch touches `frac` of the positive-capacity arcs
 * (at least 1): p_inc increases (+U[1,delta_hi]), p_dec decreases
 * (max(0, c-U[1,delta_hi])), p_ins inserts into zero-capacity slots (U[ins_lo,
 * ins_hi]), the rest deletes (c -> 0).  Arcs are distinct within a batch.
 * Output: batch b is [ofs[b], ofs[b+1]) of src/dst/w (library-owned). */
int dmf_gen_batches(const dmf_graph *g, int32_t nbatches, double frac,
                    double p_inc, double p_dec, double p_ins, int32_t delta_hi,
                    int32_t ins_lo, int32_t ins_hi, uint64_t seed,
                    int64_t **ofs, int32_t **src, int32_t **dst, int32_t **w);

/* ---- solver (CUDA) ------------------------------------------------------ */
/* Uploads the graph (the reference's cudaMalloc + H2D at
 * code/dyn_data_bench.cu:182-217) and builds the device state.  `stream` is a
 * cudaStream_t or NULL for the legacy default stream. */
int dmf_solver_create(const dmf_graph *g, int32_t s, int32_t t,
                      const dmf_opts *opts, void *stream, dmf_solver **out);
/* Static solve from the solver's current capacities: replaces staticMaxFlow,
 * code/dyn_data_bench.cu:8-97 (topo :16-75, pp code/dyn_pp_bench.cu:155-239),
 * followed by the flow readout recalculate_max_flow_kernel_39
 * (code/dyn_data.h:208-215). */
int dmf_static_maxflow(dmf_solver *sv, int64_t *flow);
/* One update batch from host arrays: replaces OnAdd_kernel
 * (code/dyn_data.h:186-206) + Incremental (code/dyn_data_bench.cu:98-170; topo
 * code/dyn_topo_bench.cu:76-119; pp code/dyn_pp_bench.cu:242-258) + kernel_39.
 * Includes the H2D copy of the batch and the D2H read of the flow value. */
int dmf_apply_updates(dmf_solver *sv, int32_t k, const int32_t *src,
                      const int32_t *dst, const int32_t *w, int64_t *flow);
/* The same with the batch already in device memory (device pointers). */
int dmf_apply_updates_device(dmf_solver *sv, int32_t k, const int32_t *d_src,
                             const int32_t *d_dst, const int32_t *d_w,
                             int64_t *flow);
/* From-scratch recompute after setting capacities: replaces update_kernel +
 * static solve of static_recalculate (code/dyn_data_bench.cu:300-492). */
int dmf_recompute(dmf_solver *sv, int32_t k, const int32_t *src,
                  const int32_t *dst, const int32_t *w, int64_t *flow);
int dmf_recompute_device(dmf_solver *sv, int32_t k, const int32_t *d_src,
                         const int32_t *d_dst, const int32_t *d_w, int64_t *flow);
/* Last flow value (host copy; no device work). */
int dmf_flow_value(const dmf_solver *sv, int64_t *flow);
/* Minimum-cut side per vertex: 1 = sink side (can reach t or a deficit in the
 * residual graph), 0 = source side.  Replaces find_cut, code/dyn_pp.h:440-449. */
int dmf_get_cut(dmf_solver *sv, uint8_t *sink_side);
/* Device state copied to host (any pointer may be NULL): capacities and
 * residuals per arc, excess and height per vertex. */
int dmf_get_state(dmf_solver *sv, int32_t *cap, int32_t *res, int64_t *excess,
                  int32_t *height);
int dmf_stats_get(const dmf_solver *sv, dmf_stats *st);
/* Phase timeline of the last solve call (needs DMF_FLAG_TRACE): entry 0 is the
 * kernel start (kind 0); entry i > 0 is the end of a phase of kind kinds[i] at
 * t_us[i] microseconds after the start.  Kinds: 1 init residuals, 2 source
 * saturation, 3 arc lookup, 4 capacity apply, 5 over-capacity repair, 6 cut
 * saturation, 7 BFS seeds, 8 BFS top-down level, 9 BFS bottom-up level,
 * 10 BFS finalize, 11 push round, 12 flow readout, 13/14 hub push rounds,
 * 15-18 push-pull phase 1, 19 reopen, 20 dead-set pull seeding, 21 pull round,
 * 23 dead-set check, 24 partial revival, 25 capacity claim (duplicate-arc
 * check).  No counterpart in the reference (which
 * times whole calls with cudaEvents, code/dyn_data_bench.cu:246-258). */
int dmf_trace_get(dmf_solver *sv, int32_t cap, int32_t *kinds, double *t_us,
                  int32_t *count);
/* Work of each timeline entry: items[i] = vertices in the frontier or worklist
 * processed by that phase, hubs[i] = hub chunks among them; with
 * DMF_FLAG_PROBE, slow_ns[i] / slow_v[i] = duration and vertex of the phase's
 * longest single work item (slow_ns / slow_v may be NULL). */
int dmf_trace_items(dmf_solver *sv, int32_t cap, int64_t *items, int64_t *hubs,
                    int64_t *slow_ns, int64_t *slow_v);
/* With DMF_FLAG_PROBE: block_ns[i] = the longest time any block spent on phase
 * i's work (from leaving the previous grid barrier to arriving at the next);
 * the phase's duration minus this is barrier and skew. */
int dmf_trace_blocks(dmf_solver *sv, int32_t cap, int64_t *block_ns);
/* Replaces the option set of a live solver (variant, cycles, interval, tile). */
int dmf_solver_set_opts(dmf_solver *sv, const dmf_opts *opts);
int dmf_solver_destroy(dmf_solver *sv);

/* ---- batched instances ---------------------------------------------------- */
/* Many independent graphs (each with its own s, t) in one device state: their
 * disjoint union, solved by one persistent launch per call, every instance's
 * flow read out separately.  No counterpart in the reference (which solves one
 * graph per process).  Vertex v of instance i is vertex vertex_base[i] + v of the
 * union. */
int dmf_multi_create(int32_t count, const dmf_graph *const *graphs,
                     const int32_t *s, const int32_t *t, const dmf_opts *opts,
                     void *stream, dmf_solver **out);
int dmf_multi_info(const dmf_solver *sv, int32_t *count, int32_t *vertex_base);
/* Static solve of every instance; flows[count]. */
int dmf_multi_static_maxflow(dmf_solver *sv, int64_t *flows);
/* One batch whose updates may touch any instances: inst[k] names the instance,
 * src/dst are that instance's vertex ids; flows[count] after the batch. */
int dmf_multi_apply_updates(dmf_solver *sv, int32_t k, const int32_t *inst,
                            const int32_t *src, const int32_t *dst,
                            const int32_t *w, int64_t *flows);
/* `steps` successive batches already in device memory (union vertex ids; batch
 * b is [ofs[b], ofs[b+1]) of d_src/d_dst/d_w, ofs on the host), run back to back
 * on the solver's stream; with use_graph != 0 the whole loop is captured once
 * into a CUDA graph and launched as one graph.  flows[steps*count] receives the
 * per-instance flows after every step; *ms the device time of the loop. */
int dmf_multi_run_batches(dmf_solver *sv, int32_t steps, const int64_t *ofs,
                          const int32_t *d_src, const int32_t *d_dst,
                          const int32_t *d_w, int32_t use_graph,
                          int64_t *flows, double *ms);

/* ---- serving loop ------------------------------------------------------------ */
/* Device-resident graphs serving update-batch requests.  Graphs are admitted in
 * the given order while the estimated device footprint of their residual state
 * (52 B per arc + 64 B per vertex) fits `hbm_budget` bytes; the rest are not
 * admitted (ids of admitted graphs are their positions among the admitted ones,
 * dmf_server_info).  The caller keeps the graphs alive until destroy.
 * Lanes: a graph with at least a quarter of the admitted arcs gets a lane of
 * its own (at most 3 such lanes), the others share one lane.  Each lane has
 * its own solver, CUDA stream and worker thread, and a fixed share of the
 * GPU's resident solve blocks (in proportion to its arcs; `opts->grid_blocks`,
 * when > 0, caps the total), so the lanes' launches run side by side: a
 * request for a small graph is served while a large graph's solve is in flight.
 * Continuous batching within a lane: its worker serves, per tick, the oldest
 * waiting request of each of its graphs with one persistent launch, while the
 * tick's updates stay inside the lane's staging budget (its share of what the
 * graphs leave of hbm_budget, at least 16 MiB); requests arriving during a tick
 * join the next.  Batches of one graph apply in submission order.  submit() validates a
 * request on the host (vertex ranges, existing arcs, no repeats) and copies it;
 * wait() blocks until it is served and returns the graph's exact max-flow after
 * it and its latency from the start of its submit() call (validation
 * included); a ticket has one waiter, and a second wait() on it returns
 * DMF_ERR_INVALID_ARG.  destroy() serves every request already submitted,
 * lets threads blocked in wait() return their results, then frees the server;
 * no call on the server may start once destroy() has.  No counterpart in the
 * reference. */
typedef struct dmf_server dmf_server;
int dmf_server_create(int32_t count, const dmf_graph *const *graphs,
                      const int32_t *s, const int32_t *t, int64_t hbm_budget,
                      const dmf_opts *opts, dmf_server **out);
int dmf_server_info(const dmf_server *srv, int32_t *admitted, int64_t *device_bytes);
/* The lane that serves admitted graph `graph`, the number of lanes, and that
 * lane's share of resident solve blocks (any output may be NULL). */
int dmf_server_lane(const dmf_server *srv, int32_t graph, int32_t *lane, int32_t *lanes,
                    int32_t *grid_blocks);
int dmf_server_submit(dmf_server *srv, int32_t graph, int32_t k, const int32_t *src,
                      const int32_t *dst, const int32_t *w, int64_t *ticket);
int dmf_server_wait(dmf_server *srv, int64_t ticket, int64_t *flow, double *latency_ms);
int dmf_server_stats(const dmf_server *srv, int64_t *ticks, int64_t *served,
                     double *mean_requests_per_tick);
int dmf_server_destroy(dmf_server *srv);

/* ---- launch geometry autotuner --------------------------------------------- */
/* Times from-scratch solves of the solver's current capacities under candidate
 * tile widths, per-thread degree bounds (thread vs warp per vertex), relabel
 * intervals and cycle counts (coordinate descent, best of `repeats` runs each),
 * keeps the fastest in the solver and returns it in *chosen.  Every candidate
 * computes the same exact flow; the state afterwards is a maximum flow of the
 * current capacities.  *chosen names the tile width explicitly, also when the
 * solver's default (tile 0: chosen from the graph) was fastest. */
int dmf_autotune(dmf_solver *sv, int32_t repeats, dmf_opts *chosen);

/* ---- learned schedule picker ----------------------------------------------- */
/* No counterpart in the reference, whose schedule is fixed (one kernel_cycles
 * value, a global relabel after every push, incremental repair; code/
 * dyn_data_bench.cu:113-167).  Per update batch a small MLP picks one of
 * DMF_SCHED_ACTIONS schedules from DMF_SCHED_FEATURES features of the batch
 * measured against the live residual state.  Every action computes the same
 * exact flow; only the time differs.  Action 0 is the plain schedule, used
 * whenever no trained model is given. */
#define DMF_SCHED_FEATURES 12
#define DMF_SCHED_HIDDEN 64
#define DMF_SCHED_ACTIONS 4
#define DMF_SCHED_WEIGHTS 5120 /* bf16: W1[64][12], W2[64][64], W3[4][64] (row = output unit) */
#define DMF_SCHED_BIASES 132   /* fp32: b1[64], b2[64], b3[4] */
/* actions */
#define DMF_ACTION_PLAIN 0       /* incremental repair, engine defaults (dead set kept) */
#define DMF_ACTION_SHORT 1       /* incremental, global relabel every 2 push rounds */
#define DMF_ACTION_REVIVE 2      /* incremental, every vertex revived at the batch's first
                                    global relabel (DMF_FLAG_REVIVE_DEAD) */
#define DMF_ACTION_RECOMPUTE 3   /* set the capacities and solve from scratch */

typedef struct dmf_sched dmf_sched; /* MLP 12-64-64-4, bf16 weights, fp32 accumulation */

/* A model on `device` (-1 = current) with He-uniform weights from `seed`;
 * untrained until dmf_sched_train or dmf_sched_set_weights. */
int dmf_sched_create(int32_t device, uint64_t seed, dmf_sched **out);
int dmf_sched_destroy(dmf_sched *sched);
/* weights: DMF_SCHED_WEIGHTS bf16 bit patterns, biases: DMF_SCHED_BIASES. */
int dmf_sched_set_weights(dmf_sched *sched, const uint16_t *weights, const float *biases);
int dmf_sched_get_weights(dmf_sched *sched, uint16_t *weights, float *biases);
/* The model predicts, per action, log2 of its time relative to the plain
 * schedule; a non-plain action is picked only when predicted to win by more
 * than `margin` log2 units (default 0.1), else the plain schedule runs. */
int dmf_sched_set_margin(dmf_sched *sched, float margin);
/* Trains on n samples X[n][12] -> Y[n][4] (the targets are per-action costs,
 * log2 of each action's time over the plain schedule's) by minibatch Adam on fp32 master weights with bf16
 * weights in the forward pass, all on the device in one kernel: `steps`
 * minibatches of `batch` (1..64) samples drawn from `seed`, learning rate `lr`.
 * loss[steps] (may be NULL) receives the minibatch mean squared error. */
int dmf_sched_train(dmf_sched *sched, int32_t n, const float *X, const float *Y, int32_t steps,
                    int32_t batch, float lr, uint64_t seed, float *loss);
/* Y[n][4] = model(X[n][12]) on the device. */
int dmf_sched_predict(dmf_sched *sched, int32_t n, const float *X, float *Y);

/* Features of a batch against the solver's current state (nothing applied):
 * feat[12]; the names are listed in dyn_maxflow_b200/sched.py. */
int dmf_solver_features(dmf_solver *sv, int32_t k, const int32_t *src, const int32_t *dst,
                        const int32_t *w, float *feat);
/* Applies a batch with a given action (0..3). */
int dmf_apply_updates_action(dmf_solver *sv, int32_t action, int32_t k, const int32_t *src,
                             const int32_t *dst, const int32_t *w, int64_t *flow);
/* Applies a batch with the action `sched` picks (sched = NULL or untrained:
 * the plain schedule); *action (may be NULL) receives it.  The time reported
 * by dmf_stats_get includes the features and the decision. */
int dmf_apply_updates_scheduled(dmf_solver *sv, dmf_sched *sched, int32_t k, const int32_t *src,
                                const int32_t *dst, const int32_t *w, int64_t *flow,
                                int32_t *action);
/* Per-batch records the two calls above keep (the traces a model is trained
 * on): feat[i*12..], action[i], ms[i] (solve time), flow[i]; up to `cap`
 * oldest-first records are returned in *count and removed from the log.  Any
 * output pointer may be NULL. */
int dmf_sched_records(dmf_solver *sv, int32_t cap, float *feat, int32_t *action, float *ms,
                      int64_t *flow, int32_t *count);
/* Makes `dst` an exact copy of `src`'s residual state (same graph and
 * options required), so that a batch can be timed under several actions from
 * the same state. */
int dmf_solver_copy_state(dmf_solver *dst, const dmf_solver *src);

/* Static solve that allocates nothing, for callers that cannot allocate device
 * memory while they run (code inside a fixed memory pool or arena, or a host
 * that forbids cudaMalloc after start-up).  No counterpart in the reference.
 * The caller passes the CSR (index[n+1], adj[m], cap[m], par[m], the layout of
 * dmf_graph_from_csr, already validated) and d_res[m] for the residuals of the
 * maximum flow, all in its own device memory; *flow receives the value.  All
 * other scratch lives in one static device array inside the library, sized for
 * n <= 262144 vertices (about 10 MiB, held by every GPU that loads the library
 * until the process exits); larger n is rejected with DMF_ERR_INVALID_ARG.
 * Every call looks up the array's device address on the current device (the
 * lookup allocates nothing, and stays right if the context was reset).  Calls
 * share the array and each clears what must start at zero: calls that overlap
 * on the GPU race and give wrong results, so serialise them.  The call blocks
 * until the result is back: it waits for `stream` (a cudaStream_t, NULL =
 * legacy default stream), so work queued on it before the call is waited for
 * too. */
int dmf_static_maxflow_noalloc(int32_t n, int32_t m, const int32_t *d_index,
                               const int32_t *d_adj, const int32_t *d_cap,
                               const int32_t *d_par, int32_t s, int32_t t,
                               int32_t *d_res, int64_t *flow, void *stream);

/* Number of CUDA devices visible (0 without a GPU); never fails. */
int dmf_device_count(void);

#ifdef __cplusplus
}
#endif
#endif /* DMF_H */
