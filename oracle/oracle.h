/*
 * oracle.h -- CPU oracle for the dynamic max-flow hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links or calls this
 * code.  It is used by tests/, by __graft_entry__.smoke() as the checker, and by
 * bench.py's CPU-baseline leg / reference arm.
 *
 * Contents:
 *   - readers for the two on-disk formats (code/graph.hpp:202-223,
 *     code/update.hpp:52-88 of ShruthiKannappan/dyn_maxflow);
 *   - a direct restatement of the CSR builder (input_create/create_bin.cpp:18-124);
 *   - an exact Dinic solver (independent of the reference algorithm);
 *   - a certificate checker (capacity bounds, pseudoflow accounting, no residual
 *     path from any active vertex, min-cut capacity == flow value);
 *   - a restatement of the reference's three GPU algorithms (data-driven
 *     push-relabel code/dyn_data.h, topology-driven code/dyn_topo.h, push-pull
 *     code/dyn_pp.h) with their host drivers, as OpenMP loops.  Each kernel is a
 *     parallel loop over the same index range as the CUDA launch; with one thread
 *     the loops run in thread-index order.
 *
 * Parity pins: the johnson8-2-4 fixture (max-flow 540, s=25, t=2) and the flow
 * values printed by the reference's own CUDA binaries on the same inputs
 * (tests/golden/).
 */
#ifndef DMF_ORACLE_H
#define DMF_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---- formats ---------------------------------------------------------- */
/* code/graph.hpp:202-223: int32 n, m, index[n+1], adj[m], w[m], par[m].
 * Returns 0 on success, -1 on open/short-read failure. Arrays are malloc'd. */
int orc_graph_read(const char *path, int32_t *n, int32_t *m, int32_t **off,
                   int32_t **adj, int32_t **w, int32_t **par);
/* code/update.hpp:52-88: int32 k, src[k], dst[k], w[k].  Unlike the reference
 * (which returns 2k entries, the first k zero-typed and skipped by the kernels),
 * this returns exactly the k records; self-loops are kept (callers skip them as
 * OnAdd_kernel does, code/dyn_data.h:194). */
int orc_updates_read(const char *path, int32_t *k, int32_t **src, int32_t **dst,
                     int32_t **w);
void orc_free(void *p);

/* input_create/create_bin.cpp:67-124 (readEdgeList) + :18-64 (writeCSR), O(deg^2)
 * as written there: self-loops dropped, duplicate arcs summed, every arc gets a
 * partner (created with capacity 0 if absent), adjacency in first-touch order.
 * n = max id + 1.  Outputs malloc'd; returns 0 or -1. */
int orc_build_csr(int64_t k, const int32_t *u, const int32_t *v, const int32_t *w,
                  int32_t *n, int32_t *m, int32_t **off, int32_t **adj,
                  int32_t **cap, int32_t **par);

/* ---- exact solvers and certificates ------------------------------------ */
/* Dinic on the CSR with capacities cap[] (arc pairs via par[]).  Independent of
 * the reference algorithm.  If flow_out != NULL it receives f(e) = cap - res. */
int64_t orc_dinic(int32_t n, int32_t m, const int32_t *off, const int32_t *adj,
                  const int32_t *cap, const int32_t *par, int32_t s, int32_t t,
                  int32_t *flow_out);

/* Certificate for a pseudoflow given by residuals res[] over capacities cap[]:
 *  (1) 0 <= res[e] and res[e] + res[par e] == cap[e] + cap[par e];
 *  (2) excess(v) = sum_out (res - cap); value = excess(t) + sum_{v!=s, ex<0} ex;
 *  (3) S' = vertices with a residual path to t or to a deficit vertex:
 *      s not in S', no vertex v != s,t with excess > 0 in S';
 *  (4) capacity of the cut (V\S', S') equals value.
 * (1)-(4) imply that value is the maximum s-t flow.  Returns 0 when all hold and
 * writes the value; otherwise a positive code naming the first failed check. */
int orc_certify(int32_t n, int32_t m, const int32_t *off, const int32_t *adj,
                const int32_t *cap, const int32_t *par, const int32_t *res,
                int32_t s, int32_t t, int64_t *value, int64_t *cut_capacity);

/* ---- restatement of the reference's GPU algorithms ---------------------- */
enum { ORC_DATA = 0, ORC_TOPO = 1, ORC_PP = 2 };

/* Runs, for one update file, what the reference bench does for one
 * kernel_cycles value (e.g. code/dyn_data_bench.cu:535-536):
 *   dynflow  = recalculate_max_flow(...)   static solve on the ORIGINAL graph,
 *              then one batch of updates through OnAdd + Incremental, then
 *              recalculate_max_flow_kernel_39;
 *   statflow = static_recalculate(...)     capacities set by update_kernel, then
 *              a from-scratch static solve.
 * w0 is not modified.  Either output pointer may be NULL.  static_flow_before
 * receives the static flow on the original graph.
 * Returns 0, or -1 if an outer loop exceeded max_iters (non-convergence).  */
int orc_ref_run(int variant, int32_t n, int32_t m, const int32_t *off,
                const int32_t *adj, const int32_t *w0, const int32_t *par,
                int32_t s, int32_t t, int32_t kernel_cycles, int32_t k,
                const int32_t *usrc, const int32_t *udst, const int32_t *uw,
                int nthreads, int64_t max_iters, int64_t *static_flow_before,
                int64_t *dynflow, int64_t *statflow);

/* Successive batches on one resident state (the state is never rebuilt between
 * batches): static solve, then for each batch b the reference's OnAdd +
 * Incremental + kernel_39 readout.  flows[b] receives the flow after batch b.
 * Batch b holds updates [bofs[b], bofs[b+1]).  With budget_ms > 0 the run
 * stops after the batch that brings the batches' total time over the budget;
 * *done (if not NULL) receives the number of batches run. */
int orc_ref_run_successive(int variant, int32_t n, int32_t m, const int32_t *off,
                           const int32_t *adj, const int32_t *w0,
                           const int32_t *par, int32_t s, int32_t t,
                           int32_t kernel_cycles, int32_t nbatches,
                           const int64_t *bofs, const int32_t *usrc,
                           const int32_t *udst, const int32_t *uw, int nthreads,
                           int64_t max_iters, int64_t *static_flow,
                           int64_t *flows, double *batch_ms, double budget_ms,
                           int32_t *done);

#ifdef __cplusplus
}
#endif
#endif
