// Internal declarations shared by the host (dmf_host.cpp) and device
// (dmf_solver.cu) halves of libdmf.so.
#pragma once

#include <cstdint>
#include <exception>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "dmf.h"

// Host CSR.  Arrays follow the on-disk layout of code/graph.hpp:202-223.
// `sidx` is built on demand: for each vertex, its arc indices sorted by
// (head, arc) -- used for O(log deg) arc lookup.
struct dmf_graph {
  int32_t n = 0, m = 0;
  std::vector<int32_t> off, adj, w, par;
  std::vector<int32_t> sidx;
};

namespace dmf {

// Records a thread-local error message and returns `status`.  Never throws.
int fail(int status, const char *fmt, ...);
// Clears the thread-local message, returns DMF_OK.
int ok();

// Runs `body` (which returns a status) and turns a C++ exception into a
// status, so that none unwinds through the C ABI: std::bad_alloc and
// std::length_error become DMF_ERR_OOM, anything else DMF_ERR_HOST.
template <class F>
int guarded(F &&body) noexcept {
  try {
    return body();
  } catch (const std::bad_alloc &) {
    return fail(DMF_ERR_OOM, "host allocation failed");
  } catch (const std::length_error &x) {
    return fail(DMF_ERR_OOM, "host allocation too large (%s)", x.what());
  } catch (const std::exception &x) {
    return fail(DMF_ERR_HOST, "%s", x.what());
  } catch (...) {
    return fail(DMF_ERR_HOST, "unknown C++ exception");
  }
}

// Validates CSR structure: offsets, ids, partner involution, capacities.
int validate(const dmf_graph &g);
// Fills g.sidx (idempotent).
void build_sorted_index(dmf_graph &g);
// Arc src->dst via g.sidx (last arc index among equal heads), or -1.
int64_t find_arc(const dmf_graph &g, int32_t src, int32_t dst);

// Builds a graph with create_bin semantics from an edge list (first-touch
// adjacency order, duplicates summed, partners created with capacity 0).
int build_from_edges(int64_t k, const int32_t *u, const int32_t *v,
                     const int32_t *w, dmf_graph **out);

// Blocks of the persistent solve kernel that the current device holds at once
// (the grid of a solver without a grid_blocks cap).
int resident_solve_blocks(int32_t *blocks);

// Device bytes of one solver's per-arc and per-vertex state for a graph of n
// vertices and m arcs: heads, partners, capacities, residuals and the arc
// table per arc; labels, excess, marks and queues per vertex.
int64_t solver_footprint(int64_t n, int64_t m);

// Grows a solver's device and pinned staging for batches of up to k updates
// now, so that later calls of that size allocate nothing (an allocation or a
// free in the middle of serving waits for every stream of the device).
int reserve_updates(dmf_solver *sv, int32_t k);

}  // namespace dmf
