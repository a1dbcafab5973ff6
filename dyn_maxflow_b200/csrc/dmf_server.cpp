// dmf_server.cpp -- serving loop over device-resident residual graphs.
//
// Admission: graphs are admitted in the order given while the estimated device
// footprint of their residual state fits the HBM budget; each admitted graph
// stays resident for the server's life, and every batch a request carries is
// applied to it (successive batches per graph, in submission order).
//
// Lanes (continuous batching over device slots): the admitted graphs are split
// into lanes.  A graph with at least a quarter of the admitted arcs gets a lane
// of its own (at most kMaxLanes - 1 such lanes); the others share one lane whose
// graphs live in one batched-instance solver (dmf_multi_*).  Every lane has its
// own solver, CUDA stream, worker thread and a fixed share of the persistent
// grid (dmf_opts.grid_blocks), in proportion to its arcs.  The shares add up to
// at most the blocks the GPU holds at once (every solve kernel is launched for
// 2 blocks of 512 threads per SM, which fill its register file), so the lanes'
// cooperative launches are always resident together and never wait for one
// another: a request for a small graph is served while a large graph's solve is
// in flight, not after it.  A lane's worker runs ticks: it takes the oldest
// waiting request of each of its graphs, while the tick's updates fit the
// lane's staging budget, and serves them with one launch; requests arriving
// meanwhile join its next tick.  Instances are independent, so each result
// equals the result of the same request sequence served alone.  No counterpart
// in the reference (a one-shot bench).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <parallel/algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

#include "dmf_internal.h"

using dmf::guarded;

namespace {

using Clock = std::chrono::steady_clock;

constexpr int kMaxLanes = 4;
// Updates per tick a lane's staging is sized for at creation.
constexpr int64_t kStageReserve = 1 << 20;
// Host threads that validate one request (the lanes' workers and other
// submitters run beside them).
constexpr int kSubmitThreads = 8;

struct Request {
  int64_t ticket;
  int32_t graph;
  std::vector<int32_t> src, dst, w;
  Clock::time_point t_submit;
  bool claimed = false;  // a wait() holds it
  bool done = false;
  int status = DMF_OK;
  std::string error;
  int64_t flow = 0;
  double latency_ms = 0;
};

struct Lane {
  std::vector<int32_t> graphs;  // server graph ids, in instance order
  bool multi = false;           // batched-instance solver (else one graph, plain solver)
  dmf_solver *sv = nullptr;
  cudaStream_t stream = nullptr;
  int32_t grid_blocks = 0;
  int64_t stage_budget = 0;
  std::condition_variable cv_work;
  std::thread worker;
  // worker-owned, reused from tick to tick (they grow, never shrink)
  std::vector<Request *> batch;
  std::vector<int64_t> flows;
  std::vector<int32_t> I, A, B, W;
};

}  // namespace

struct dmf_server {
  std::vector<const dmf_graph *> graphs;  // admitted (borrowed; caller keeps them alive)
  std::vector<int32_t> s, t;
  int64_t budget = 0, device_bytes = 0;
  std::vector<std::unique_ptr<Lane>> lanes;
  std::vector<int32_t> lane_of, inst_of;  // per graph: its lane and its instance in the lane
  std::mutex mu;
  std::condition_variable cv_done;
  std::vector<std::deque<Request *>> pending;  // per graph, FIFO
  std::map<int64_t, Request *> all;
  int64_t next_ticket = 1;
  bool stop = false;  // destroy(): serve what is pending, then end the workers
  int waiters = 0;    // threads inside wait()
  int64_t ticks = 0, served = 0, batched_sum = 0;
};

static int64_t footprint(const dmf_graph *g) { return dmf::solver_footprint(g->n, g->m); }

static void tick_loop(dmf_server *S, Lane *L) {
  std::vector<Request *> &batch = L->batch;
  for (;;) {
    batch.clear();  // capacity = the lane's graphs: the selection below never allocates
    {
      std::unique_lock<std::mutex> lk(S->mu);
      L->cv_work.wait(lk, [&] {
        if (S->stop) return true;
        for (int32_t g : L->graphs)
          if (!S->pending[g].empty()) return true;
        return false;
      });
      int64_t bytes = 0;
      for (int32_t g : L->graphs) {
        if (S->pending[g].empty()) continue;
        Request *r = S->pending[g].front();
        const int64_t b = 16LL * (int64_t)r->src.size();
        if (!batch.empty() && bytes + b > L->stage_budget) continue;  // waits for the next tick
        bytes += b;
        S->pending[g].pop_front();
        batch.push_back(r);
      }
      if (batch.empty()) return;  // stopping, and every submitted request is served
    }
    // a failure here (staging growth included) fails this tick's requests and
    // leaves the worker running
    int st = guarded([&]() -> int {
      if (!L->multi) {
        Request *r = batch[0];
        return dmf_apply_updates(L->sv, (int32_t)r->src.size(), r->src.data(), r->dst.data(), r->w.data(),
                                 &L->flows[0]);
      }
      L->I.clear();
      L->A.clear();
      L->B.clear();
      L->W.clear();
      for (Request *r : batch) {
        L->I.insert(L->I.end(), r->src.size(), S->inst_of[r->graph]);
        L->A.insert(L->A.end(), r->src.begin(), r->src.end());
        L->B.insert(L->B.end(), r->dst.begin(), r->dst.end());
        L->W.insert(L->W.end(), r->w.begin(), r->w.end());
      }
      return dmf_multi_apply_updates(L->sv, (int32_t)L->A.size(), L->I.data(), L->A.data(), L->B.data(),
                                     L->W.data(), L->flows.data());
    });
    const char *err = st ? dmf_last_error() : "";
    const auto now = Clock::now();
    {
      std::lock_guard<std::mutex> lk(S->mu);
      for (Request *r : batch) {
        r->status = st;
        try {
          r->error = err;
        } catch (...) {
          // the status alone reaches the waiter
        }
        r->flow = L->flows[L->multi ? S->inst_of[r->graph] : 0];
        r->latency_ms = std::chrono::duration<double, std::milli>(now - r->t_submit).count();
        r->done = true;
      }
      S->ticks++;
      S->served += (int64_t)batch.size();
      S->batched_sum += (int64_t)batch.size();
    }
    S->cv_done.notify_all();
  }
}

// Splits the admitted graphs into lanes and gives each its share of `grid`
// resident blocks (see the file comment).
static void plan_lanes(dmf_server *S, int32_t grid) {
  const int G = (int)S->graphs.size();
  int64_t total = 0;
  for (const dmf_graph *g : S->graphs) total += g->m;
  std::vector<int32_t> order(G);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return S->graphs[a]->m > S->graphs[b]->m; });
  std::vector<std::vector<int32_t>> parts;
  std::vector<int32_t> rest;
  for (int32_t g : order) {
    const bool own = (int)parts.size() < kMaxLanes - 1 && 4 * (int64_t)S->graphs[g]->m >= total;
    if (own) parts.push_back({g});
    else rest.push_back(g);
  }
  if (!rest.empty()) {
    std::sort(rest.begin(), rest.end());
    parts.push_back(rest);
  }
  S->lane_of.assign(G, 0);
  S->inst_of.assign(G, 0);
  std::vector<int64_t> weight;
  for (size_t l = 0; l < parts.size(); l++) {
    std::unique_ptr<Lane> L(new Lane());
    L->graphs = parts[l];
    L->multi = parts[l].size() > 1;
    int64_t w = 1;
    for (size_t i = 0; i < parts[l].size(); i++) {
      S->lane_of[parts[l][i]] = (int32_t)l;
      S->inst_of[parts[l][i]] = (int32_t)i;
      w += S->graphs[parts[l][i]]->m;
    }
    weight.push_back(w);
    L->batch.reserve(parts[l].size());
    L->flows.resize(parts[l].size());
    S->lanes.push_back(std::move(L));
  }
  // shares in proportion to the arcs, at least 1/16 of the grid each, summing to <= grid
  const int nl = (int)S->lanes.size();
  const int32_t floor_share = std::max<int32_t>(1, grid / 16);
  int64_t wsum = 0;
  for (int64_t w : weight) wsum += w;
  int32_t used = 0;
  for (int l = 0; l < nl; l++) {
    const int32_t share = nl == 1 ? grid : std::max<int32_t>(floor_share, (int32_t)((__int128)grid * weight[l] / wsum));
    S->lanes[l]->grid_blocks = share;
    used += share;
  }
  while (used > grid) {  // take the excess from the largest shares
    auto it = std::max_element(S->lanes.begin(), S->lanes.end(),
                               [](const std::unique_ptr<Lane> &a, const std::unique_ptr<Lane> &b) {
                                 return a->grid_blocks < b->grid_blocks;
                               });
    (*it)->grid_blocks--;
    used--;
  }
  const int64_t spare = std::max<int64_t>(S->budget - S->device_bytes, 0);
  for (auto &L : S->lanes) L->stage_budget = std::max<int64_t>(spare / nl, 16LL << 20);
}

static void free_server(dmf_server *S) {
  for (auto &L : S->lanes) {
    if (L->sv) dmf_solver_destroy(L->sv);
    if (L->stream) cudaStreamDestroy(L->stream);
  }
  delete S;
}

extern "C" {

int dmf_server_create(int32_t count, const dmf_graph *const *graphs, const int32_t *s, const int32_t *t,
                      int64_t hbm_budget, const dmf_opts *opts, dmf_server **out) {
  if (count < 1 || !graphs || !s || !t || !out || hbm_budget <= 0)
    return dmf::fail(DMF_ERR_INVALID_ARG, "bad arguments");
  for (int i = 0; i < count; i++)
    if (!graphs[i]) return dmf::fail(DMF_ERR_INVALID_ARG, "graph %d is null", i);
  dmf_server *S = nullptr;
  int st = guarded([&]() -> int {
    S = new dmf_server();
    S->budget = hbm_budget;
    for (int i = 0; i < count; i++) {
      const int64_t f = footprint(graphs[i]);
      if (S->device_bytes + f > hbm_budget) continue;  // not admitted
      S->device_bytes += f;
      S->graphs.push_back(graphs[i]);
      S->s.push_back(s[i]);
      S->t.push_back(t[i]);
    }
    if (S->graphs.empty())
      return dmf::fail(DMF_ERR_OOM, "no graph fits the HBM budget of %lld bytes", (long long)hbm_budget);
    S->pending.resize(S->graphs.size());
    dmf_opts o;
    if (opts) o = *opts;
    else dmf_opts_default(&o);
    if (o.device >= 0 && cudaSetDevice(o.device) != cudaSuccess)
      return dmf::fail(DMF_ERR_CUDA, "cudaSetDevice(%d) failed", o.device);
    int32_t grid = 0;  // the blocks the GPU holds at once
    if (int rc = dmf::resident_solve_blocks(&grid)) return rc;
    const int32_t cap = o.grid_blocks > 0 ? std::min(o.grid_blocks, grid) : grid;
    plan_lanes(S, cap);
    for (auto &L : S->lanes) {
      if (cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking) != cudaSuccess)
        return dmf::fail(DMF_ERR_CUDA, "cudaStreamCreate failed");
      dmf_opts lo = o;
      lo.grid_blocks = L->grid_blocks;
      int rc;
      if (L->multi) {
        std::vector<const dmf_graph *> gs;
        std::vector<int32_t> ss, ts;
        for (int32_t g : L->graphs) {
          gs.push_back(S->graphs[g]);
          ss.push_back(S->s[g]);
          ts.push_back(S->t[g]);
        }
        rc = dmf_multi_create((int32_t)gs.size(), gs.data(), ss.data(), ts.data(), &lo, L->stream, &L->sv);
        if (!rc) rc = dmf_multi_static_maxflow(L->sv, L->flows.data());
      } else {
        const int32_t g = L->graphs[0];
        rc = dmf_solver_create(S->graphs[g], S->s[g], S->t[g], &lo, L->stream, &L->sv);
        if (!rc) rc = dmf_static_maxflow(L->sv, &L->flows[0]);
      }
      // staging for the usual tick up front (a lane that shares graphs batches
      // several requests per tick); larger ticks still grow it
      int64_t arcs = 0;
      for (int32_t g : L->graphs) arcs += S->graphs[g]->m;
      if (!rc) rc = dmf::reserve_updates(L->sv, (int32_t)std::min<int64_t>(arcs, L->multi ? kStageReserve * 4 : kStageReserve));
      if (rc) return rc;
    }
    for (auto &L : S->lanes) L->worker = std::thread(tick_loop, S, L.get());
    return dmf::ok();
  });
  if (st) {
    if (S) {
      char msg[1024];
      std::snprintf(msg, sizeof msg, "%s", dmf_last_error());
      {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
      }
      for (auto &L : S->lanes) {
        L->cv_work.notify_all();
        if (L->worker.joinable()) L->worker.join();
      }
      free_server(S);
      dmf::fail(st, "%s", msg);
    }
    return st;
  }
  *out = S;
  return dmf::ok();
}

int dmf_server_info(const dmf_server *S, int32_t *admitted, int64_t *device_bytes) {
  if (!S) return dmf::fail(DMF_ERR_INVALID_ARG, "null server");
  if (admitted) *admitted = (int32_t)S->graphs.size();
  if (device_bytes) *device_bytes = S->device_bytes;
  return dmf::ok();
}

int dmf_server_lane(const dmf_server *S, int32_t graph, int32_t *lane, int32_t *lanes, int32_t *grid_blocks) {
  if (!S) return dmf::fail(DMF_ERR_INVALID_ARG, "null server");
  if (graph < 0 || graph >= (int32_t)S->graphs.size())
    return dmf::fail(DMF_ERR_INVALID_ARG, "graph %d was not admitted", graph);
  const int32_t l = S->lane_of[graph];
  if (lane) *lane = l;
  if (lanes) *lanes = (int32_t)S->lanes.size();
  if (grid_blocks) *grid_blocks = S->lanes[l]->grid_blocks;
  return dmf::ok();
}

int dmf_server_submit(dmf_server *S, int32_t graph, int32_t k, const int32_t *src, const int32_t *dst,
                      const int32_t *w, int64_t *ticket) {
  if (!S || !ticket || k < 0 || (k > 0 && (!src || !dst || !w))) return dmf::fail(DMF_ERR_INVALID_ARG, "bad arguments");
  if (graph < 0 || graph >= (int32_t)S->graphs.size())
    return dmf::fail(DMF_ERR_INVALID_ARG, "graph %d was not admitted", graph);
  const auto t_arrival = Clock::now();  // latency counts from here, validation included
  const dmf_graph *g = S->graphs[graph];
  // Requests are checked on their own, so one bad request never fails a tick:
  // every update's arc is looked up (in parallel for large requests), then the
  // arc ids are sorted to find repeats.  The first bad update is reported.
  std::vector<int64_t> arcs((size_t)k);
  int32_t bad_range = INT32_MAX, bad_cap = INT32_MAX, bad_arc = INT32_MAX;
#pragma omp parallel for num_threads(kSubmitThreads) schedule(static) reduction(min : bad_range, bad_cap, bad_arc) \
    if (k >= 16384)
  for (int32_t i = 0; i < k; i++) {
    arcs[i] = -1;
    if (src[i] < 0 || dst[i] < 0 || src[i] >= g->n || dst[i] >= g->n) {
      bad_range = std::min(bad_range, i);
      continue;
    }
    if (w[i] < 0 || w[i] > (1 << 30) - 1) {
      bad_cap = std::min(bad_cap, i);
      continue;
    }
    if (src[i] == dst[i]) continue;
    arcs[i] = dmf::find_arc(*g, src[i], dst[i]);
    if (arcs[i] < 0) bad_arc = std::min(bad_arc, i);
  }
  const int32_t first_bad = std::min(bad_range, std::min(bad_cap, bad_arc));
  if (first_bad != INT32_MAX) {
    const int32_t i = first_bad;
    if (i == bad_range) return dmf::fail(DMF_ERR_INVALID_ARG, "update %d: vertex out of range", i);
    if (i == bad_cap) return dmf::fail(DMF_ERR_INVALID_ARG, "update %d: capacity out of range", i);
    return dmf::fail(DMF_ERR_UNKNOWN_ARC, "update %d: arc %d->%d not in graph %d", i, src[i], dst[i], graph);
  }
  if (k >= 16384) __gnu_parallel::sort(arcs.begin(), arcs.end());
  else std::sort(arcs.begin(), arcs.end());
  const auto first_arc = std::upper_bound(arcs.begin(), arcs.end(), (int64_t)-1);  // skip ignored self-loops
  if (std::adjacent_find(first_arc, arcs.end()) != arcs.end())
    return dmf::fail(DMF_ERR_DUP_ARC, "an arc repeats within the request");
  return guarded([&]() -> int {
    std::unique_ptr<Request> r(new Request());
    r->graph = graph;
    r->src.assign(src, src + k);
    r->dst.assign(dst, dst + k);
    r->w.assign(w, w + k);
    r->t_submit = t_arrival;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      const int64_t tk = S->next_ticket;
      auto ins = S->all.emplace(tk, r.get());
      try {
        S->pending[graph].push_back(r.get());
      } catch (...) {
        S->all.erase(ins.first);
        throw;
      }
      S->next_ticket++;
      r->ticket = tk;
      *ticket = tk;
      r.release();  // owned by the server until its wait() returns
    }
    S->lanes[S->lane_of[graph]]->cv_work.notify_one();
    return dmf::ok();
  });
}

int dmf_server_wait(dmf_server *S, int64_t ticket, int64_t *flow, double *latency_ms) {
  if (!S) return dmf::fail(DMF_ERR_INVALID_ARG, "null server");
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->all.find(ticket);
  if (it == S->all.end()) return dmf::fail(DMF_ERR_INVALID_ARG, "unknown ticket %lld", (long long)ticket);
  Request *r = it->second;
  if (r->claimed) return dmf::fail(DMF_ERR_INVALID_ARG, "ticket %lld is already being waited on", (long long)ticket);
  r->claimed = true;
  S->waiters++;
  S->cv_done.wait(lk, [&] { return r->done; });
  S->waiters--;
  S->all.erase(ticket);
  std::unique_ptr<Request> own(r);
  const int st = r->status;
  if (flow) *flow = r->flow;
  if (latency_ms) *latency_ms = r->latency_ms;
  if (st) dmf::fail(st, "%s", r->error.c_str());
  lk.unlock();
  S->cv_done.notify_all();  // destroy() may be waiting for the last waiter
  return st ? st : dmf::ok();
}

int dmf_server_stats(const dmf_server *S, int64_t *ticks, int64_t *served, double *mean_per_tick) {
  if (!S) return dmf::fail(DMF_ERR_INVALID_ARG, "null server");
  auto *M = const_cast<dmf_server *>(S);
  std::lock_guard<std::mutex> lk(M->mu);
  if (ticks) *ticks = S->ticks;
  if (served) *served = S->served;
  if (mean_per_tick) *mean_per_tick = S->ticks ? (double)S->batched_sum / S->ticks : 0.0;
  return dmf::ok();
}

int dmf_server_destroy(dmf_server *S) {
  if (!S) return dmf::ok();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  // the workers serve every request already submitted before they end, so a
  // thread blocked in wait() gets its result; no call may start after this one
  for (auto &L : S->lanes) L->cv_work.notify_all();
  for (auto &L : S->lanes)
    if (L->worker.joinable()) L->worker.join();
  {
    std::unique_lock<std::mutex> lk(S->mu);
    S->cv_done.wait(lk, [&] { return S->waiters == 0; });
  }
  for (auto &kv : S->all) delete kv.second;  // served, never waited on
  free_server(S);
  return dmf::ok();
}

}  // extern "C"
