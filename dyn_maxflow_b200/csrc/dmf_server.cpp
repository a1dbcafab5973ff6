// dmf_server.cpp -- serving loop over device-resident residual graphs.
//
// Admission: graphs are admitted in the order given while the estimated device
// footprint of their residual state fits the HBM budget; each admitted graph
// stays resident for the server's life, and every batch a request carries is
// applied to it (successive batches per graph, in submission order).
//
// Continuous batching: all admitted graphs live in one batched-instance solver
// (dmf_multi_*).  A worker thread runs ticks; a tick takes, for every graph,
// its oldest waiting request (while the tick's batch stays inside the staging
// budget) and serves them all with one persistent launch, which relabels and
// pushes only inside the touched graphs.  Requests that arrive during a tick
// join the next one.  Instances are independent, so each result equals the
// result of the same request sequence served alone.  No counterpart in the
// reference (a one-shot bench).
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
#include <thread>
#include <vector>

#include "dmf_internal.h"

using dmf::guarded;

namespace {

using Clock = std::chrono::steady_clock;

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

}  // namespace

struct dmf_server {
  std::vector<const dmf_graph *> graphs;  // admitted (borrowed; caller keeps them alive)
  std::vector<int32_t> s, t;
  int64_t budget = 0, device_bytes = 0, stage_budget = 0;
  dmf_solver *sv = nullptr;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::vector<std::deque<Request *>> pending;  // per graph, FIFO
  std::map<int64_t, Request *> all;
  int64_t next_ticket = 1;
  bool stop = false;  // destroy(): serve what is pending, then end the worker
  int waiters = 0;    // threads inside wait()
  std::thread worker;
  int64_t ticks = 0, served = 0, batched_sum = 0;
  // worker-owned staging, sized at create so a tick's selection never allocates
  std::vector<Request *> batch;
  std::vector<int64_t> flows;
};

static int64_t footprint(const dmf_graph *g) {
  // residual state bytes per arc and per vertex (see the solver's data layout)
  return 28LL * g->m + 64LL * g->n;
}

static void tick_loop(dmf_server *S) {
  const int G = (int)S->graphs.size();
  std::vector<Request *> &batch = S->batch;
  for (;;) {
    batch.clear();  // capacity G: the selection below never allocates
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait(lk, [&] {
        if (S->stop) return true;
        for (auto &q : S->pending)
          if (!q.empty()) return true;
        return false;
      });
      int64_t bytes = 0;
      for (int g = 0; g < G; g++) {
        if (S->pending[g].empty()) continue;
        Request *r = S->pending[g].front();
        const int64_t b = 16LL * (int64_t)r->src.size();
        if (!batch.empty() && bytes + b > S->stage_budget) continue;  // waits for the next tick
        bytes += b;
        S->pending[g].pop_front();
        batch.push_back(r);
      }
      if (batch.empty()) return;  // stopping, and every submitted request is served
    }
    // a failure here (staging allocation included) fails this tick's requests
    // and leaves the worker running
    int st = guarded([&]() -> int {
      std::vector<int32_t> I, A, B, W;
      for (Request *r : batch) {
        I.insert(I.end(), r->src.size(), r->graph);
        A.insert(A.end(), r->src.begin(), r->src.end());
        B.insert(B.end(), r->dst.begin(), r->dst.end());
        W.insert(W.end(), r->w.begin(), r->w.end());
      }
      return dmf_multi_apply_updates(S->sv, (int32_t)A.size(), I.data(), A.data(), B.data(), W.data(),
                                     S->flows.data());
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
        r->flow = S->flows[r->graph];
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
    S->stage_budget = std::max<int64_t>(hbm_budget - S->device_bytes, 16LL << 20);
    const size_t G = S->graphs.size();
    S->pending.resize(G);
    S->batch.reserve(G);
    S->flows.resize(G);
    int rc = dmf_multi_create((int32_t)G, S->graphs.data(), S->s.data(), S->t.data(), opts, nullptr, &S->sv);
    if (rc) return rc;
    if ((rc = dmf_multi_static_maxflow(S->sv, S->flows.data()))) return rc;
    S->worker = std::thread(tick_loop, S);
    return dmf::ok();
  });
  if (st) {
    if (S) {
      char msg[1024];
      std::snprintf(msg, sizeof msg, "%s", dmf_last_error());
      dmf_solver_destroy(S->sv);
      delete S;
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
#pragma omp parallel for schedule(static) reduction(min : bad_range, bad_cap, bad_arc) if (k >= 16384)
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
    S->cv_work.notify_one();
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
  S->cv_work.notify_all();
  // the worker serves every request already submitted before it ends, so a
  // thread blocked in wait() gets its result; no call may start after this one
  if (S->worker.joinable()) S->worker.join();
  {
    std::unique_lock<std::mutex> lk(S->mu);
    S->cv_done.wait(lk, [&] { return S->waiters == 0; });
  }
  for (auto &kv : S->all) delete kv.second;  // served, never waited on
  dmf_solver_destroy(S->sv);
  delete S;
  return dmf::ok();
}

}  // extern "C"
