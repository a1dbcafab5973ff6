// dmf_cli.cpp -- drop-in command-line entry points dyn_data_bench,
// dyn_topo_bench, dyn_pp_bench (and the *_large forms), built on libdmf.so.
//
// Same argv and stdout lines as the reference benches:
//   dyn_data_bench  <graph.bin> <update_prefix> <source> <sink>      (files _p1.._p10)
//   dyn_*_bench_large <graph.bin> <update_prefix> <source> <sink> <i> (file _p<i>)
// see code/dyn_data_bench.cu:495-567, dyn_topo_bench.cu:399-476,
// dyn_pp_bench.cu:624-695 and dyn_data_bench_large.cu:500-517.  For every file
// and each kernel_cycles value in {avg_deg-1, avg_deg, avg_deg+1} it runs the
// dynamic path (fresh device state of the original graph, static solve, one
// batch) and the from-scratch path, and prints PANIC when the flows differ.
// The "updates size" line prints 2k, as the reference does (code/update.hpp:72,83
// returns k zero-typed records followed by the k updates).
// With DMF_CLI_JSON=1 a JSON record per run is printed as well.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "dmf.h"

#ifndef DMF_CLI_VARIANT
#define DMF_CLI_VARIANT "data"
#endif
#ifndef DMF_CLI_LARGE
#define DMF_CLI_LARGE 0
#endif

static int variant_id(const char *v) {
  if (!std::strcmp(v, "topo")) return DMF_VARIANT_TOPO;
  if (!std::strcmp(v, "pp")) return DMF_VARIANT_PP;
  return DMF_VARIANT_DATA;
}

static int die(int st, const char *what) {
  std::fprintf(stderr, "%s failed: [%s] %s\n", what, dmf_status_string(st), dmf_last_error());
  return 1;
}

int main(int argc, char **argv) {
  const int need = DMF_CLI_LARGE ? 6 : 5;
  if (argc < need) {
    std::fprintf(stderr, "usage: %s <graph.bin> <update_prefix> <source> <sink>%s\n", argv[0],
                 DMF_CLI_LARGE ? " <i>" : "");
    return 1;
  }
  const int variant = variant_id(DMF_CLI_VARIANT);
  const bool json = std::getenv("DMF_CLI_JSON") && std::atoi(std::getenv("DMF_CLI_JSON"));
  const int source = std::atoi(argv[3]), sink = std::atoi(argv[4]);
  std::printf("source:%d sink:%d\n", source, sink);
  // what a failing step leaves behind is released before the exit
  dmf_graph *g = nullptr;
  dmf_solver *sv = nullptr;
  int32_t *us = nullptr, *ud = nullptr, *uw = nullptr;
  auto release_batch = [&]() {
    dmf_solver_destroy(sv);  // NULL is fine
    sv = nullptr;
    dmf_free(us);
    dmf_free(ud);
    dmf_free(uw);
    us = ud = uw = nullptr;
  };
  auto fail_step = [&](int status, const char *what) {
    const int r = die(status, what);  // first: a successful destroy clears the last error
    release_batch();
    dmf_graph_free(g);
    return r;
  };
  int st = dmf_graph_load(argv[1], &g);
  if (st) return die(st, "graph load");
  int32_t V = 0, E = 0;
  dmf_graph_info(g, &V, &E);
  if (variant == DMF_VARIANT_TOPO) {
    std::printf("V:%d\n", V);
    std::printf("E:%d\n", E);
  }
  int first = 1, last = 10;
  if (DMF_CLI_LARGE) first = last = std::atoi(argv[5]);
  int rc = 0;
  for (int i = first; i <= last; i++) {
    std::string fname = std::string(argv[2]) + "_p" + std::to_string(i) + ".bin";
    std::printf("Processing file: %s\n", fname.c_str());
    int32_t k = 0;
    st = dmf_updates_load(fname.c_str(), &k, &us, &ud, &uw);
    if (st) {
      // the reference prints the loader error and continues with an empty batch
      std::fprintf(stderr, "Error: %s\n", dmf_last_error());
      k = 0;
    }
    std::printf("updates size:%d\n", 2 * k);
    const int avg_deg = V > 0 ? E / V : 0;
    int cycles[3], nc = 0;
    if (avg_deg > 1) cycles[nc++] = avg_deg - 1;
    if (avg_deg > 0) cycles[nc++] = avg_deg;
    cycles[nc++] = avg_deg + 1;
    for (int ci = 0; ci < nc; ci++) {
      const int kc = cycles[ci];
      std::printf("=======kernel cycles %d =======\n", kc);
      dmf_opts o;
      dmf_opts_default(&o);
      o.variant = variant;
      o.kernel_cycles = kc;
      // dynamic path: recalculate_max_flow (code/dyn_data_bench.cu:171-298)
      if ((st = dmf_solver_create(g, source, sink, &o, nullptr, &sv))) return fail_step(st, "solver create");
      int64_t f0 = 0, dyn = 0, stat = 0;
      dmf_stats sst;
      if ((st = dmf_static_maxflow(sv, &f0))) return fail_step(st, "static solve");
      dmf_stats_get(sv, &sst);
      if (variant == DMF_VARIANT_PP) std::printf("static main push cnt:%lld GPU Time: %.6f ms\n",
                                                 (long long)sst.push_rounds, sst.last_ms);
      else std::printf("static GPU Time: %.6f ms\n", sst.last_ms);
      if (variant == DMF_VARIANT_TOPO) std::printf("flow:%lld  kernel cycles:%d\n", (long long)f0, kc);
      if ((st = dmf_apply_updates(sv, k, us, ud, uw, &dyn))) return fail_step(st, "apply updates");
      dmf_stats dst;
      dmf_stats_get(sv, &dst);
      std::printf("total GPU Time: %.6f ms\n", dst.last_ms);
      std::printf("DYN TIME:%.6fms true_cnt=%d cnt=%d per batch time:%.6f\n", dst.last_ms, 1, 1, dst.last_ms);
      std::printf("Dynamic flow:%lld\n", (long long)dyn);
      dmf_solver_destroy(sv);
      sv = nullptr;
      // from-scratch path: static_recalculate (code/dyn_data_bench.cu:325-492)
      if ((st = dmf_solver_create(g, source, sink, &o, nullptr, &sv))) return fail_step(st, "solver create");
      if ((st = dmf_recompute(sv, k, us, ud, uw, &stat))) return fail_step(st, "recompute");
      dmf_stats rst;
      dmf_stats_get(sv, &rst);
      if (variant == DMF_VARIANT_PP) std::printf("static  UPDATE GPU Time: %.6f ms\n", rst.last_ms);
      else std::printf("STATIC UPDATE GPU Time: %.6f ms\n", rst.last_ms);
      dmf_solver_destroy(sv);
      sv = nullptr;
      if (dyn != stat) {
        std::printf("<<<<<<<<<<<<<<<<<<<<<<<<PANIC NOT MATCHING dynflow:%lld statflow:%lld>>>>>>>>>>>>>>>>>>>>>>>>>>>\n",
                    (long long)dyn, (long long)stat);
        rc = 3;
      }
      if (json)
        std::printf("{\"file\": \"%s\", \"variant\": \"%s\", \"kernel_cycles\": %d, \"k\": %d, \"static_flow\": %lld, "
                    "\"dynamic_flow\": %lld, \"recompute_flow\": %lld, \"static_ms\": %.6f, \"dynamic_ms\": %.6f, "
                    "\"recompute_ms\": %.6f}\n",
                    fname.c_str(), DMF_CLI_VARIANT, kc, k, (long long)f0, (long long)dyn, (long long)stat,
                    sst.last_ms, dst.last_ms, rst.last_ms);
    }
    release_batch();
  }
  dmf_graph_free(g);
  return rc;
}
