// dmf_tool.cpp -- input tooling on libdmf.so's host API (no GPU needed).
//
//   dmf_tool weight <in.mtx> <out.txt>
//       edge list -> "u v w", w ~ U[1,100] from std::mt19937(42) with
//       std::uniform_int_distribution (input_create/weight.cpp:14-58); lines that
//       are empty or start with '%' are skipped.
//   dmf_tool cb <in.txt> <out.bin>
//       "u v w" text -> CSR .bin with create_bin semantics
//       (input_create/create_bin.cpp:67-141), in O(k log k).
//   dmf_tool cb_update <in.txt> <out.bin>
//       first line k, then k lines "u v w" -> update .bin
//       (input_create/create_update_bin.cpp:11-66).
//   dmf_tool gen-grid <rows> <cols> <seed> <out.bin>       (caps U[1,100], s/t arcs 1000)
//   dmf_tool gen-rmat <scale> <seed> <reserve> <out.bin>   (16*2^scale samples, caps U[1,1000])
//   dmf_tool gen-batches <graph.bin> <nbatches> <frac> <seed> <prefix> [cumulative]
//       successive mixed batches (40/40/10/10) written as <prefix>_p<i>.bin; with
//       "cumulative", file i holds the net capacities of batches 1..i, the form
//       the reference benches replay against the original graph.
// Prints the source/sink for the generators.  Exit status 0 on success.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "dmf.h"

static int usage() {
  std::fprintf(stderr,
               "usage: dmf_tool weight|cb|cb_update <in> <out>\n"
               "       dmf_tool gen-grid <rows> <cols> <seed> <out.bin>\n"
               "       dmf_tool gen-rmat <scale> <seed> <reserve> <out.bin>\n"
               "       dmf_tool gen-batches <graph.bin> <nbatches> <frac> <seed> <prefix> [cumulative]\n");
  return 2;
}

static int die(int st, const char *what) {
  std::fprintf(stderr, "%s: [%s] %s\n", what, dmf_status_string(st), dmf_last_error());
  return 1;
}

static int cmd_weight(const char *in, const char *out) {
  std::ifstream fin(in);
  std::ofstream fout(out);
  if (!fin || !fout) {
    std::fprintf(stderr, "cannot open %s or %s\n", in, out);
    return 1;
  }
  std::mt19937 rng(42);
  std::uniform_int_distribution<int> dist(1, 100);
  std::string line;
  while (std::getline(fin, line)) {
    if (line.empty() || line[0] == '%') continue;
    std::istringstream iss(line);
    int u, v;
    if (!(iss >> u >> v)) continue;
    fout << u << " " << v << " " << dist(rng) << "\n";
  }
  return 0;
}

static int cmd_cb(const char *in, const char *out) {
  std::ifstream fin(in);
  if (!fin) {
    std::fprintf(stderr, "cannot open %s\n", in);
    return 1;
  }
  std::vector<int32_t> U, V, W;
  std::string line;
  while (std::getline(fin, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream iss(line);
    int u = 0, v = 0, w = 0;
    iss >> u >> v >> w;
    U.push_back(u);
    V.push_back(v);
    W.push_back(w);
  }
  dmf_graph *g = nullptr;
  int st = dmf_graph_from_edges((int64_t)U.size(), U.data(), V.data(), W.data(), &g);
  if (st) return die(st, "build");
  st = dmf_graph_save(g, out);
  int32_t n = 0, m = 0;
  dmf_graph_info(g, &n, &m);
  dmf_graph_free(g);
  if (st) return die(st, "save");
  std::printf("CSR written to %s (%d nodes, %d edges)\n", out, n, m);
  return 0;
}

static int cmd_cb_update(const char *in, const char *out) {
  std::ifstream fin(in);
  if (!fin) {
    std::fprintf(stderr, "cannot open %s\n", in);
    return 1;
  }
  std::string line;
  int k = 0;
  if (!std::getline(fin, line) || !(std::istringstream(line) >> k) || k < 0) {
    std::fprintf(stderr, "%s: first line must hold the batch size\n", in);
    return 1;
  }
  std::vector<int32_t> S, D, W;
  while ((int)S.size() < k && std::getline(fin, line)) {
    std::istringstream iss(line);
    int u = 0, v = 0, w = 0;
    iss >> u >> v >> w;
    S.push_back(u);
    D.push_back(v);
    W.push_back(w);
  }
  // the reference writes k records even when the text holds fewer (unset ones
  // are whatever malloc returned); here missing records are an error
  if ((int)S.size() < k) {
    std::fprintf(stderr, "%s: %d records announced, %zu present\n", in, k, S.size());
    return 1;
  }
  int st = dmf_updates_save(out, k, S.data(), D.data(), W.data());
  return st ? die(st, "save") : 0;
}

int main(int argc, char **argv) {
  if (argc < 2) return usage();
  const std::string c = argv[1];
  if ((c == "weight" || c == "cb" || c == "cb_update") && argc == 4) {
    if (c == "weight") return cmd_weight(argv[2], argv[3]);
    if (c == "cb") return cmd_cb(argv[2], argv[3]);
    return cmd_cb_update(argv[2], argv[3]);
  }
  dmf_graph *g = nullptr;
  int32_t s = 0, t = 0;
  int st = 0;
  if (c == "gen-grid" && argc == 6) {
    st = dmf_gen_grid(std::atoi(argv[2]), std::atoi(argv[3]), std::strtoull(argv[4], nullptr, 10), 1, 100, 1000,
                      &g, &s, &t);
    if (!st) st = dmf_graph_save(g, argv[5]);
  } else if (c == "gen-rmat" && argc == 6) {
    const int scale = std::atoi(argv[2]);
    st = dmf_gen_rmat(scale, (int64_t)16 << scale, 0.57, 0.19, 0.19, std::strtoull(argv[3], nullptr, 10), 1, 1000,
                      std::atoll(argv[4]), &g, &s, &t);
    if (!st) st = dmf_graph_save(g, argv[5]);
  } else if (c == "gen-batches" && (argc == 7 || argc == 8)) {
    st = dmf_graph_load(argv[2], &g);
    if (st) return die(st, "load");
    const int nb = std::atoi(argv[3]);
    int64_t *ofs = nullptr;
    int32_t *S = nullptr, *D = nullptr, *W = nullptr;
    st = dmf_gen_batches(g, nb, std::atof(argv[4]), 0.4, 0.4, 0.1, 500, 1, 1000, std::strtoull(argv[5], nullptr, 10),
                         &ofs, &S, &D, &W);
    if (st) {
      dmf_graph_free(g);
      return die(st, "gen-batches");
    }
    const bool cumulative = argc == 8 && std::strcmp(argv[7], "cumulative") == 0;
    std::map<std::pair<int32_t, int32_t>, int32_t> net;
    for (int b = 0; b < nb && !st; b++) {
      std::vector<int32_t> fs, fd, fw;
      for (int64_t i = ofs[b]; i < ofs[b + 1]; i++) {
        if (cumulative) net[{S[i], D[i]}] = W[i];
        else {
          fs.push_back(S[i]);
          fd.push_back(D[i]);
          fw.push_back(W[i]);
        }
      }
      if (cumulative)
        for (auto &kv : net) {
          fs.push_back(kv.first.first);
          fd.push_back(kv.first.second);
          fw.push_back(kv.second);
        }
      const std::string name = std::string(argv[6]) + "_p" + std::to_string(b + 1) + ".bin";
      st = dmf_updates_save(name.c_str(), (int32_t)fs.size(), fs.data(), fd.data(), fw.data());
    }
    dmf_free(ofs);
    dmf_free(S);
    dmf_free(D);
    dmf_free(W);
    dmf_graph_free(g);
    return st ? die(st, "save") : 0;
  } else {
    return usage();
  }
  dmf_graph_free(g);  // NULL when generation failed
  if (st) return die(st, c.c_str());
  std::printf("source:%d sink:%d\n", s, t);
  return 0;
}
