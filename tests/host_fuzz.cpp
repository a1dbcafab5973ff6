// Randomised inputs for the host half of the library (dmf_host.cpp), built
// with AddressSanitizer and UndefinedBehaviorSanitizer by
// tests/test_host_sanitizers.py: corrupted and truncated graph and update
// files through the loaders, random edge lists through the create_bin-style
// builder, corrupted CSR arrays through the validator, random capacity
// updates (bad ids, missing arcs, negative capacities), and generator edge
// parameters.  Every call must return a status; the sanitizers report any
// out-of-bounds access, overflow or leak.
//
//   host_fuzz <graph.bin> <updates.bin> <scratch file> <iterations>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "dmf.h"

static std::vector<char> read_file(const char *path) {
  std::vector<char> b;
  FILE *f = std::fopen(path, "rb");
  if (!f) return b;
  int c;
  while ((c = std::fgetc(f)) != EOF) b.push_back((char)c);
  std::fclose(f);
  return b;
}

static void write_file(const char *path, const std::vector<char> &b) {
  FILE *f = std::fopen(path, "wb");
  if (!f) std::exit(2);
  if (!b.empty()) std::fwrite(b.data(), 1, b.size(), f);
  std::fclose(f);
}

static void fuzz_loaders(const std::vector<char> &G, const std::vector<char> &U, const char *scratch, int iters,
                         std::mt19937_64 &rng) {
  int graphs = 0, updates = 0;
  for (int it = 0; it < iters; it++) {
    const bool graph = it % 2 == 0;
    std::vector<char> b = graph ? G : U;
    switch (rng() % 4) {
      case 0:  // truncated
        b.resize(rng() % (b.size() + 1));
        break;
      case 1:  // random bytes anywhere
        for (int k = 0; k < 4; k++) b[rng() % b.size()] = (char)rng();
        break;
      case 2: {  // a random header word (n, m or k)
        const int32_t v = (int32_t)rng();
        std::memcpy(b.data() + 4 * (rng() % 2), &v, 4);
        break;
      }
      default: {  // a small (possibly negative) value in any word
        const int32_t v = (int32_t)(rng() % 64) - 8;
        std::memcpy(b.data() + 4 * (rng() % (b.size() / 4)), &v, 4);
        break;
      }
    }
    write_file(scratch, b);
    if (graph) {
      dmf_graph *g = nullptr;
      if (dmf_graph_load(scratch, &g) == DMF_OK) {
        graphs++;
        int32_t n = 0, m = 0;
        dmf_graph_info(g, &n, &m);
        dmf_graph_find_arc(g, (int32_t)(rng() % (n + 2)) - 1, (int32_t)(rng() % (n + 2)) - 1);
        dmf_graph_free(g);
      }
    } else {
      int32_t k = 0, *s = nullptr, *d = nullptr, *w = nullptr;
      if (dmf_updates_load(scratch, &k, &s, &d, &w) == DMF_OK) {
        updates++;
        dmf_free(s);
        dmf_free(d);
        dmf_free(w);
      }
    }
  }
  std::printf("loaders: %d files, %d graphs and %d update files accepted\n", iters, graphs, updates);
}

static void fuzz_builders(int iters, std::mt19937_64 &rng) {
  int built = 0, csr_ok = 0, caps_ok = 0;
  for (int it = 0; it < iters; it++) {
    const int k = (int)(rng() % 200), nv = 1 + (int)(rng() % 40);
    std::vector<int32_t> u(k), v(k), w(k);
    for (int i = 0; i < k; i++) {
      u[i] = (int32_t)(rng() % nv) - (rng() % 50 == 0 ? 1 : 0);
      v[i] = (int32_t)(rng() % nv);
      w[i] = rng() % 30 == 0 ? (int32_t)rng() : (int32_t)(rng() % 1000) - (rng() % 40 == 0 ? 1 : 0);
    }
    dmf_graph *g = nullptr;
    if (dmf_graph_from_edges(k, u.data(), v.data(), w.data(), &g) != DMF_OK) continue;
    built++;
    int32_t n = 0, m = 0;
    dmf_graph_info(g, &n, &m);
    const int32_t *idx, *adj, *cap, *par;
    dmf_graph_arrays(g, &idx, &adj, &cap, &par);
    std::vector<int32_t> I(idx, idx + n + 1), A(adj, adj + m), C(cap, cap + m), P(par, par + m);
    if (m > 0 && rng() % 2) {
      switch (rng() % 4) {
        case 0: A[rng() % m] = (int32_t)(rng() % (n + 3)) - 1; break;
        case 1: P[rng() % m] = (int32_t)(rng() % (m + 3)) - 1; break;
        case 2: C[rng() % m] = (int32_t)rng(); break;
        default: I[1 + rng() % n] = (int32_t)(rng() % (m + 3)) - 1; break;
      }
    }
    dmf_graph *h = nullptr;
    if (dmf_graph_from_csr(n, m, I.data(), A.data(), C.data(), P.data(), &h) == DMF_OK) {
      csr_ok++;
      dmf_graph_free(h);
    }
    const int q = (int)(rng() % 20);
    std::vector<int32_t> s(q), d(q), c(q);
    for (int i = 0; i < q; i++) {
      s[i] = (int32_t)(rng() % (n + 2)) - 1;
      d[i] = (int32_t)(rng() % (n + 2)) - 1;
      c[i] = (int32_t)(rng() % 2000) - 10;
    }
    if (dmf_graph_set_caps(g, q, s.data(), d.data(), c.data()) == DMF_OK) caps_ok++;
    dmf_graph_free(g);
  }
  std::printf("builders: %d edge lists built, %d CSR copies accepted, %d capacity sets accepted\n", built, csr_ok,
              caps_ok);
}

static void extreme_ids() {
  // the largest vertex id leaves no room for the vertex count
  const int32_t u1[1] = {2147483647}, v1[1] = {1}, u2[2] = {0, 2147483647}, v2[2] = {2147483647, 2147483647},
                w[2] = {5, 6};
  dmf_graph *g = nullptr;
  if (dmf_graph_from_edges(1, u1, v1, w, &g) == DMF_OK) dmf_graph_free(g);
  if (dmf_graph_from_edges(2, u2, v2, w, &g) == DMF_OK) dmf_graph_free(g);
  // an empty graph and an empty update file are written without touching data
  const int32_t none = 0;
  if (dmf_graph_from_edges(0, &none, &none, &none, &g) == DMF_OK) {
    dmf_graph_save(g, "/dev/null");
    dmf_graph_free(g);
  }
  dmf_updates_save("/dev/null", 0, nullptr, nullptr, nullptr);
  std::printf("extreme ids: done\n");
}

static void generator_edges() {
  dmf_graph *g = nullptr;
  int32_t s = 0, t = 0;
  if (dmf_gen_rmat(1, 1, 0.57, 0.19, 0.19, 3, 1, 1000, 0, &g, &s, &t) == DMF_OK) dmf_graph_free(g);
  if (dmf_gen_rmat(3, 4, 0.25, 0.25, 0.25, 3, 0, 0, 50, &g, &s, &t) == DMF_OK) dmf_graph_free(g);
  if (dmf_gen_grid(1, 1, 0, 1, 100, 1000, &g, &s, &t) == DMF_OK) dmf_graph_free(g);
  if (dmf_gen_grid(2, 1, 0, 1, 100, 1000, &g, &s, &t) == DMF_OK) {
    int64_t *o = nullptr;
    int32_t *a = nullptr, *b = nullptr, *c = nullptr;
    // every arc with capacity touched, many inserts asked for: more than exist
    if (dmf_gen_batches(g, 3, 1.0, 0.3, 0.3, 0.4, 5, 0, 0, 1, &o, &a, &b, &c) == DMF_OK) {
      dmf_free(o);
      dmf_free(a);
      dmf_free(b);
      dmf_free(c);
    }
    dmf_graph_free(g);
  }
  std::printf("generators: edge parameters done\n");
}

int main(int argc, char **argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: host_fuzz <graph.bin> <updates.bin> <scratch file> <iterations>\n");
    return 2;
  }
  const std::vector<char> G = read_file(argv[1]), U = read_file(argv[2]);
  if (G.size() < 8 || U.size() < 4) return 2;
  const int iters = std::atoi(argv[4]);
  std::mt19937_64 rng(1);
  fuzz_loaders(G, U, argv[3], iters, rng);
  fuzz_builders(iters, rng);
  extreme_ids();
  generator_edges();
  return 0;
}
