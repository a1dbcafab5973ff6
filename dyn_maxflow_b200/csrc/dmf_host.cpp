// dmf_host.cpp -- host half of libdmf.so: errors, the two .bin formats, the
// CSR builder with create_bin semantics, and the seeded generators.
//
// Reference formats (ShruthiKannappan/dyn_maxflow):
//   graph  : code/graph.hpp:202-223, written by input_create/create_bin.cpp:18-64
//   updates: code/update.hpp:52-88, written by input_create/create_update_bin.cpp:41-49
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>
#include <unordered_set>

#ifdef _OPENMP
#include <parallel/algorithm>
#endif

#ifdef _OPENMP
#include <omp.h>
#endif

#include "dmf_internal.h"

namespace dmf {

static thread_local std::string g_err;

int fail(int status, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  try {
    g_err = buf;
  } catch (...) {
    // no room for the message: the status alone still reaches the caller
  }
  return status;
}

int ok() {
  g_err.clear();
  return DMF_OK;
}

int validate(const dmf_graph &g) {
  const int32_t n = g.n, m = g.m;
  if (n < 0 || m < 0) return fail(DMF_ERR_BAD_FILE, "negative sizes n=%d m=%d", n, m);
  if ((int64_t)g.off.size() != (int64_t)n + 1 || (int64_t)g.adj.size() != m ||
      (int64_t)g.w.size() != m || (int64_t)g.par.size() != m)
    return fail(DMF_ERR_BAD_FILE, "array sizes do not match n=%d m=%d", n, m);
  if (g.off[0] != 0 || g.off[n] != m)
    return fail(DMF_ERR_BAD_FILE, "offsets must start at 0 and end at m (got %d, %d)", g.off[0], g.off[n]);
  for (int32_t v = 0; v < n; v++)
    if (g.off[v] > g.off[v + 1]) return fail(DMF_ERR_BAD_FILE, "offsets decrease at vertex %d", v);
  // (code << 32) | (INT32_MAX - arc): the most severe defect, at its lowest arc,
  // whatever the thread count
  int64_t worst = 0;
#pragma omp parallel for schedule(static) reduction(max : worst)
  for (int32_t v = 0; v < n; v++) {
    for (int32_t e = g.off[v]; e < g.off[v + 1]; e++) {
      int32_t h = g.adj[e], p = g.par[e];
      int code = 0;
      if (h < 0 || h >= n) code = 1;
      else if (h == v) code = 2;
      else if (p < 0 || p >= m) code = 3;
      else if (g.par[p] != e || g.adj[p] != v || p < g.off[h] || p >= g.off[h + 1]) code = 4;
      else if (g.w[e] < 0) code = 5;
      else if ((int64_t)g.w[e] + g.w[p] > INT32_MAX) code = 6;
      if (code) worst = std::max(worst, ((int64_t)code << 32) | (int64_t)(INT32_MAX - e));
    }
  }
  const int bad = (int)(worst >> 32);
  const int64_t bad_e = INT32_MAX - (worst & 0xffffffffll);
  switch (bad) {
    case 0: return DMF_OK;
    case 1: return fail(DMF_ERR_BAD_FILE, "arc %lld: head out of range", (long long)bad_e);
    case 2: return fail(DMF_ERR_BAD_FILE, "arc %lld: self-loop", (long long)bad_e);
    case 3: return fail(DMF_ERR_BAD_FILE, "arc %lld: partner index out of range", (long long)bad_e);
    case 4: return fail(DMF_ERR_BAD_FILE, "arc %lld: partner is not the reverse arc", (long long)bad_e);
    case 5: return fail(DMF_ERR_BAD_FILE, "arc %lld: negative capacity", (long long)bad_e);
    default: return fail(DMF_ERR_OVERFLOW, "arc %lld: capacity + partner capacity exceeds int32", (long long)bad_e);
  }
}

void build_sorted_index(dmf_graph &g) {
  if ((int64_t)g.sidx.size() == g.m) return;
  g.sidx.resize(g.m);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t v = 0; v < g.n; v++) {
    int32_t *b = g.sidx.data() + g.off[v], *e = g.sidx.data() + g.off[v + 1];
    std::iota(b, e, g.off[v]);
    std::sort(b, e, [&](int32_t x, int32_t y) {
      return g.adj[x] != g.adj[y] ? g.adj[x] < g.adj[y] : x < y;
    });
  }
}

int64_t find_arc(const dmf_graph &g, int32_t src, int32_t dst) {
  if (src < 0 || src >= g.n) return -1;
  const int32_t *b = g.sidx.data() + g.off[src], *e = g.sidx.data() + g.off[src + 1];
  // last arc among equal heads (OnAdd_kernel keeps the last match, code/dyn_data.h:196-201)
  const int32_t *it = std::upper_bound(b, e, dst, [&](int32_t d, int32_t x) { return d < g.adj[x]; });
  if (it == b || g.adj[*(it - 1)] != dst) return -1;
  return *(it - 1);
}

// create_bin semantics (input_create/create_bin.cpp:67-124), in O(k log deg):
// events 2j = arc (u_j, v_j) with weight w_j, 2j+1 = arc (v_j, u_j) weight 0,
// bucketed by tail in event order; per tail, duplicates merged (weights summed)
// and unique arcs kept in order of their first event.
//
// The bucketing runs in parallel and keeps event order: the tails are cut into
// ranges of about equal event counts; each thread scatters a contiguous slice
// of the edges into the ranges (so every range receives its events in edge
// order), then each range is bucketed by tail on its own.
int build_from_edges(int64_t k, const int32_t *u, const int32_t *v, const int32_t *w,
                     dmf_graph **out) {
  if (k < 0 || (k > 0 && (!u || !v || !w))) return fail(DMF_ERR_INVALID_ARG, "bad edge arrays");
  int32_t maxnode = -1;
  int64_t kept = 0, first_bad = INT64_MAX;
#pragma omp parallel for schedule(static) reduction(max : maxnode) reduction(+ : kept) reduction(min : first_bad)
  for (int64_t i = 0; i < k; i++) {
    if (u[i] < 0 || v[i] < 0) {
      first_bad = std::min(first_bad, i);
      continue;
    }
    if (u[i] == v[i]) continue;
    maxnode = std::max(maxnode, std::max(u[i], v[i]));
    kept++;
  }
  if (first_bad != INT64_MAX)
    return fail(DMF_ERR_INVALID_ARG, "negative vertex id at edge %lld", (long long)first_bad);
  if (maxnode == INT32_MAX)  // the vertex count would not fit int32
    return fail(DMF_ERR_INVALID_ARG, "vertex id %d leaves no room for the vertex count", maxnode);
  const int32_t n = maxnode + 1;
  std::vector<int64_t> bofs((size_t)n + 1, 0);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < k; i++) {
    if (u[i] == v[i]) continue;
#pragma omp atomic
    bofs[u[i] + 1]++;
#pragma omp atomic
    bofs[v[i] + 1]++;
  }
  for (int32_t x = 0; x < n; x++) bofs[x + 1] += bofs[x];
  struct Ev { int32_t head; int32_t wt; };
  std::vector<Ev> ev((size_t)(2 * kept));
  {
    int nth = 1;
#ifdef _OPENMP
    nth = omp_get_max_threads();
#endif
    // tail ranges [vb[r], vb[r+1]) of about equal event counts
    const int R = std::max(1, std::min(std::min(8 * nth, 65535), n > 0 ? n : 1));
    std::vector<int32_t> vb((size_t)R + 1, n);
    vb[0] = 0;
    for (int r = 1; r < R; r++) {
      const int64_t want = (int64_t)((__int128)2 * kept * r / R);
      vb[r] = (int32_t)(std::lower_bound(bofs.begin(), bofs.begin() + n, want) - bofs.begin());
      vb[r] = std::max(vb[r], vb[r - 1]);
    }
    std::vector<uint16_t> rng_of(n > 0 ? (size_t)n : 1);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < R; r++)
      for (int32_t x = vb[r]; x < vb[r + 1]; x++) rng_of[x] = (uint16_t)r;
    // edge slices: slice t counts its events per range, then scatters them
    const int T = nth;
    std::vector<int64_t> cnt((size_t)T * R, 0);
    struct TEv { int32_t tail; int32_t head; int32_t wt; };
    std::vector<TEv> staged((size_t)(2 * kept));
#pragma omp parallel num_threads(T)
    {
      int t = 0;
#ifdef _OPENMP
      t = omp_get_thread_num();
      const int tt = omp_get_num_threads();
#else
      const int tt = 1;
#endif
      const int64_t b = (int64_t)((__int128)k * t / tt), e = (int64_t)((__int128)k * (t + 1) / tt);
      int64_t *c = cnt.data() + (size_t)t * R;
      for (int64_t i = b; i < e; i++) {
        if (u[i] == v[i]) continue;
        c[rng_of[u[i]]]++;
        c[rng_of[v[i]]]++;
      }
#pragma omp barrier
#pragma omp single
      {
        for (int r = 0; r < R; r++) {
          int64_t pos = bofs[vb[r]];
          for (int q = 0; q < tt; q++) {
            const int64_t x = cnt[(size_t)q * R + r];
            cnt[(size_t)q * R + r] = pos;
            pos += x;
          }
        }
      }
      for (int64_t i = b; i < e; i++) {
        if (u[i] == v[i]) continue;
        staged[c[rng_of[u[i]]]++] = {u[i], v[i], w[i]};
        staged[c[rng_of[v[i]]]++] = {v[i], u[i], 0};
      }
    }
    std::vector<uint16_t>().swap(rng_of);
    // per range: events into their tails' buckets, in order
    std::vector<int64_t> fill(bofs.begin(), bofs.end() - 1);
#pragma omp parallel for schedule(dynamic, 1)
    for (int r = 0; r < R; r++)
      for (int64_t j = bofs[vb[r]]; j < bofs[vb[r + 1]]; j++) {
        const TEv &s = staged[j];
        ev[fill[s.tail]++] = {s.head, s.wt};
      }
  }
  // per tail: unique heads in first-event order, weights summed
  std::vector<int32_t> ucount(n, 0);
  int overflow = 0, nomem = 0;
#pragma omp parallel
  {
    // an exception may not leave the parallel region: a failed allocation
    // is flagged and reported after it
    std::vector<int64_t> ord;
    std::vector<Ev> tmp;
#pragma omp for schedule(dynamic, 256) reduction(| : overflow, nomem)
    for (int32_t x = 0; x < n; x++) {
      int64_t b = bofs[x], e = bofs[x + 1], len = e - b;
      try {
        ord.resize(len);
        tmp.resize(len);
      } catch (...) {
        nomem = 1;
        continue;
      }
      std::iota(ord.begin(), ord.end(), b);
      std::stable_sort(ord.begin(), ord.end(), [&](int64_t p, int64_t q) { return ev[p].head < ev[q].head; });
      // merge equal heads into the first occurrence (smallest position)
      int64_t nu = 0;
      for (int64_t i = 0; i < len;) {
        int64_t j = i;
        int64_t first = ord[i];
        int64_t sum = 0;
        while (j < len && ev[ord[j]].head == ev[ord[i]].head) { sum += ev[ord[j]].wt; j++; }
        if (sum > INT32_MAX) overflow = 1;
        ord[nu++] = first;
        ev[first].wt = (int32_t)sum;
        i = j;
      }
      ord.resize(nu);
      std::sort(ord.begin(), ord.end());  // first-touch order
      // compact unique arcs to the front of the bucket, in order
      for (int64_t i = 0; i < nu; i++) tmp[i] = ev[ord[i]];
      for (int64_t i = 0; i < nu; i++) ev[b + i] = tmp[i];
      ucount[x] = (int32_t)nu;
    }
  }
  if (nomem) return fail(DMF_ERR_OOM, "host allocation failed");
  if (overflow) return fail(DMF_ERR_OVERFLOW, "summed duplicate capacity exceeds int32");
  int64_t m64 = 0;
  for (int32_t x = 0; x < n; x++) m64 += ucount[x];
  if (m64 > INT32_MAX) return fail(DMF_ERR_INVALID_ARG, "too many arcs (%lld) for int32 indices", (long long)m64);
  std::unique_ptr<dmf_graph> g(new dmf_graph());
  g->n = n;
  g->m = (int32_t)m64;
  g->off.resize((size_t)n + 1);
  g->adj.resize(g->m);
  g->w.resize(g->m);
  g->par.resize(g->m);
  g->off[0] = 0;
  for (int32_t x = 0; x < n; x++) g->off[x + 1] = g->off[x] + ucount[x];
#pragma omp parallel for schedule(static)
  for (int32_t x = 0; x < n; x++)
    for (int32_t i = 0; i < ucount[x]; i++) {
      g->adj[g->off[x] + i] = ev[bofs[x] + i].head;
      g->w[g->off[x] + i] = ev[bofs[x] + i].wt;
    }
  std::vector<Ev>().swap(ev);
  build_sorted_index(*g);
  // Partners: every arc x->h has exactly one reverse arc h->x (heads are unique
  // per tail after the merge).  The pair is resolved once, from its smaller
  // endpoint, by a binary search over h's heads laid out in sorted order.
  {
    std::vector<int32_t> sh((size_t)g->m);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t x = 0; x < n; x++)
      for (int32_t i = g->off[x]; i < g->off[x + 1]; i++) sh[i] = g->adj[g->sidx[i]];
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t x = 0; x < n; x++)
      for (int32_t e = g->off[x]; e < g->off[x + 1]; e++) {
        const int32_t h = g->adj[e];
        if (h < x) continue;
        const int32_t *b = sh.data() + g->off[h], *end = sh.data() + g->off[h + 1];
        const int32_t p = g->sidx[g->off[h] + (int32_t)(std::lower_bound(b, end, x) - b)];
        g->par[e] = p;
        g->par[p] = e;
      }
  }
  *out = g.release();
  return ok();
}

}  // namespace dmf

using namespace dmf;

// ---------------------------------------------------------------------------
// small deterministic RNG: splitmix64 seeding + xoshiro256**
// ---------------------------------------------------------------------------
namespace {

inline uint64_t splitmix64(uint64_t &x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    uint64_t x = seed;
    for (auto &w : s) w = splitmix64(x);
  }
  static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return r;
  }
  // uniform integer in [lo, hi] (hi >= lo), multiply-shift
  int64_t uniform(int64_t lo, int64_t hi) {
    uint64_t span = (uint64_t)(hi - lo) + 1;
    return lo + (int64_t)(((unsigned __int128)next() * span) >> 64);
  }
  double unit() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
};

}  // namespace

// ---------------------------------------------------------------------------
// C ABI: errors, graphs, formats
// ---------------------------------------------------------------------------
extern "C" {

const char *dmf_last_error(void) { return g_err.c_str(); }

const char *dmf_status_string(int st) {
  switch (st) {
    case DMF_OK: return "ok";
    case DMF_ERR_INVALID_ARG: return "invalid argument";
    case DMF_ERR_BAD_FILE: return "bad file";
    case DMF_ERR_UNKNOWN_ARC: return "unknown arc";
    case DMF_ERR_DUP_ARC: return "duplicate arc in batch";
    case DMF_ERR_OOM: return "out of memory";
    case DMF_ERR_NO_CONVERGENCE: return "no convergence";
    case DMF_ERR_CUDA: return "cuda error";
    case DMF_ERR_TIMEOUT: return "device wait timed out";
    case DMF_ERR_OVERFLOW: return "capacity overflow";
    case DMF_ERR_NOT_SOLVED: return "not solved";
    case DMF_ERR_HOST: return "host runtime error";
    default: return "unknown status";
  }
}

void dmf_opts_default(dmf_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->variant = DMF_VARIANT_DATA;
  o->device = -1;
}

void dmf_free(void *p) { std::free(p); }

int dmf_graph_load(const char *path, dmf_graph **out) {
  if (!path || !out) return fail(DMF_ERR_INVALID_ARG, "null argument");
  return guarded([&]() -> int {
    std::unique_ptr<FILE, int (*)(FILE *)> f(std::fopen(path, "rb"), &std::fclose);
    if (!f) return fail(DMF_ERR_BAD_FILE, "cannot open %s", path);
    std::fseek(f.get(), 0, SEEK_END);
    long long size = std::ftell(f.get());
    std::fseek(f.get(), 0, SEEK_SET);
    int32_t hdr[2] = {0, 0};
    if (std::fread(hdr, 4, 2, f.get()) != 2) return fail(DMF_ERR_BAD_FILE, "%s: shorter than the 8-byte header", path);
    long long want = 8 + 4LL * ((long long)hdr[0] + 1) + 12LL * hdr[1];
    if (hdr[0] < 0 || hdr[1] < 0 || size != want)
      return fail(DMF_ERR_BAD_FILE, "%s: size %lld does not match n=%d m=%d (expected %lld)", path, size, hdr[0],
                  hdr[1], want);
    std::unique_ptr<dmf_graph> g(new dmf_graph());
    g->n = hdr[0];
    g->m = hdr[1];
    g->off.resize((size_t)g->n + 1);
    g->adj.resize(g->m);
    g->w.resize(g->m);
    g->par.resize(g->m);
    bool okr = std::fread(g->off.data(), 4, g->off.size(), f.get()) == g->off.size() &&
               std::fread(g->adj.data(), 4, g->m, f.get()) == (size_t)g->m &&
               std::fread(g->w.data(), 4, g->m, f.get()) == (size_t)g->m &&
               std::fread(g->par.data(), 4, g->m, f.get()) == (size_t)g->m;
    f.reset();
    if (!okr) return fail(DMF_ERR_BAD_FILE, "%s: short read", path);
    int st = validate(*g);
    if (st) {
      std::string msg = std::string(path) + ": " + g_err;
      return fail(st, "%s", msg.c_str());
    }
    build_sorted_index(*g);
    *out = g.release();
    return ok();
  });
}

int dmf_graph_from_csr(int32_t n, int32_t m, const int32_t *index, const int32_t *adj,
                       const int32_t *w, const int32_t *par, dmf_graph **out) {
  if (!out || n < 0 || m < 0 || !index || (m > 0 && (!adj || !w || !par)))
    return fail(DMF_ERR_INVALID_ARG, "bad CSR arguments");
  return guarded([&]() -> int {
    std::unique_ptr<dmf_graph> g(new dmf_graph());
    g->n = n;
    g->m = m;
    g->off.assign(index, index + (size_t)n + 1);
    g->adj.assign(adj, adj + m);
    g->w.assign(w, w + m);
    g->par.assign(par, par + m);
    int st = validate(*g);
    if (st) return st;
    build_sorted_index(*g);
    *out = g.release();
    return ok();
  });
}

int dmf_graph_from_edges(int64_t k, const int32_t *u, const int32_t *v, const int32_t *w,
                         dmf_graph **out) {
  if (!out) return fail(DMF_ERR_INVALID_ARG, "null out");
  return guarded([&] { return build_from_edges(k, u, v, w, out); });
}

}  // extern "C"

namespace {
// `count` int32 words; an empty array writes nothing (its pointer may be null,
// which fwrite does not accept even for a zero count).
bool put_words(FILE *f, const int32_t *p, size_t count) { return count == 0 || std::fwrite(p, 4, count, f) == count; }
}  // namespace

extern "C" {

int dmf_graph_save(const dmf_graph *g, const char *path) {
  if (!g || !path) return fail(DMF_ERR_INVALID_ARG, "null argument");
  FILE *f = std::fopen(path, "wb");
  if (!f) return fail(DMF_ERR_BAD_FILE, "cannot open %s for writing", path);
  bool okw = std::fwrite(&g->n, 4, 1, f) == 1 && std::fwrite(&g->m, 4, 1, f) == 1 &&
             put_words(f, g->off.data(), g->off.size()) && put_words(f, g->adj.data(), (size_t)g->m) &&
             put_words(f, g->w.data(), (size_t)g->m) && put_words(f, g->par.data(), (size_t)g->m);
  okw = (std::fclose(f) == 0) && okw;
  return okw ? ok() : fail(DMF_ERR_BAD_FILE, "write to %s failed", path);
}

int dmf_graph_info(const dmf_graph *g, int32_t *n, int32_t *m) {
  if (!g) return fail(DMF_ERR_INVALID_ARG, "null graph");
  if (n) *n = g->n;
  if (m) *m = g->m;
  return ok();
}

int dmf_graph_arrays(const dmf_graph *g, const int32_t **index, const int32_t **adj,
                     const int32_t **w, const int32_t **par) {
  if (!g) return fail(DMF_ERR_INVALID_ARG, "null graph");
  if (index) *index = g->off.data();
  if (adj) *adj = g->adj.data();
  if (w) *w = g->w.data();
  if (par) *par = g->par.data();
  return ok();
}

int64_t dmf_graph_find_arc(const dmf_graph *g, int32_t src, int32_t dst) {
  if (!g) return -1;
  return find_arc(*g, src, dst);
}

int dmf_graph_set_caps(dmf_graph *g, int32_t k, const int32_t *src, const int32_t *dst,
                       const int32_t *w) {
  if (!g || k < 0 || (k > 0 && (!src || !dst || !w))) return fail(DMF_ERR_INVALID_ARG, "bad arguments");
  for (int32_t i = 0; i < k; i++) {
    if (src[i] == dst[i]) continue;
    int64_t e = find_arc(*g, src[i], dst[i]);
    if (e < 0) return fail(DMF_ERR_UNKNOWN_ARC, "update %d: arc %d->%d not in graph", i, src[i], dst[i]);
    if (w[i] < 0) return fail(DMF_ERR_INVALID_ARG, "update %d: negative capacity", i);
    if ((int64_t)w[i] + g->w[g->par[e]] > INT32_MAX) return fail(DMF_ERR_OVERFLOW, "update %d overflows", i);
    g->w[e] = w[i];
  }
  return ok();
}

void dmf_graph_free(dmf_graph *g) { delete g; }

int dmf_updates_load(const char *path, int32_t *k, int32_t **src, int32_t **dst, int32_t **w) {
  if (!path || !k || !src || !dst || !w) return fail(DMF_ERR_INVALID_ARG, "null argument");
  FILE *f = std::fopen(path, "rb");
  if (!f) return fail(DMF_ERR_BAD_FILE, "cannot open %s", path);
  std::fseek(f, 0, SEEK_END);
  long long size = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  int32_t kk = 0;
  if (std::fread(&kk, 4, 1, f) != 1 || kk < 0 || size != 4 + 12LL * kk) {
    std::fclose(f);
    return fail(DMF_ERR_BAD_FILE, "%s: size %lld does not match k=%d", path, size, kk);
  }
  size_t bytes = sizeof(int32_t) * ((size_t)kk + 1);
  int32_t *a = (int32_t *)std::malloc(bytes), *b = (int32_t *)std::malloc(bytes),
          *c = (int32_t *)std::malloc(bytes);
  bool okr = a && b && c && std::fread(a, 4, kk, f) == (size_t)kk && std::fread(b, 4, kk, f) == (size_t)kk &&
             std::fread(c, 4, kk, f) == (size_t)kk;
  std::fclose(f);
  if (!okr) {
    std::free(a); std::free(b); std::free(c);
    return fail(DMF_ERR_BAD_FILE, "%s: short read", path);
  }
  *k = kk;
  *src = a;
  *dst = b;
  *w = c;
  return ok();
}

int dmf_updates_save(const char *path, int32_t k, const int32_t *src, const int32_t *dst,
                     const int32_t *w) {
  if (!path || k < 0 || (k > 0 && (!src || !dst || !w))) return fail(DMF_ERR_INVALID_ARG, "bad arguments");
  FILE *f = std::fopen(path, "wb");
  if (!f) return fail(DMF_ERR_BAD_FILE, "cannot open %s for writing", path);
  bool okw = std::fwrite(&k, 4, 1, f) == 1 && put_words(f, src, (size_t)k) && put_words(f, dst, (size_t)k) &&
             put_words(f, w, (size_t)k);
  okw = (std::fclose(f) == 0) && okw;
  return okw ? ok() : fail(DMF_ERR_BAD_FILE, "write to %s failed", path);
}

// ---------------------------------------------------------------------------
// generators
// ---------------------------------------------------------------------------
int dmf_gen_grid(int32_t rows, int32_t cols, uint64_t seed, int32_t cap_lo, int32_t cap_hi,
                 int32_t st_cap, dmf_graph **out, int32_t *s, int32_t *t) {
  if (!out || rows < 1 || cols < 1 || (int64_t)rows * cols < 2 || (int64_t)rows * cols > INT32_MAX ||
      cap_lo < 0 || cap_hi < cap_lo || st_cap < 0)
    return fail(DMF_ERR_INVALID_ARG, "bad grid parameters");
  return guarded([&]() -> int {
    Rng rng(seed);
    std::vector<int32_t> U, V, W;
    int64_t nv = (int64_t)rows * cols;
    U.reserve(4 * nv + rows * 2);
    auto emit = [&](int32_t a, int32_t b, int32_t c) { U.push_back(a); V.push_back(b); W.push_back(c); };
    for (int32_t r = 0; r < rows; r++)
      for (int32_t c = 0; c < cols; c++) {
        int32_t x = r * cols + c;
        if (c + 1 < cols) {
          emit(x, x + 1, (int32_t)rng.uniform(cap_lo, cap_hi));
          emit(x + 1, x, (int32_t)rng.uniform(cap_lo, cap_hi));
        }
        if (r + 1 < rows) {
          emit(x, x + cols, (int32_t)rng.uniform(cap_lo, cap_hi));
          emit(x + cols, x, (int32_t)rng.uniform(cap_lo, cap_hi));
        }
      }
    int32_t src = 0, snk = (int32_t)(nv - 1);
    for (int32_t r = 1; r < rows; r++) emit(src, r * cols, st_cap);
    for (int32_t r = 0; r + 1 < rows; r++) emit(r * cols + cols - 1, snk, st_cap);
    int st = build_from_edges((int64_t)U.size(), U.data(), V.data(), W.data(), out);
    if (st) return st;
    if (s) *s = src;
    if (t) *t = snk;
    return ok();
  });
}

int dmf_gen_rmat(int32_t scale, int64_t narcs, double a, double b, double c, uint64_t seed,
                 int32_t cap_lo, int32_t cap_hi, int64_t reserve, dmf_graph **out, int32_t *s,
                 int32_t *t) {
  if (!out || scale < 1 || scale > 30 || narcs < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0 ||
      cap_lo < 0 || cap_hi < cap_lo || reserve < 0)
    return fail(DMF_ERR_INVALID_ARG, "bad R-MAT parameters");
  return guarded([&]() -> int {
    const double ab = a + b, abc = a + b + c;
    // arc i draws from its own counter-derived stream, so the output does not
    // depend on the thread count
    auto sample = [&](uint64_t idx, uint64_t salt) -> uint64_t {
      Rng r(seed ^ (salt * 0xD1B54A32D192ED03ull) ^ (idx * 0x9E3779B97F4A7C15ull));
      uint64_t uu = 0, vv = 0;
      for (int32_t l = 0; l < scale; l++) {
        double p = r.unit();
        uint64_t bu = p >= ab, bv = (p >= a && p < ab) || p >= abc;
        uu = (uu << 1) | bu;
        vv = (vv << 1) | bv;
      }
      return (uu << 32) | vv;
    };
    std::vector<uint64_t> keys((size_t)narcs);
  #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < narcs; i++) keys[i] = sample((uint64_t)i, 1);
#ifdef _OPENMP
    __gnu_parallel::sort(keys.begin(), keys.end());
#else
    std::sort(keys.begin(), keys.end());
#endif
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    keys.erase(std::remove_if(keys.begin(), keys.end(), [](uint64_t k) { return (k >> 32) == (k & 0xffffffffu); }),
               keys.end());
    const int32_t nv = 1 << scale;
    // source / sink on the sampled arcs
    std::vector<int64_t> outd(nv, 0), ind(nv, 0);
    const int64_t nk = (int64_t)keys.size();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nk; i++) {
      const uint64_t k = keys[i];
#pragma omp atomic
      outd[k >> 32]++;
#pragma omp atomic
      ind[k & 0xffffffffu]++;
    }
    int32_t src = 0, snk = -1;
    for (int32_t x = 0; x < nv; x++) if (outd[x] > outd[src]) src = x;
    for (int32_t x = 0; x < nv; x++)
      if (x != src && (snk < 0 || ind[x] > ind[snk])) snk = x;
    // reserved insert slots: further R-MAT samples, in sample order, that are
    // not arcs in either direction and not taken already in either direction.
    // The candidates of a window are drawn and checked against the arcs in
    // parallel; only the survivors go through the sequential taken-set check.
    std::vector<uint64_t> extra;
    if (reserve > 0) {
      std::unordered_set<uint64_t> taken;
      const uint64_t limit = (uint64_t)reserve * 64 + 1024;
      const uint64_t win = std::max<uint64_t>(1 << 16, 2 * (uint64_t)reserve);
      std::vector<uint64_t> cand;
      std::vector<uint8_t> okc;
      for (uint64_t base = 0; base < limit && (int64_t)extra.size() < reserve; base += win) {
        const uint64_t cnt = std::min(win, limit - base);
        cand.resize(cnt);
        okc.resize(cnt);
#pragma omp parallel for schedule(static)
        for (int64_t j = 0; j < (int64_t)cnt; j++) {
          const uint64_t k = sample(base + (uint64_t)j, 2);
          const uint64_t rk = (k << 32) | (k >> 32);
          cand[j] = k;
          okc[j] = (k >> 32) != (k & 0xffffffffu) && !std::binary_search(keys.begin(), keys.end(), k) &&
                   !std::binary_search(keys.begin(), keys.end(), rk);
        }
        for (uint64_t j = 0; j < cnt && (int64_t)extra.size() < reserve; j++) {
          if (!okc[j]) continue;
          const uint64_t k = cand[j], rk = (k << 32) | (k >> 32);
          if (taken.count(k) || taken.count(rk)) continue;
          taken.insert(k);
          extra.push_back(k);
        }
      }
    }
    const size_t na = keys.size(), ne = extra.size();
    std::vector<int32_t> U(na + ne), V(na + ne), W(na + ne);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)na; i++) {
      U[i] = (int32_t)(keys[i] >> 32);
      V[i] = (int32_t)(keys[i] & 0xffffffffu);
    }
    Rng caps(seed ^ 0xC0FFEEull);
    for (size_t i = 0; i < na; i++) W[i] = (int32_t)caps.uniform(cap_lo, cap_hi);
    for (size_t i = 0; i < ne; i++) {
      U[na + i] = (int32_t)(extra[i] >> 32);
      V[na + i] = (int32_t)(extra[i] & 0xffffffffu);
      W[na + i] = 0;
    }
    std::vector<uint64_t>().swap(keys);
    // keep all 2^scale vertices even if the highest ids are isolated
    dmf_graph *built = nullptr;
    int st = build_from_edges((int64_t)U.size(), U.data(), V.data(), W.data(), &built);
    if (st) return st;
    std::unique_ptr<dmf_graph> g(built);
    if (g->n < nv) {
      g->off.resize((size_t)nv + 1, g->m);
      g->n = nv;
    }
    *out = g.release();
    if (s) *s = src;
    if (t) *t = snk;
    return ok();
  });
}

int dmf_gen_batches(const dmf_graph *g, int32_t nb, double frac, double p_inc, double p_dec, double p_ins,
                    int32_t delta_hi, int32_t ins_lo, int32_t ins_hi, uint64_t seed, int64_t **ofs,
                    int32_t **src, int32_t **dst, int32_t **w) {
  if (!g || nb < 0 || !(frac > 0) || frac > 1 || p_inc < 0 || p_dec < 0 || p_ins < 0 ||
      p_inc + p_dec + p_ins > 1.0 + 1e-9 || delta_hi < 1 || ins_lo < 0 || ins_hi < ins_lo || !ofs || !src ||
      !dst || !w)
    return fail(DMF_ERR_INVALID_ARG, "bad batch parameters");
  return guarded([&]() -> int {
    const int32_t m = g->m;
    std::vector<int32_t> cap(g->w);
    std::vector<int32_t> tail(m);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t x = 0; x < g->n; x++)
      for (int32_t e = g->off[x]; e < g->off[x + 1]; e++) tail[e] = x;
    // Candidate lists, in arc order: `pos` = arcs with capacity > 0, `absent` =
    // arcs whose pair has capacity 0 both ways.  Built once, then updated after
    // each batch from the arcs it touched (and their partners), which is all
    // that can change membership.
    auto is_pos = [&](int32_t e) { return cap[e] > 0; };
    auto is_absent = [&](int32_t e) { return cap[e] == 0 && cap[g->par[e]] == 0; };
    std::vector<int32_t> pos, absent;
    {
      int nth = 1;
#ifdef _OPENMP
      nth = omp_get_max_threads();
#endif
      std::vector<int64_t> cp((size_t)nth + 1, 0), ca((size_t)nth + 1, 0);
#pragma omp parallel num_threads(nth)
      {
        int t = 0, tt = 1;
#ifdef _OPENMP
        t = omp_get_thread_num();
        tt = omp_get_num_threads();
#endif
        const int32_t b = (int32_t)((int64_t)m * t / tt), e = (int32_t)((int64_t)m * (t + 1) / tt);
        int64_t np = 0, na = 0;
        for (int32_t x = b; x < e; x++) {
          np += is_pos(x);
          na += is_absent(x);
        }
        cp[t + 1] = np;
        ca[t + 1] = na;
#pragma omp barrier
#pragma omp single
        {
          for (int q = 0; q < tt; q++) {
            cp[q + 1] += cp[q];
            ca[q + 1] += ca[q];
          }
          pos.resize(cp[tt]);
          absent.resize(ca[tt]);
        }
        int64_t ip = cp[t], ia = ca[t];
        for (int32_t x = b; x < e; x++) {
          if (is_pos(x)) pos[ip++] = x;
          if (is_absent(x)) absent[ia++] = x;
        }
      }
    }
    // list := (list without `drop`) merged with `add`; all three sorted, `drop`
    // a subset of `list`, `add` disjoint from it, list entries distinct.  The
    // list is cut into slices of equal length; a slice's first entry bounds its
    // value range, which selects its part of `drop` and `add` by binary search,
    // and each slice merges into its own part of the output: the result is the
    // sequential merge's, entry for entry.  `spare` is the list's previous
    // buffer, reused so that the output is not cleared on every batch.
    auto refresh = [](std::vector<int32_t> &list, std::vector<int32_t> &spare, const std::vector<int32_t> &drop,
                      const std::vector<int32_t> &add) {
      if (drop.empty() && add.empty()) return;
      const int64_t L = (int64_t)list.size();
      spare.resize((size_t)(L - (int64_t)drop.size() + (int64_t)add.size()));
      int32_t *out = spare.data();
      int R = 1;
#ifdef _OPENMP
      R = (int)std::max<int64_t>(1, std::min<int64_t>(4 * omp_get_max_threads(), L / 65536));
#endif
      std::vector<int64_t> ib((size_t)R + 1), db((size_t)R + 1), ab((size_t)R + 1);
      for (int r = 0; r <= R; r++) ib[r] = L * r / R;
      db[0] = ab[0] = 0;
      db[R] = (int64_t)drop.size();
      ab[R] = (int64_t)add.size();
      for (int r = 1; r < R; r++) {
        const int32_t v = list[ib[r]];
        db[r] = std::lower_bound(drop.begin(), drop.end(), v) - drop.begin();
        ab[r] = std::lower_bound(add.begin(), add.end(), v) - add.begin();
      }
#pragma omp parallel for schedule(static)
      for (int r = 0; r < R; r++) {
        int64_t o = ib[r] - db[r] + ab[r], i = ib[r], d = db[r], a = ab[r];
        const int64_t ie = ib[r + 1], de = db[r + 1], ae = ab[r + 1];
        while (i < ie) {
          const int32_t x = list[i];
          if (d < de && drop[d] == x) {
            d++;
            i++;
            continue;
          }
          if (a < ae && add[a] < x) {
            out[o++] = add[a++];
            continue;
          }
          out[o++] = x;
          i++;
        }
        while (a < ae) out[o++] = add[a++];
      }
      list.swap(spare);
    };
    std::vector<int32_t> pos_spare, absent_spare;
    Rng rng(seed);
    std::vector<int64_t> O(1, 0);
    std::vector<int32_t> S, D, Wn;
    std::vector<uint8_t> chosen(m, 0);
    for (int32_t bi = 0; bi < nb; bi++) {
      int64_t K = std::max<int64_t>(1, (int64_t)std::llround(frac * (double)pos.size()));
      int64_t n_ins = absent.empty() ? 0 : std::min<int64_t>((int64_t)absent.size(), std::llround(p_ins * K));
      int64_t n_inc = std::llround(p_inc * K), n_dec = std::llround(p_dec * K);
      int64_t n_del = std::max<int64_t>(0, K - n_inc - n_dec - n_ins);
      int64_t need = std::min<int64_t>((int64_t)pos.size(), n_inc + n_dec + n_del);
      std::vector<int32_t> picks;
      while ((int64_t)picks.size() < need) {
        int32_t e = pos[rng.uniform(0, (int64_t)pos.size() - 1)];
        if (chosen[e]) continue;
        chosen[e] = 1;
        picks.push_back(e);
      }
      std::vector<int32_t> ins;
      while ((int64_t)ins.size() < n_ins) {
        int32_t e = absent[rng.uniform(0, (int64_t)absent.size() - 1)];
        if (chosen[e]) continue;
        chosen[e] = 1;
        ins.push_back(e);
      }
      // arcs whose membership may change: the touched ones and their partners
      std::vector<int32_t> touched;
      touched.reserve(2 * (picks.size() + ins.size()));
      for (int32_t e : picks) { touched.push_back(e); touched.push_back(g->par[e]); }
      for (int32_t e : ins) { touched.push_back(e); touched.push_back(g->par[e]); }
#ifdef _OPENMP
      __gnu_parallel::sort(touched.begin(), touched.end());
#else
      std::sort(touched.begin(), touched.end());
#endif
      touched.erase(std::unique(touched.begin(), touched.end()), touched.end());
      std::vector<uint8_t> was((size_t)touched.size());
#pragma omp parallel for schedule(static)
      for (int64_t j = 0; j < (int64_t)touched.size(); j++)
        was[j] = (uint8_t)(is_pos(touched[j]) | (is_absent(touched[j]) << 1));
      int64_t i = 0;
      for (int32_t e : picks) {
        int32_t nc;
        if (i < n_inc) nc = (int32_t)std::min<int64_t>((int64_t)cap[e] + rng.uniform(1, delta_hi),
                                                      (int64_t)INT32_MAX - cap[g->par[e]]);
        else if (i < n_inc + n_dec) nc = (int32_t)std::max<int64_t>(0, (int64_t)cap[e] - rng.uniform(1, delta_hi));
        else nc = 0;
        i++;
        S.push_back(tail[e]); D.push_back(g->adj[e]); Wn.push_back(nc);
        cap[e] = nc;
        chosen[e] = 0;
      }
      for (int32_t e : ins) {
        int32_t nc = (int32_t)rng.uniform(ins_lo, ins_hi);
        S.push_back(tail[e]); D.push_back(g->adj[e]); Wn.push_back(nc);
        cap[e] = nc;
        chosen[e] = 0;
      }
      O.push_back((int64_t)S.size());
      std::vector<int32_t> pdrop, padd, adrop, aadd;
#pragma omp parallel for schedule(static)
      for (int64_t j = 0; j < (int64_t)touched.size(); j++)
        was[j] |= (uint8_t)((is_pos(touched[j]) << 2) | (is_absent(touched[j]) << 3));
      for (size_t j = 0; j < touched.size(); j++) {
        const int32_t e = touched[j];
        const bool p0 = was[j] & 1, a0 = (was[j] >> 1) & 1, p1 = (was[j] >> 2) & 1, a1 = (was[j] >> 3) & 1;
        if (p0 && !p1) pdrop.push_back(e);
        if (!p0 && p1) padd.push_back(e);
        if (a0 && !a1) adrop.push_back(e);
        if (!a0 && a1) aadd.push_back(e);
      }
      if (bi + 1 < nb) {
        refresh(pos, pos_spare, pdrop, padd);
        refresh(absent, absent_spare, adrop, aadd);
      }
    }
    size_t kk = S.size();
    auto *o_ofs = (int64_t *)std::malloc(sizeof(int64_t) * O.size());
    auto *o_src = (int32_t *)std::malloc(sizeof(int32_t) * (kk + 1));
    auto *o_dst = (int32_t *)std::malloc(sizeof(int32_t) * (kk + 1));
    auto *o_w = (int32_t *)std::malloc(sizeof(int32_t) * (kk + 1));
    if (!o_ofs || !o_src || !o_dst || !o_w) {
      std::free(o_ofs); std::free(o_src); std::free(o_dst); std::free(o_w);
      return fail(DMF_ERR_OOM, "host allocation failed");
    }
    std::memcpy(o_ofs, O.data(), sizeof(int64_t) * O.size());
    if (kk) {
      std::memcpy(o_src, S.data(), 4 * kk);
      std::memcpy(o_dst, D.data(), 4 * kk);
      std::memcpy(o_w, Wn.data(), 4 * kk);
    }
    *ofs = o_ofs;
    *src = o_src;
    *dst = o_dst;
    *w = o_w;
    return ok();
  });
}

}  // extern "C"
