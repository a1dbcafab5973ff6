/*
 * oracle.c -- CPU oracle for the dynamic max-flow hot path (see oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, by __graft_entry__.smoke() as the
 * checker and by bench.py's CPU-baseline leg.  The product library never links it.
 *
 * Every function restating the reference cites the file:line of
 * ShruthiKannappan/dyn_maxflow it follows.  Widening: excess is int64 here
 * (int32 in the reference); residuals and capacities stay int32 as there.
 */
#include "oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define LD(p) __atomic_load_n((p), __ATOMIC_RELAXED)
#define ST(p, v) __atomic_store_n((p), (v), __ATOMIC_RELAXED)
#define FADD(p, v) __atomic_fetch_add((p), (v), __ATOMIC_RELAXED)

void orc_free(void *p) { free(p); }

/* ======================================================================= */
/* formats                                                                  */
/* ======================================================================= */

static int read_all(FILE *f, void *dst, size_t bytes) {
  return fread(dst, 1, bytes, f) == bytes ? 0 : -1;
}

/* code/graph.hpp:202-223 */
int orc_graph_read(const char *path, int32_t *n, int32_t *m, int32_t **off,
                   int32_t **adj, int32_t **w, int32_t **par) {
  FILE *f = fopen(path, "rb");
  if (!f) return -1;
  int32_t hdr[2];
  if (read_all(f, hdr, sizeof hdr) || hdr[0] < 0 || hdr[1] < 0) {
    fclose(f);
    return -1;
  }
  *n = hdr[0];
  *m = hdr[1];
  *off = (int32_t *)malloc(sizeof(int32_t) * ((size_t)hdr[0] + 1));
  *adj = (int32_t *)malloc(sizeof(int32_t) * ((size_t)hdr[1] + 1));
  *w = (int32_t *)malloc(sizeof(int32_t) * ((size_t)hdr[1] + 1));
  *par = (int32_t *)malloc(sizeof(int32_t) * ((size_t)hdr[1] + 1));
  int rc = read_all(f, *off, sizeof(int32_t) * ((size_t)hdr[0] + 1)) ||
           read_all(f, *adj, sizeof(int32_t) * (size_t)hdr[1]) ||
           read_all(f, *w, sizeof(int32_t) * (size_t)hdr[1]) ||
           read_all(f, *par, sizeof(int32_t) * (size_t)hdr[1]);
  fclose(f);
  if (rc) {
    free(*off); free(*adj); free(*w); free(*par);
    return -1;
  }
  return 0;
}

/* code/update.hpp:52-88 */
int orc_updates_read(const char *path, int32_t *k, int32_t **src, int32_t **dst,
                     int32_t **w) {
  FILE *f = fopen(path, "rb");
  if (!f) return -1;
  int32_t kk;
  if (read_all(f, &kk, sizeof kk) || kk < 0) {
    fclose(f);
    return -1;
  }
  *k = kk;
  *src = (int32_t *)malloc(sizeof(int32_t) * ((size_t)kk + 1));
  *dst = (int32_t *)malloc(sizeof(int32_t) * ((size_t)kk + 1));
  *w = (int32_t *)malloc(sizeof(int32_t) * ((size_t)kk + 1));
  int rc = read_all(f, *src, sizeof(int32_t) * (size_t)kk) ||
           read_all(f, *dst, sizeof(int32_t) * (size_t)kk) ||
           read_all(f, *w, sizeof(int32_t) * (size_t)kk);
  fclose(f);
  if (rc) {
    free(*src); free(*dst); free(*w);
    return -1;
  }
  return 0;
}

/* input_create/create_bin.cpp:67-124 (readEdgeList) and :18-64 (writeCSR).
 * Kept quadratic in the degree, exactly as written there. */
typedef struct { int32_t to, weight, pidx; } orc_arc;
typedef struct { orc_arc *a; int32_t len, cap; } orc_vec;

static int32_t vec_push(orc_vec *v, int32_t to, int32_t weight) {
  if (v->len == v->cap) {
    v->cap = v->cap ? 2 * v->cap : 4;
    v->a = (orc_arc *)realloc(v->a, sizeof(orc_arc) * (size_t)v->cap);
  }
  v->a[v->len].to = to;
  v->a[v->len].weight = weight;
  v->a[v->len].pidx = -1;
  return v->len++;
}

int orc_build_csr(int64_t k, const int32_t *u, const int32_t *v, const int32_t *w,
                  int32_t *n_out, int32_t *m_out, int32_t **off, int32_t **adj,
                  int32_t **cap, int32_t **par) {
  int32_t maxnode = -1;
  for (int64_t i = 0; i < k; i++) {
    if (u[i] == v[i]) continue; /* create_bin.cpp:85 */
    if (u[i] < 0 || v[i] < 0) return -1;
    if (u[i] > maxnode) maxnode = u[i];
    if (v[i] > maxnode) maxnode = v[i];
  }
  int32_t n = maxnode + 1;
  orc_vec *g = (orc_vec *)calloc((size_t)(n > 0 ? n : 1), sizeof(orc_vec));
  for (int64_t i = 0; i < k; i++) {
    int32_t a = u[i], b = v[i];
    if (a == b) continue;
    int32_t fi = -1;
    for (int32_t j = 0; j < g[a].len; j++)
      if (g[a].a[j].to == b) { fi = j; break; }
    if (fi == -1) fi = vec_push(&g[a], b, w[i]); /* :106 */
    else g[a].a[fi].weight += w[i];              /* :107 duplicates summed */
    int32_t ri = -1;
    for (int32_t j = 0; j < g[b].len; j++)
      if (g[b].a[j].to == a) { ri = j; break; }
    if (ri == -1) ri = vec_push(&g[b], a, 0); /* :116 partner with capacity 0 */
    g[a].a[fi].pidx = ri;
    g[b].a[ri].pidx = fi;
  }
  int64_t m = 0;
  for (int32_t x = 0; x < n; x++) m += g[x].len;
  if (m > INT32_MAX) return -1;
  *off = (int32_t *)malloc(sizeof(int32_t) * ((size_t)n + 1));
  *adj = (int32_t *)malloc(sizeof(int32_t) * ((size_t)m + 1));
  *cap = (int32_t *)malloc(sizeof(int32_t) * ((size_t)m + 1));
  *par = (int32_t *)malloc(sizeof(int32_t) * ((size_t)m + 1));
  int32_t pos = 0;
  for (int32_t x = 0; x < n; x++) { /* writeCSR :31-40 */
    (*off)[x] = pos;
    for (int32_t j = 0; j < g[x].len; j++) {
      (*adj)[pos] = g[x].a[j].to;
      (*cap)[pos] = g[x].a[j].weight;
      pos++;
    }
  }
  (*off)[n] = pos;
  pos = 0;
  for (int32_t x = 0; x < n; x++) /* :41-45 */
    for (int32_t j = 0; j < g[x].len; j++)
      (*par)[pos++] = g[x].a[j].pidx + (*off)[g[x].a[j].to];
  for (int32_t x = 0; x < n; x++) free(g[x].a);
  free(g);
  *n_out = n;
  *m_out = (int32_t)m;
  return 0;
}

/* ======================================================================= */
/* Dinic (independent exact solver)                                         */
/* ======================================================================= */

int64_t orc_dinic(int32_t n, int32_t m, const int32_t *off, const int32_t *adj,
                  const int32_t *cap, const int32_t *par, int32_t s, int32_t t,
                  int32_t *flow_out) {
  if (s == t || s < 0 || t < 0 || s >= n || t >= n) return -1;
  int32_t *r = (int32_t *)malloc(sizeof(int32_t) * ((size_t)m + 1));
  int32_t *lvl = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  int32_t *it = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  int32_t *q = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  int32_t *stk_v = (int32_t *)malloc(sizeof(int32_t) * ((size_t)n + 1));
  int32_t *stk_e = (int32_t *)malloc(sizeof(int32_t) * ((size_t)n + 1));
  memcpy(r, cap, sizeof(int32_t) * (size_t)m);
  int64_t total = 0;
  for (;;) {
    for (int32_t i = 0; i < n; i++) lvl[i] = -1;
    int32_t qh = 0, qt = 0;
    lvl[s] = 0;
    q[qt++] = s;
    while (qh < qt) {
      int32_t x = q[qh++];
      for (int32_t e = off[x]; e < off[x + 1]; e++)
        if (r[e] > 0 && lvl[adj[e]] < 0) {
          lvl[adj[e]] = lvl[x] + 1;
          q[qt++] = adj[e];
        }
    }
    if (lvl[t] < 0) break;
    for (int32_t i = 0; i < n; i++) it[i] = off[i];
    /* iterative blocking-flow DFS */
    for (;;) {
      int32_t depth = 0;
      stk_v[0] = s;
      int found = 0;
      while (depth >= 0) {
        int32_t x = stk_v[depth];
        if (x == t) { found = 1; break; }
        int advanced = 0;
        for (; it[x] < off[x + 1]; it[x]++) {
          int32_t e = it[x], y = adj[e];
          if (r[e] > 0 && lvl[y] == lvl[x] + 1) {
            stk_e[depth] = e;
            stk_v[++depth] = y;
            advanced = 1;
            break;
          }
        }
        if (!advanced) {
          lvl[x] = -1; /* dead end */
          depth--;
          if (depth >= 0) it[stk_v[depth]]++;
        }
      }
      if (!found) break;
      int32_t bott = INT32_MAX;
      for (int32_t d = 0; d < depth; d++)
        if (r[stk_e[d]] < bott) bott = r[stk_e[d]];
      for (int32_t d = 0; d < depth; d++) {
        r[stk_e[d]] -= bott;
        r[par[stk_e[d]]] += bott;
      }
      total += bott;
    }
  }
  if (flow_out)
    for (int32_t e = 0; e < m; e++) flow_out[e] = cap[e] - r[e];
  free(r); free(lvl); free(it); free(q); free(stk_v); free(stk_e);
  return total;
}

/* ======================================================================= */
/* certificate                                                              */
/* ======================================================================= */

int orc_certify(int32_t n, int32_t m, const int32_t *off, const int32_t *adj,
                const int32_t *cap, const int32_t *par, const int32_t *res,
                int32_t s, int32_t t, int64_t *value, int64_t *cut_capacity) {
  if (n <= 0 || s == t || s < 0 || t < 0 || s >= n || t >= n) return 10;
  for (int32_t e = 0; e < m; e++) {
    int32_t p = par[e];
    if (p < 0 || p >= m || par[p] != e) return 11;
    if (res[e] < 0) return 1;
    if ((int64_t)res[e] + res[p] != (int64_t)cap[e] + cap[p]) return 2;
  }
  int64_t *ex = (int64_t *)calloc((size_t)n, sizeof(int64_t));
  int32_t *tail = (int32_t *)malloc(sizeof(int32_t) * ((size_t)m + 1));
  for (int32_t v = 0; v < n; v++)
    for (int32_t e = off[v]; e < off[v + 1]; e++) {
      ex[v] += (int64_t)res[e] - cap[e];
      tail[e] = v;
    }
  int64_t val = ex[t];
  for (int32_t v = 0; v < n; v++)
    if (v != s && ex[v] < 0) val += ex[v];
  /* S': vertices with a residual path to t or to a deficit vertex. A residual
   * arc w->x is arc par[e] for e = x->w, residual res[par[e]]. */
  uint8_t *in = (uint8_t *)calloc((size_t)n, 1);
  int32_t *q = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  int32_t qh = 0, qt = 0;
  for (int32_t v = 0; v < n; v++)
    if (v == t || (v != s && ex[v] < 0)) { in[v] = 1; q[qt++] = v; }
  while (qh < qt) {
    int32_t x = q[qh++];
    for (int32_t e = off[x]; e < off[x + 1]; e++) {
      int32_t w = adj[e];
      if (!in[w] && res[par[e]] > 0) { in[w] = 1; q[qt++] = w; }
    }
  }
  int rc = 0;
  if (in[s]) rc = 3; /* an augmenting path from s exists */
  for (int32_t v = 0; v < n && !rc; v++)
    if (v != s && v != t && ex[v] > 0 && in[v]) rc = 4; /* active vertex left */
  int64_t cutc = 0;
  for (int32_t e = 0; e < m && !rc; e++) {
    int32_t a = tail[e], b = adj[e];
    if (!in[a] && in[b]) {
      if (res[e] != 0) rc = 5;
      cutc += cap[e];
    }
  }
  if (!rc && cutc != val) rc = 6;
  if (value) *value = val;
  if (cut_capacity) *cut_capacity = cutc;
  free(ex); free(tail); free(in); free(q);
  return rc;
}

/* ======================================================================= */
/* restatement of the reference GPU algorithms                              */
/* ======================================================================= */

typedef struct {
  int32_t n, m, s, t, kc, nth;
  const int32_t *off, *adj, *par;
  int32_t *w, *res, *rev, *height, *level, *set, *set2, *part;
  int64_t *excess;
  int32_t set_ptr, set2_ptr, part_ptr;
  uint8_t *partB, *partfinal;
  int64_t max_iters;
} st_t;

#define PFOR _Pragma("omp parallel for schedule(dynamic, 64) num_threads(S->nth)")

/* staticMaxFlow_kernel_1 / init_kernel: code/dyn_data.h:25-35, dyn_pp.h:25-35 */
static void k_init(st_t *S) {
  PFOR
  for (int32_t v = 0; v < S->n; v++) {
    for (int32_t e = S->off[v]; e < S->off[v + 1]; e++) {
      S->res[e] = S->w[e];
      S->rev[e] = S->w[S->par[e]];
    }
    S->excess[v] = 0;
  }
}

/* staticMaxFlow_kernel_7 (<<<1,1>>>): code/dyn_data.h:39-56; with drain_sink the
 * push-pull version code/dyn_pp.h:39-72 that also drains the sink's in-arcs. */
static void k_saturate(st_t *S, int drain_sink) {
  int32_t v = S->s;
  for (int32_t e = S->off[v]; e < S->off[v + 1]; e++) {
    int32_t vv = S->adj[e], d = S->res[e];
    if (d > 0) {
      S->excess[vv] += d;
      S->excess[v] -= d;
      S->res[e] -= d;
      S->rev[e] += d;
      int32_t p = S->par[e];
      S->res[p] += d;
      S->rev[p] -= d;
    }
  }
  if (!drain_sink) return;
  v = S->t;
  for (int32_t e = S->off[v]; e < S->off[v + 1]; e++) {
    int32_t vv = S->adj[e], d = S->rev[e];
    if (d > 0) {
      S->excess[v] += d;
      S->excess[vv] -= d;
      S->res[e] += d;
      S->rev[e] -= d;
      int32_t p = S->par[e];
      S->res[p] -= d;
      S->rev[p] += d;
    }
  }
}

/* my_init_1: code/dyn_data.h:60-67 (also dyn_pp.h:551-558);
 * staticMaxFlow_kernel_10: code/dyn_topo.h:60-71 (same seeds). */
static void k_bfs_init(st_t *S) {
  PFOR
  for (int32_t v = 0; v < S->n; v++) {
    S->height[v] = S->n;
    S->level[v] = -1;
    if (v == S->t) S->level[v] = 0;
    if (v != S->s && S->excess[v] < 0) S->level[v] = 0;
  }
}

/* staticMaxFlow_kernel_11: code/dyn_data.h:72-87 (dyn_topo.h:74-89, dyn_pp.h:560-575) */
static int k_bfs_level(st_t *S, int32_t hops) {
  int flag = 0;
  PFOR
  for (int32_t v = 0; v < S->n; v++) {
    if (LD(&S->level[v]) == hops) {
      S->height[v] = hops;
      for (int32_t e = S->off[v]; e < S->off[v + 1]; e++) {
        int32_t w = S->adj[e];
        if (S->rev[e] > 0 && LD(&S->level[w]) == -1) {
          ST(&S->level[w], hops + 1);
          ST(&flag, 1);
        }
      }
    }
  }
  return flag;
}

static int64_t g_bfs_levels; /* statistics for the CPU baseline */

static void bfs_loop(st_t *S) {
  int32_t hops = 0;
  int f;
  do {
    f = k_bfs_level(S, hops);
    hops++;
    g_bfs_levels++;
  } while (f);
}

/* create_wl: code/dyn_data.h:217-238 (ballot compaction; here increasing v). */
static void k_create_wl(st_t *S) {
  int32_t c = 0;
  for (int32_t v = 0; v < S->n; v++)
    if (S->excess[v] > 0 && S->height[v] < S->n && v != S->s && v != S->t)
      S->set[c++] = v;
  S->set_ptr = c;
}

/* one push/relabel cycle body of staticMaxFlow_kernel_14 / push_kernel,
 * code/dyn_data.h:95-127.  Restrict: 0 none, 1 only partB neighbours
 * (pp_push_kernel dyn_pp.h:204).  Returns 0 when the vertex is not active. */
static int pr_cycle(st_t *S, int32_t v, int restrict_b) {
  int64_t ex1 = LD(&S->excess[v]);
  if (!(ex1 > 0 && LD(&S->height[v]) < S->n)) return 0;
  int32_t hh = INT_MAX, v0 = -1, fe = -1;
  for (int32_t e = S->off[v]; e < S->off[v + 1]; e++) {
    int32_t vv = S->adj[e];
    if (restrict_b && !S->partB[vv]) continue;
    int32_t h1 = LD(&S->height[vv]);
    if (h1 < hh && LD(&S->res[e]) > 0) { v0 = vv; hh = h1; fe = e; }
  }
  if (LD(&S->height[v]) > hh && v0 != -1) {
    int32_t fec = LD(&S->res[fe]);
    int32_t p = S->par[fe];
    int64_t d = ex1 < fec ? ex1 : fec;
    FADD(&S->excess[v], -d);
    FADD(&S->excess[v0], d);
    FADD(&S->res[fe], -(int32_t)d);
    FADD(&S->rev[fe], (int32_t)d);
    FADD(&S->res[p], (int32_t)d);
    FADD(&S->rev[p], -(int32_t)d);
  } else if (v0 != -1) {
    ST(&S->height[v], hh + 1);
  }
  return 1;
}

/* staticMaxFlow_kernel_14 (data) / push_kernel: code/dyn_data.h:89-131, dyn_pp.h:145-185 */
static void k_push_wl(st_t *S, const int32_t *set, int32_t cnt, int restrict_b) {
  PFOR
  for (int32_t i = 0; i < cnt; i++) {
    int32_t v = set[i];
    int32_t cycle = S->kc;
    while (cycle--)
      if (!pr_cycle(S, v, restrict_b)) break;
  }
}

/* staticMaxFlow_kernel_14 (topo): code/dyn_topo.h:90-136 */
static int k_push_topo(st_t *S) {
  int flag = 0;
  PFOR
  for (int32_t v = 0; v < S->n; v++) {
    if (LD(&S->excess[v]) > 0 && v != S->s && v != S->t &&
        LD(&S->height[v]) < S->n) {
      ST(&flag, 1);
      int32_t cycle = S->kc;
      do {
        if (!pr_cycle(S, v, 0)) break;
        cycle = cycle - 1;
      } while (cycle > 0);
    }
  }
  return flag;
}

/* body of staticMaxFlow_kernel_17 / remove_push (code/dyn_data.h:132-153,
 * dyn_pp.h:307-328); filter 1 = partB neighbours (pp_remove_push dyn_pp.h:365),
 * 2 = partfinal neighbours (remove_push_final dyn_pp.h:289). */
static void remove_body(st_t *S, int32_t v, int filter) {
  int32_t h = LD(&S->height[v]);
  for (int32_t e = S->off[v]; e < S->off[v + 1]; e++) {
    int32_t vv = S->adj[e];
    if (filter == 1 && !S->partB[vv]) continue;
    if (filter == 2 && !S->partfinal[vv]) continue;
    if (LD(&S->rev[e]) > 0 && LD(&S->height[vv]) > h + 1) {
      int32_t d = LD(&S->rev[e]);
      ST(&S->rev[e], LD(&S->rev[e]) - d);
      ST(&S->res[e], LD(&S->res[e]) + d);
      int32_t p = S->par[e];
      ST(&S->rev[p], LD(&S->rev[p]) + d);
      ST(&S->res[p], LD(&S->res[p]) - d);
      FADD(&S->excess[vv], -(int64_t)d);
      FADD(&S->excess[v], (int64_t)d);
    }
  }
}

static void k_remove_wl(st_t *S, const int32_t *set, int32_t cnt, int filter) {
  PFOR
  for (int32_t i = 0; i < cnt; i++) remove_body(S, set[i], filter);
}

/* staticMaxFlow_kernel_17 (topo): code/dyn_topo.h:137-157 */
static void k_remove_all(st_t *S) {
  PFOR
  for (int32_t v = 0; v < S->n; v++) remove_body(S, v, 0);
}

/* incremental_kernel_20: code/dyn_data.h:157-172 */
static void k_inc20(st_t *S) {
  PFOR
  for (int32_t v = 0; v < S->n; v++)
    for (int32_t e = S->off[v]; e < S->off[v + 1]; e++) {
      if (S->res[e] < 0) { S->rev[e] += S->res[e]; S->res[e] = 0; }
      if (S->rev[e] < 0) { S->res[e] += S->rev[e]; S->rev[e] = 0; }
    }
}

/* incremental_kernel_22: code/dyn_data.h:173-183 */
static void k_inc22(st_t *S) {
  PFOR
  for (int32_t v = 0; v < S->n; v++) {
    int64_t e1 = 0;
    for (int32_t e = S->off[v]; e < S->off[v + 1]; e++)
      e1 += (int64_t)S->res[e] - S->w[e];
    S->excess[v] = e1;
  }
}

/* find the arc src->dst as OnAdd_kernel does (last match), code/dyn_data.h:196-201 */
static int32_t find_arc(const st_t *S, int32_t src, int32_t dst) {
  int32_t ue = -1;
  for (int32_t e = S->off[src]; e < S->off[src + 1]; e++)
    if (S->adj[e] == dst) ue = e;
  return ue;
}

/* OnAdd_kernel: code/dyn_data.h:186-206 (identical in dyn_topo.h, dyn_pp.h).
 * A missing arc is an out-of-bounds write in the reference; here it is an error. */
static int k_onadd(st_t *S, int32_t k, const int32_t *us, const int32_t *ud,
                   const int32_t *uw) {
  for (int32_t i = 0; i < k; i++) {
    if (us[i] == ud[i]) continue;
    int32_t ue = find_arc(S, us[i], ud[i]);
    if (ue < 0) return -1;
    int32_t nc = uw[i];
    S->res[ue] = S->res[ue] + nc - S->w[ue];
    int32_t p = S->par[ue];
    S->rev[p] = S->rev[p] + nc - S->w[ue];
    S->w[ue] = nc;
  }
  return 0;
}

/* update_kernel: code/dyn_data_bench.cu:300-322 (sets the capacity only) */
static int k_update_w(st_t *S, int32_t k, const int32_t *us, const int32_t *ud,
                      const int32_t *uw) {
  for (int32_t i = 0; i < k; i++) {
    if (us[i] == ud[i]) continue; /* loadUpdateFile drops these, update.hpp:82 */
    int32_t ue = find_arc(S, us[i], ud[i]);
    if (ue < 0) return -1;
    S->w[ue] = uw[i];
  }
  return 0;
}

/* recalculate_max_flow_kernel_39: code/dyn_data.h:208-215 */
static void k_flow39(st_t *S) {
  int64_t add = 0;
  for (int32_t v = 0; v < S->n; v++)
    if (S->excess[v] < 0 && v != S->s) add += S->excess[v];
  S->excess[S->t] += add;
}

/* the data-driven outer loop shared by staticMaxFlow and Incremental,
 * code/dyn_data_bench.cu:33-87 and :113-167 */
static int data_loop(st_t *S) {
  k_bfs_init(S);
  bfs_loop(S);
  k_create_wl(S);
  int64_t it = 0;
  while (S->set_ptr > 0) {
    if (++it > S->max_iters) return -1;
    k_push_wl(S, S->set, S->set_ptr, 0);
    k_remove_wl(S, S->set, S->set_ptr, 0);
    k_bfs_init(S);
    bfs_loop(S);
    k_create_wl(S);
  }
  return 0;
}

/* topology-driven loop, code/dyn_topo_bench.cu:41-61 and :94-117 */
static int topo_loop(st_t *S) {
  int64_t it = 0;
  int f;
  do {
    if (++it > S->max_iters) return -1;
    k_bfs_init(S); /* staticMaxFlow_kernel_10 */
    bfs_loop(S);
    f = k_push_topo(S);
    k_remove_all(S);
  } while (f);
  return 0;
}

/* ---- push-pull (code/dyn_pp.h, code/dyn_pp_bench.cu) -------------------- */

/* pp_bfs_init: code/dyn_pp.h:76-83 */
static void k_pp_bfs_init(st_t *S) {
  PFOR
  for (int32_t v = 0; v < S->n; v++) {
    S->level[v] = -1;
    S->height[v] = S->n;
    if (v == S->s || v == S->t) S->level[v] = 0;
    if ((S->partB[v] && S->excess[v] < 0) || (!S->partB[v] && S->excess[v] > 0))
      S->level[v] = 0;
  }
}

/* pp_bfs: code/dyn_pp.h:99-120 */
static int k_pp_bfs(st_t *S, int32_t hops) {
  int flag = 0;
  PFOR
  for (int32_t v = 0; v < S->n; v++) {
    int push = S->partB[v];
    if (LD(&S->level[v]) == hops) {
      S->height[v] = hops;
      for (int32_t e = S->off[v]; e < S->off[v + 1]; e++) {
        int32_t w = S->adj[e];
        if (w == S->s || w == S->t) continue;
        if (push && S->rev[e] > 0 && LD(&S->level[w]) == -1) {
          ST(&S->level[w], hops + 1);
          ST(&flag, 1);
        }
        if (!push && S->res[e] > 0 && LD(&S->level[w]) == -1) {
          ST(&S->level[w], hops + 1);
          ST(&flag, 1);
        }
      }
    }
  }
  return flag;
}

/* final_bfs_init / final_bfs: code/dyn_pp.h:86-93, :123-140 */
static void k_final_bfs_init(st_t *S, int32_t nodes) {
  PFOR
  for (int32_t i = 0; i < nodes; i++) {
    int32_t v = S->part[i];
    S->level[v] = -1;
    S->height[v] = S->n;
    if (S->excess[v] < 0) S->level[v] = 0;
  }
}
static int k_final_bfs(st_t *S, int32_t nodes, int32_t hops) {
  int flag = 0;
  PFOR
  for (int32_t i = 0; i < nodes; i++) {
    int32_t v = S->part[i];
    if (LD(&S->level[v]) == hops) {
      S->height[v] = hops;
      for (int32_t e = S->off[v]; e < S->off[v + 1]; e++) {
        int32_t w = S->adj[e];
        if (S->partB[w]) continue;
        if (S->rev[e] > 0 && LD(&S->level[w]) == -1) {
          ST(&S->level[w], hops + 1);
          ST(&flag, 1);
        }
      }
    }
  }
  return flag;
}

/* pull_kernel: code/dyn_pp.h:237-280 */
static void k_pull(st_t *S, const int32_t *set, int32_t cnt) {
  PFOR
  for (int32_t i = 0; i < cnt; i++) {
    int32_t v = set[i];
    int32_t cycle = S->kc;
    while (cycle--) {
      int64_t ex1 = -LD(&S->excess[v]);
      if (!(ex1 > 0)) break;
      int32_t hh = INT_MAX, v0 = -1, fe = -1;
      for (int32_t e = S->off[v]; e < S->off[v + 1]; e++) {
        int32_t vv = S->adj[e];
        if (S->partB[vv]) continue;
        int32_t h1 = LD(&S->height[vv]);
        if (h1 < hh && LD(&S->rev[e]) > 0) { v0 = vv; hh = h1; fe = e; }
      }
      if (LD(&S->height[v]) > hh && v0 != -1) {
        int32_t rec = LD(&S->rev[fe]);
        int32_t p = S->par[fe];
        int64_t d = ex1 < rec ? ex1 : rec;
        FADD(&S->excess[v0], -d);
        FADD(&S->excess[v], d);
        FADD(&S->rev[fe], -(int32_t)d);
        FADD(&S->res[fe], (int32_t)d);
        FADD(&S->rev[p], (int32_t)d);
        FADD(&S->res[p], -(int32_t)d);
      } else if (v0 != -1) {
        ST(&S->height[v], hh + 1);
      }
    }
  }
}

/* remove_pull: code/dyn_pp.h:381-403 */
static void k_remove_pull(st_t *S, const int32_t *set, int32_t cnt) {
  PFOR
  for (int32_t i = 0; i < cnt; i++) {
    int32_t v = set[i];
    int32_t h = LD(&S->height[v]);
    for (int32_t e = S->off[v]; e < S->off[v + 1]; e++) {
      int32_t vv = S->adj[e];
      if (S->partB[vv]) continue;
      if (LD(&S->res[e]) > 0 && LD(&S->height[vv]) > h + 1) {
        int32_t d = LD(&S->res[e]);
        ST(&S->rev[e], LD(&S->rev[e]) + d);
        ST(&S->res[e], LD(&S->res[e]) - d);
        int32_t p = S->par[e];
        ST(&S->rev[p], LD(&S->rev[p]) - d);
        ST(&S->res[p], LD(&S->res[p]) + d);
        FADD(&S->excess[v], -(int64_t)d);
        FADD(&S->excess[vv], (int64_t)d);
      }
    }
  }
}

/* incremental_kernel_20 (push-pull, fused with kernel_22 and cut saturation):
 * code/dyn_pp.h:405-436.  The cut saturation reads the mirror values of the
 * pre-launch state, as each GPU thread only touches its own arcs' entries. */
static void k_pp_inc20(st_t *S) {
  PFOR
  for (int32_t v = 0; v < S->n; v++) {
    int self = S->partB[v];
    int64_t e1 = 0;
    for (int32_t e = S->off[v]; e < S->off[v + 1]; e++) {
      int32_t nbr = S->adj[e];
      if (S->res[e] < 0) { S->rev[e] += S->res[e]; S->res[e] = 0; }
      if (S->rev[e] < 0) { S->res[e] += S->rev[e]; S->rev[e] = 0; }
      if (self != S->partB[nbr]) {
        if (self) { int32_t d = S->rev[e]; S->rev[e] -= d; S->res[e] += d; }
        else { int32_t d = S->res[e]; S->res[e] -= d; S->rev[e] += d; }
      }
      e1 += (int64_t)S->res[e] - S->w[e];
    }
    S->excess[v] = e1;
  }
}

/* find_cut: dyn_pp.h:440-449; find_final_cut: dyn_pp.h:452-460 */
static void k_find_cut(st_t *S) {
  for (int32_t v = 0; v < S->n; v++) S->partB[v] = S->level[v] != -1;
}
static void k_find_final_cut(st_t *S) {
  for (int32_t v = 0; v < S->n; v++)
    if (!S->partB[v] && S->level[v] != -1) S->partB[v] = 1;
}

/* create_pp_wl: code/dyn_pp.h:499-545 */
static void k_create_pp_wl(st_t *S) {
  int32_t c1 = 0, c2 = 0;
  for (int32_t v = 0; v < S->n; v++) {
    if (v == S->t || v == S->s) continue;
    if (S->partB[v]) {
      if (S->excess[v] > 0 && S->height[v] < S->n) S->set[c1++] = v;
    } else {
      if (S->excess[v] < 0 && S->height[v] < S->n) S->set2[c2++] = v;
    }
  }
  S->set_ptr = c1;
  S->set2_ptr = c2;
}

/* find_part: code/dyn_pp.h:330-356.  The reference never clears d_part_ptr and
 * relies on d_set2_ptr, which aliases it (dyn_pp_bench.cu:255), being 0. */
static void k_find_part(st_t *S) {
  int32_t c = S->part_ptr;
  for (int32_t v = 0; v < S->n; v++) {
    S->partfinal[v] = 0;
    if (S->level[v] == -1) {
      S->partB[v] = 0;
      S->partfinal[v] = 1;
      S->part[c++] = v;
    }
    S->level[v] = -1;
    S->height[v] = S->n;
  }
  S->part_ptr = c;
}

/* create_final_wl: code/dyn_pp.h:619-642 */
static void k_create_final_wl(st_t *S, int32_t nodes) {
  int32_t c = 0;
  for (int32_t i = 0; i < nodes; i++) {
    int32_t v = S->part[i];
    if (S->excess[v] > 0 && S->height[v] < S->n) S->set[c++] = v;
  }
  S->set_ptr = c;
}

/* part_pp: code/dyn_pp_bench.cu:6-88 (the two streams become one sequence of
 * the push-stream kernels followed by the pull-stream kernels) */
static int pp_part(st_t *S) {
  k_pp_bfs_init(S);
  int32_t hops = 0;
  while (k_pp_bfs(S, hops++)) g_bfs_levels++;
  k_create_pp_wl(S);
  int64_t it = 0;
  while (S->set_ptr + S->set2_ptr > 0) {
    if (++it > S->max_iters) return -1;
    if (S->set_ptr > 0) {
      k_push_wl(S, S->set, S->set_ptr, 1);
      k_remove_wl(S, S->set, S->set_ptr, 1);
    }
    if (S->set2_ptr > 0) {
      k_pull(S, S->set2, S->set2_ptr);
      k_remove_pull(S, S->set2, S->set2_ptr);
    }
    k_pp_bfs_init(S);
    hops = 0;
    while (k_pp_bfs(S, hops++)) g_bfs_levels++;
    k_create_pp_wl(S);
  }
  return 0;
}

/* part_final: code/dyn_pp_bench.cu:91-152 */
static int pp_final(st_t *S) {
  S->part_ptr = S->set2_ptr; /* aliasing, see k_find_part */
  k_find_part(S);
  int32_t nodes = S->part_ptr;
  if (nodes == 0) return 0;
  k_final_bfs_init(S, nodes);
  int32_t hops = 0;
  while (k_final_bfs(S, nodes, hops++)) g_bfs_levels++;
  k_create_final_wl(S, nodes);
  int64_t it = 0;
  while (S->set_ptr > 0) {
    if (++it > S->max_iters) return -1;
    k_push_wl(S, S->set, S->set_ptr, 0);
    k_remove_wl(S, S->set, S->set_ptr, 2);
    k_final_bfs_init(S, nodes);
    hops = 0;
    while (k_final_bfs(S, nodes, hops++)) g_bfs_levels++;
    k_create_final_wl(S, nodes);
  }
  k_find_final_cut(S);
  return 0;
}

/* staticMaxFlow for each variant.  data: code/dyn_data_bench.cu:8-97;
 * topo: code/dyn_topo_bench.cu:16-75; pp: code/dyn_pp_bench.cu:155-239. */
static int static_solve(st_t *S, int variant) {
  k_init(S);
  k_saturate(S, variant == ORC_PP);
  if (variant == ORC_TOPO) return topo_loop(S);
  int rc = data_loop(S);
  if (variant == ORC_PP) k_find_cut(S);
  return rc;
}

/* Incremental.  data: code/dyn_data_bench.cu:98-170; topo: dyn_topo_bench.cu:76-119;
 * pp: dyn_pp_bench.cu:242-258. */
static int incremental(st_t *S, int variant) {
  if (variant == ORC_PP) {
    k_pp_inc20(S);
    if (pp_part(S)) return -1;
    return pp_final(S);
  }
  k_inc20(S);
  k_inc22(S);
  k_saturate(S, 0);
  if (variant == ORC_TOPO) return topo_loop(S);
  return data_loop(S);
}

static void st_alloc(st_t *S, int32_t n, int32_t m, const int32_t *off,
                     const int32_t *adj, const int32_t *w0, const int32_t *par,
                     int32_t s, int32_t t, int32_t kc, int nth, int64_t max_iters) {
  memset(S, 0, sizeof *S);
  S->n = n; S->m = m; S->s = s; S->t = t; S->kc = kc;
  S->nth = nth > 0 ? nth : 1;
  S->max_iters = max_iters > 0 ? max_iters : 1000000;
  S->off = off; S->adj = adj; S->par = par;
  size_t M = (size_t)m + 1, N = (size_t)n + 1;
  S->w = (int32_t *)malloc(sizeof(int32_t) * M);
  memcpy(S->w, w0, sizeof(int32_t) * (size_t)m);
  S->res = (int32_t *)calloc(M, sizeof(int32_t));
  S->rev = (int32_t *)calloc(M, sizeof(int32_t));
  S->excess = (int64_t *)calloc(N, sizeof(int64_t));
  S->height = (int32_t *)calloc(N, sizeof(int32_t));
  S->level = (int32_t *)calloc(N, sizeof(int32_t));
  S->set = (int32_t *)calloc(N, sizeof(int32_t));
  S->set2 = (int32_t *)calloc(N, sizeof(int32_t));
  S->part = (int32_t *)calloc(N, sizeof(int32_t));
  S->partB = (uint8_t *)calloc(N, 1);
  S->partfinal = (uint8_t *)calloc(N, 1);
}

static void st_free(st_t *S) {
  free(S->w); free(S->res); free(S->rev); free(S->excess); free(S->height);
  free(S->level); free(S->set); free(S->set2); free(S->part); free(S->partB);
  free(S->partfinal);
}

static int args_ok(int32_t n, int32_t s, int32_t t) {
  return n > 0 && s >= 0 && t >= 0 && s < n && t < n && s != t;
}

int orc_ref_run(int variant, int32_t n, int32_t m, const int32_t *off,
                const int32_t *adj, const int32_t *w0, const int32_t *par,
                int32_t s, int32_t t, int32_t kc, int32_t k, const int32_t *us,
                const int32_t *ud, const int32_t *uw, int nthreads,
                int64_t max_iters, int64_t *static_flow_before, int64_t *dynflow,
                int64_t *statflow) {
  if (!args_ok(n, s, t)) return -2;
  st_t S;
  int rc = 0;
  /* recalculate_max_flow: code/dyn_data_bench.cu:171-298 */
  st_alloc(&S, n, m, off, adj, w0, par, s, t, kc, nthreads, max_iters);
  rc = static_solve(&S, variant);
  if (!rc && static_flow_before) {
    int64_t f = S.excess[t];
    if (variant == ORC_PP) /* pp static reads through kernel_39, dyn_pp_bench.cu:443 */
      for (int32_t v = 0; v < n; v++)
        if (S.excess[v] < 0 && v != s) f += S.excess[v];
    *static_flow_before = f;
  }
  if (!rc && k_onadd(&S, k, us, ud, uw)) rc = -3;
  if (!rc) rc = incremental(&S, variant);
  if (!rc) {
    k_flow39(&S);
    if (dynflow) *dynflow = S.excess[t];
  }
  st_free(&S);
  if (rc) return rc;
  /* static_recalculate: code/dyn_data_bench.cu:325-492 */
  st_alloc(&S, n, m, off, adj, w0, par, s, t, kc, nthreads, max_iters);
  if (k_update_w(&S, k, us, ud, uw)) rc = -3;
  if (!rc) rc = static_solve(&S, variant);
  if (!rc) {
    if (variant == ORC_PP) k_flow39(&S); /* dyn_pp_bench.cu:443-448 */
    if (statflow) *statflow = S.excess[t];
  }
  st_free(&S);
  return rc;
}

static double now_ms(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

int orc_ref_run_successive(int variant, int32_t n, int32_t m, const int32_t *off,
                           const int32_t *adj, const int32_t *w0,
                           const int32_t *par, int32_t s, int32_t t, int32_t kc,
                           int32_t nb, const int64_t *bofs, const int32_t *us,
                           const int32_t *ud, const int32_t *uw, int nthreads,
                           int64_t max_iters, int64_t *static_flow,
                           int64_t *flows, double *batch_ms, double budget_ms,
                           int32_t *done) {
  if (done) *done = 0;
  if (!args_ok(n, s, t)) return -2;
  st_t S;
  st_alloc(&S, n, m, off, adj, w0, par, s, t, kc, nthreads, max_iters);
  int rc = static_solve(&S, variant);
  if (!rc && static_flow) {
    int64_t f = S.excess[t];
    for (int32_t v = 0; v < n; v++)
      if (S.excess[v] < 0 && v != s) f += S.excess[v];
    *static_flow = f;
  }
  double spent = 0;
  for (int32_t b = 0; b < nb && !rc; b++) {
    if (budget_ms > 0 && spent > budget_ms) break;
    double t0 = now_ms();
    int64_t lo = bofs[b], hi = bofs[b + 1];
    if (k_onadd(&S, (int32_t)(hi - lo), us + lo, ud + lo, uw + lo)) { rc = -3; break; }
    rc = incremental(&S, variant);
    if (rc) break;
    /* kernel_39 folded without mutating the state, so the next batch starts
     * from the resident pseudoflow as the device-resident engine does. */
    int64_t f = S.excess[t];
    for (int32_t v = 0; v < n; v++)
      if (S.excess[v] < 0 && v != s) f += S.excess[v];
    if (flows) flows[b] = f;
    const double dt = now_ms() - t0;
    if (batch_ms) batch_ms[b] = dt;
    spent += dt;
    if (done) *done = b + 1;
  }
  st_free(&S);
  return rc;
}
