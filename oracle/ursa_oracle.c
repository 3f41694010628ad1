/*
 * ursa_oracle.c -- CPU restatement of ursa-core (cldixon/ursa) for the hot
 * path: CSR topology + degree, PageRank, BFS / shortest paths, k-hop, weak
 * connected components, triangle count, clustering, Brandes betweenness.
 *
 * TEST INFRASTRUCTURE ONLY (the parity checker and the timed CPU baseline).
 * The product library never links or calls this file.
 *
 * Pinning: the reference's Rust toolchain is absent here, so the restatement
 * is pinned against the golden values of the reference's own unit tests and
 * its NetworkX cross-check (tests/test_oracle_golden.py).
 *
 * Floating point: compiled with -ffp-contract=off so no a*b+c is fused (Rust
 * never contracts), giving the same IEEE-754 results as the Rust source.
 * Citations are ursa-core/src/<file>:<line>.
 */
#define _GNU_SOURCE
#include "ursa_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Thread helpers: contiguous-range parallel-for. Results never depend on the */
/* split because every parallel sweep writes disjoint outputs or fixed-size   */
/* chunk partials that are combined in order afterwards.                      */
/* ------------------------------------------------------------------------ */

static int g_threads = 1;

void orc_set_threads(int threads) { g_threads = threads < 1 ? 1 : threads; }
int orc_get_threads(void) { return g_threads; }

typedef void (*range_fn)(void *ctx, uint64_t lo, uint64_t hi, int tid);

typedef struct {
  range_fn fn;
  void *ctx;
  uint64_t lo, hi;
  int tid;
} range_job;

static void *range_tramp(void *p) {
  range_job *j = (range_job *)p;
  j->fn(j->ctx, j->lo, j->hi, j->tid);
  return NULL;
}

/* Split [0, n) into `parts` contiguous ranges and run them concurrently. */
static void par_ranges(uint64_t n, int parts, range_fn fn, void *ctx) {
  if (parts < 1) parts = 1;
  if ((uint64_t)parts > n) parts = n ? (int)n : 1;
  if (parts == 1) {
    fn(ctx, 0, n, 0);
    return;
  }
  pthread_t th[256];
  range_job jobs[256];
  if (parts > 256) parts = 256;
  uint64_t step = (n + parts - 1) / parts;
  for (int t = 0; t < parts; t++) {
    uint64_t lo = step * t, hi = lo + step;
    if (lo > n) lo = n;
    if (hi > n) hi = n;
    jobs[t] = (range_job){fn, ctx, lo, hi, t};
  }
  for (int t = 1; t < parts; t++) pthread_create(&th[t], NULL, range_tramp, &jobs[t]);
  range_tramp(&jobs[0]);
  for (int t = 1; t < parts; t++) pthread_join(th[t], NULL);
}

static int par_threads_for(uint64_t work) {
  /* Small inputs run serially: the split would cost more than it saves. */
  if (work < (1u << 14)) return 1;
  return g_threads;
}

/* ------------------------------------------------------------------------ */
/* Topology (topology.rs)                                                     */
/* ------------------------------------------------------------------------ */

typedef struct {
  uint64_t *offsets;  /* n + 1 */
  uint32_t *targets;  /* m */
  uint32_t *edge_ids; /* m */
} orc_adj;

struct orc_topo {
  uint64_t n, m;
  orc_adj out;
  orc_adj inc;
  int has_inc;
  uint64_t *u_offsets;
  uint32_t *u_targets;
  int has_und;
  pthread_mutex_t lock;
};

/* Adjacency::build_serial (topology.rs:79-107): degree histogram into
 * offsets[k+1], prefix sum, then scatter in original row order. */
static orc_adj adj_build_serial(uint64_t n, const uint32_t *keys,
                                const uint32_t *other, uint64_t m) {
  orc_adj a;
  a.offsets = (uint64_t *)calloc(n + 1, sizeof(uint64_t));
  a.targets = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
  a.edge_ids = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
  for (uint64_t r = 0; r < m; r++) a.offsets[(uint64_t)keys[r] + 1] += 1;
  for (uint64_t i = 0; i < n; i++) a.offsets[i + 1] += a.offsets[i];
  uint64_t *cursor = (uint64_t *)malloc((n ? n : 1) * sizeof(uint64_t));
  memcpy(cursor, a.offsets, n * sizeof(uint64_t));
  for (uint64_t r = 0; r < m; r++) {
    uint64_t pos = cursor[keys[r]]++;
    a.targets[pos] = other[r];
    a.edge_ids[pos] = (uint32_t)r;
  }
  free(cursor);
  return a;
}

/* Adjacency::build_parallel (topology.rs:115-187): per-chunk histograms, a
 * global prefix, per-chunk base cursors, and a disjoint parallel scatter.
 * Byte-identical to the serial build. */
typedef struct {
  uint64_t n, m, chunk;
  const uint32_t *keys, *other;
  uint32_t **hists;
  uint32_t *targets, *edge_ids;
} pbuild_ctx;

static void pbuild_hist(void *p, uint64_t lo, uint64_t hi, int tid) {
  pbuild_ctx *c = (pbuild_ctx *)p;
  (void)tid;
  for (uint64_t ch = lo; ch < hi; ch++) {
    uint32_t *h = (uint32_t *)calloc(c->n ? c->n : 1, sizeof(uint32_t));
    uint64_t s = ch * c->chunk, e = s + c->chunk;
    if (e > c->m) e = c->m;
    for (uint64_t r = s; r < e; r++) h[c->keys[r]] += 1;
    c->hists[ch] = h;
  }
}

static void pbuild_scatter(void *p, uint64_t lo, uint64_t hi, int tid) {
  pbuild_ctx *c = (pbuild_ctx *)p;
  (void)tid;
  for (uint64_t ch = lo; ch < hi; ch++) {
    uint32_t *base = c->hists[ch];
    uint64_t s = ch * c->chunk, e = s + c->chunk;
    if (e > c->m) e = c->m;
    for (uint64_t r = s; r < e; r++) {
      uint32_t k = c->keys[r];
      uint32_t pos = base[k]++;
      c->targets[pos] = c->other[r];
      c->edge_ids[pos] = (uint32_t)r;
    }
  }
}

static orc_adj adj_build_parallel(uint64_t n, const uint32_t *keys,
                                  const uint32_t *other, uint64_t m,
                                  int n_chunks) {
  orc_adj a;
  pbuild_ctx c;
  c.n = n;
  c.m = m;
  c.chunk = (m + n_chunks - 1) / n_chunks;
  c.keys = keys;
  c.other = other;
  uint64_t nch = (m + c.chunk - 1) / c.chunk;
  c.hists = (uint32_t **)calloc(nch, sizeof(uint32_t *));
  par_ranges(nch, (int)nch, pbuild_hist, &c);
  a.offsets = (uint64_t *)calloc(n + 1, sizeof(uint64_t));
  for (uint64_t ch = 0; ch < nch; ch++)
    for (uint64_t k = 0; k < n; k++) a.offsets[k + 1] += c.hists[ch][k];
  for (uint64_t i = 0; i < n; i++) a.offsets[i + 1] += a.offsets[i];
  uint32_t *running = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
  for (uint64_t k = 0; k < n; k++) running[k] = (uint32_t)a.offsets[k];
  for (uint64_t ch = 0; ch < nch; ch++) {
    uint32_t *h = c.hists[ch];
    for (uint64_t k = 0; k < n; k++) {
      uint32_t cnt = h[k];
      h[k] = running[k];
      running[k] += cnt;
    }
  }
  free(running);
  a.targets = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
  a.edge_ids = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
  c.targets = a.targets;
  c.edge_ids = a.edge_ids;
  par_ranges(nch, (int)nch, pbuild_scatter, &c);
  for (uint64_t ch = 0; ch < nch; ch++) free(c.hists[ch]);
  free(c.hists);
  return a;
}

/* Adjacency::build dispatch (topology.rs:54-75): parallel at >= 2^16 edges. */
static orc_adj adj_build(uint64_t n, const uint32_t *keys, const uint32_t *other,
                         uint64_t m) {
  const uint64_t PARALLEL_MIN_EDGES = 1u << 16;
  int n_chunks = g_threads;
  if (m < PARALLEL_MIN_EDGES || n_chunks <= 1 || n == 0)
    return adj_build_serial(n, keys, other, m);
  return adj_build_parallel(n, keys, other, m, n_chunks);
}

static void adj_free(orc_adj *a) {
  free(a->offsets);
  free(a->targets);
  free(a->edge_ids);
  memset(a, 0, sizeof(*a));
}

orc_topo *orc_topo_build(uint64_t n, const uint32_t *src, const uint32_t *dst,
                         uint64_t m) {
  if (m > 0xFFFFFFFFull) return NULL; /* topology.rs:61-65 */
  if (n > 0x100000000ull) return NULL;
  for (uint64_t r = 0; r < m; r++)
    if ((uint64_t)src[r] >= n || (uint64_t)dst[r] >= n) return NULL;
  orc_topo *t = (orc_topo *)calloc(1, sizeof(orc_topo));
  t->n = n;
  t->m = m;
  t->out = adj_build(n, src, dst, m);
  pthread_mutex_init(&t->lock, NULL);
  return t;
}

void orc_topo_free(orc_topo *t) {
  if (!t) return;
  adj_free(&t->out);
  if (t->has_inc) adj_free(&t->inc);
  free(t->u_offsets);
  free(t->u_targets);
  pthread_mutex_destroy(&t->lock);
  free(t);
}

uint64_t orc_topo_n_nodes(const orc_topo *t) { return t->n; }
uint64_t orc_topo_n_edges(const orc_topo *t) { return t->m; }

/* Topology::reconstruct_endpoints + incoming (topology.rs:307-321,343-348):
 * un-permute the out-CSR into row order (serial), then build by destination. */
static const orc_adj *topo_incoming(orc_topo *t) {
  pthread_mutex_lock(&t->lock);
  if (!t->has_inc) {
    uint64_t m = t->m;
    uint32_t *src_by_row = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
    uint32_t *dst_by_row = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
    for (uint64_t u = 0; u < t->n; u++) {
      for (uint64_t k = t->out.offsets[u]; k < t->out.offsets[u + 1]; k++) {
        uint32_t row = t->out.edge_ids[k];
        src_by_row[row] = (uint32_t)u;
        dst_by_row[row] = t->out.targets[k];
      }
    }
    t->inc = adj_build(t->n, dst_by_row, src_by_row, m);
    free(src_by_row);
    free(dst_by_row);
    t->has_inc = 1;
  }
  pthread_mutex_unlock(&t->lock);
  return &t->inc;
}

static const orc_adj *topo_adj(orc_topo *t, int dir) {
  return dir == 1 ? topo_incoming(t) : &t->out;
}

void orc_topo_csr(orc_topo *t, int dir, uint64_t *offsets, uint32_t *targets,
                  uint32_t *edge_ids) {
  const orc_adj *a = topo_adj(t, dir);
  if (offsets) memcpy(offsets, a->offsets, (t->n + 1) * sizeof(uint64_t));
  if (targets) memcpy(targets, a->targets, t->m * sizeof(uint32_t));
  if (edge_ids) memcpy(edge_ids, a->edge_ids, t->m * sizeof(uint32_t));
}

/* build_undirected (topology.rs:360-389): per node, out ∪ in neighbours with
 * self-loops filtered, sort_unstable + dedup, then flatten. */
typedef struct {
  orc_topo *t;
  uint32_t **lists;
  uint64_t *lens;
} und_ctx;

static int cmp_u32(const void *a, const void *b) {
  uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return (x > y) - (x < y);
}

static void und_node(void *p, uint64_t lo, uint64_t hi, int tid) {
  und_ctx *c = (und_ctx *)p;
  (void)tid;
  const orc_adj *o = &c->t->out, *in = &c->t->inc;
  for (uint64_t u = lo; u < hi; u++) {
    uint64_t d = (o->offsets[u + 1] - o->offsets[u]) + (in->offsets[u + 1] - in->offsets[u]);
    uint32_t *l = (uint32_t *)malloc((d ? d : 1) * sizeof(uint32_t));
    uint64_t len = 0;
    for (uint64_t k = o->offsets[u]; k < o->offsets[u + 1]; k++)
      if (o->targets[k] != u) l[len++] = o->targets[k];
    for (uint64_t k = in->offsets[u]; k < in->offsets[u + 1]; k++)
      if (in->targets[k] != u) l[len++] = in->targets[k];
    qsort(l, len, sizeof(uint32_t), cmp_u32);
    uint64_t w = 0;
    for (uint64_t i = 0; i < len; i++)
      if (w == 0 || l[w - 1] != l[i]) l[w++] = l[i];
    c->lists[u] = l;
    c->lens[u] = w;
  }
}

static void topo_undirected(orc_topo *t) {
  topo_incoming(t);
  pthread_mutex_lock(&t->lock);
  if (!t->has_und) {
    uint64_t n = t->n;
    und_ctx c = {t, (uint32_t **)calloc(n ? n : 1, sizeof(uint32_t *)),
                 (uint64_t *)calloc(n ? n : 1, sizeof(uint64_t))};
    par_ranges(n, par_threads_for(n + t->m), und_node, &c);
    t->u_offsets = (uint64_t *)calloc(n + 1, sizeof(uint64_t));
    for (uint64_t u = 0; u < n; u++) t->u_offsets[u + 1] = t->u_offsets[u] + c.lens[u];
    t->u_targets = (uint32_t *)malloc((t->u_offsets[n] ? t->u_offsets[n] : 1) * sizeof(uint32_t));
    for (uint64_t u = 0; u < n; u++) {
      memcpy(t->u_targets + t->u_offsets[u], c.lists[u], c.lens[u] * sizeof(uint32_t));
      free(c.lists[u]);
    }
    free(c.lists);
    free(c.lens);
    t->has_und = 1;
  }
  pthread_mutex_unlock(&t->lock);
}

uint64_t orc_topo_undirected_len(orc_topo *t) {
  topo_undirected(t);
  return t->u_offsets[t->n];
}

void orc_topo_undirected(orc_topo *t, uint64_t *offsets, uint32_t *targets) {
  topo_undirected(t);
  if (offsets) memcpy(offsets, t->u_offsets, (t->n + 1) * sizeof(uint64_t));
  if (targets) memcpy(targets, t->u_targets, t->u_offsets[t->n] * sizeof(uint32_t));
}

/* ------------------------------------------------------------------------ */
/* degree (algo/degree.rs:12-30)                                              */
/* ------------------------------------------------------------------------ */

void orc_degree(orc_topo *t, int dir, uint32_t *out) {
  uint64_t n = t->n;
  if (dir == 0) {
    for (uint64_t u = 0; u < n; u++) out[u] = (uint32_t)(t->out.offsets[u + 1] - t->out.offsets[u]);
  } else if (dir == 1) {
    const orc_adj *in = topo_incoming(t);
    for (uint64_t u = 0; u < n; u++) out[u] = (uint32_t)(in->offsets[u + 1] - in->offsets[u]);
  } else {
    const orc_adj *in = topo_incoming(t);
    for (uint64_t u = 0; u < n; u++)
      out[u] = (uint32_t)(t->out.offsets[u + 1] - t->out.offsets[u]) +
               (uint32_t)(in->offsets[u + 1] - in->offsets[u]);
  }
}

/* ------------------------------------------------------------------------ */
/* PageRank (algo/pagerank.rs)                                                */
/* ------------------------------------------------------------------------ */

typedef struct {
  const orc_adj *inc;
  const uint32_t *out_deg;    /* unweighted */
  const double *out_str;      /* weighted */
  const double *weights;      /* weighted */
  const double *rank;
  double *next;
  double base, d;
} pr_ctx;

/* pagerank.rs:113-123: acc += rank[v] / od over in-neighbours, od > 0. */
static void pr_sweep(void *p, uint64_t lo, uint64_t hi, int tid) {
  pr_ctx *c = (pr_ctx *)p;
  (void)tid;
  for (uint64_t u = lo; u < hi; u++) {
    double acc = 0.0;
    for (uint64_t k = c->inc->offsets[u]; k < c->inc->offsets[u + 1]; k++) {
      uint32_t v = c->inc->targets[k];
      uint32_t od = c->out_deg[v];
      if (od > 0) acc += c->rank[v] / (double)od;
    }
    c->next[u] = c->base + c->d * acc;
  }
}

/* pagerank.rs:159-166: acc += w * rank[v] / os for os > 0. */
static void prw_sweep(void *p, uint64_t lo, uint64_t hi, int tid) {
  pr_ctx *c = (pr_ctx *)p;
  (void)tid;
  for (uint64_t u = lo; u < hi; u++) {
    double acc = 0.0;
    for (uint64_t k = c->inc->offsets[u]; k < c->inc->offsets[u + 1]; k++) {
      uint32_t v = c->inc->targets[k];
      uint32_t e = c->inc->edge_ids[k];
      double os = c->out_str[v];
      if (os > 0.0) acc += c->weights[e] * c->rank[v] / os;
    }
    c->next[u] = c->base + c->d * acc;
  }
}

#define L1_CHUNK 8192u

/* l1_delta (pagerank.rs:44-52): 8192-element chunks summed sequentially,
 * chunk partials summed in order. */
typedef struct {
  const double *a, *b;
  uint64_t n;
  double *partials;
} l1c;

static void l1_run(void *p, uint64_t lo, uint64_t hi, int tid) {
  l1c *c = (l1c *)p;
  (void)tid;
  for (uint64_t ch = lo; ch < hi; ch++) {
    uint64_t s = ch * L1_CHUNK, e = s + L1_CHUNK;
    if (e > c->n) e = c->n;
    double acc = 0.0;
    for (uint64_t i = s; i < e; i++) acc += fabs(c->a[i] - c->b[i]);
    c->partials[ch] = acc;
  }
}

static double l1_delta(const double *a, const double *b, uint64_t n) {
  uint64_t nch = (n + L1_CHUNK - 1) / L1_CHUNK;
  double *partials = (double *)malloc((nch ? nch : 1) * sizeof(double));
  l1c c = {a, b, n, partials};
  par_ranges(nch, par_threads_for(n), l1_run, &c);
  double s = 0.0;
  for (uint64_t ch = 0; ch < nch; ch++) s += partials[ch];
  free(partials);
  return s;
}

/* Per-iteration L1 residuals of this thread's last power_iterate call (test
 * infrastructure: lets a test show that a differing iteration count sits
 * next to tol).  Not part of the reference. */
#define ORC_MAX_DELTAS 4096u
static __thread double g_deltas[ORC_MAX_DELTAS];
static __thread uint32_t g_n_deltas;

uint32_t orc_pagerank_deltas(double *out, uint32_t cap) {
  uint32_t k = g_n_deltas < cap ? g_n_deltas : cap;
  for (uint32_t i = 0; i < k; i++) out[i] = g_deltas[i];
  return g_n_deltas;
}

/* power_iterate (pagerank.rs:63-94). Returns iterations run; the final
 * rank vector (no renormalisation) is copied to out. */
static uint32_t power_iterate(uint64_t n, double d, uint32_t max_iter, double tol,
                              const uint64_t *dangling, uint64_t n_dangling,
                              pr_ctx *ctx, range_fn sweep, uint64_t work,
                              double *out) {
  double nf = (double)n;
  double *rank = (double *)malloc(n * sizeof(double));
  double *next = (double *)calloc(n, sizeof(double));
  for (uint64_t i = 0; i < n; i++) rank[i] = 1.0 / nf;
  uint32_t it;
  g_n_deltas = 0;
  for (it = 0; it < max_iter;) {
    double dangling_mass = 0.0;
    for (uint64_t i = 0; i < n_dangling; i++) dangling_mass += rank[dangling[i]];
    double base = (1.0 - d) / nf + d * dangling_mass / nf;
    ctx->rank = rank;
    ctx->next = next;
    ctx->base = base;
    ctx->d = d;
    par_ranges(n, par_threads_for(work), sweep, ctx);
    double delta = l1_delta(next, rank, n);
    if (it < ORC_MAX_DELTAS) g_deltas[it] = delta;
    g_n_deltas = it + 1 < ORC_MAX_DELTAS ? it + 1 : ORC_MAX_DELTAS;
    double *tmp = rank;
    rank = next;
    next = tmp;
    it++;
    if (delta < tol) break;
  }
  memcpy(out, rank, n * sizeof(double));
  free(rank);
  free(next);
  return it;
}

uint32_t orc_pagerank(orc_topo *t, double damping, uint32_t max_iter,
                      double tol, double *out) {
  uint64_t n = t->n;
  if (n == 0) return 0;
  uint32_t *out_deg = (uint32_t *)malloc(n * sizeof(uint32_t));
  for (uint64_t u = 0; u < n; u++) out_deg[u] = (uint32_t)(t->out.offsets[u + 1] - t->out.offsets[u]);
  const orc_adj *inc = topo_incoming(t);
  uint64_t *dangling = (uint64_t *)malloc(n * sizeof(uint64_t));
  uint64_t nd = 0;
  for (uint64_t u = 0; u < n; u++)
    if (out_deg[u] == 0) dangling[nd++] = u;
  pr_ctx ctx = {0};
  ctx.inc = inc;
  ctx.out_deg = out_deg;
  uint32_t it = power_iterate(n, damping, max_iter, tol, dangling, nd, &ctx,
                              pr_sweep, n + t->m, out);
  free(out_deg);
  free(dangling);
  return it;
}

uint32_t orc_pagerank_weighted(orc_topo *t, const double *weights,
                               double damping, uint32_t max_iter, double tol,
                               double *out) {
  uint64_t n = t->n;
  if (n == 0) return 0;
  /* pagerank.rs:148-150: serial out-strength, summed in out-CSR slot order. */
  double *out_str = (double *)malloc(n * sizeof(double));
  for (uint64_t v = 0; v < n; v++) {
    double s = 0.0;
    for (uint64_t k = t->out.offsets[v]; k < t->out.offsets[v + 1]; k++)
      s += weights[t->out.edge_ids[k]];
    out_str[v] = s;
  }
  const orc_adj *inc = topo_incoming(t);
  uint64_t *dangling = (uint64_t *)malloc(n * sizeof(uint64_t));
  uint64_t nd = 0;
  for (uint64_t u = 0; u < n; u++)
    if (out_str[u] <= 0.0) dangling[nd++] = u;
  pr_ctx ctx = {0};
  ctx.inc = inc;
  ctx.out_str = out_str;
  ctx.weights = weights;
  uint32_t it = power_iterate(n, damping, max_iter, tol, dangling, nd, &ctx,
                              prw_sweep, n + t->m, out);
  free(out_str);
  free(dangling);
  return it;
}

/* ------------------------------------------------------------------------ */
/* BFS family (algo/bfs.rs)                                                   */
/* ------------------------------------------------------------------------ */

/* Topology::for_each_neighbor (topology.rs:395-404): Out, In, or out then in. */
#define FOR_EACH_NEIGHBOR(T, DIR, U, V, BODY)                                   \
  do {                                                                          \
    if ((DIR) == 0 || (DIR) == 2) {                                             \
      const orc_adj *a_ = &(T)->out;                                            \
      for (uint64_t k_ = a_->offsets[U]; k_ < a_->offsets[(U) + 1]; k_++) {     \
        uint32_t V = a_->targets[k_];                                           \
        BODY;                                                                   \
      }                                                                         \
    }                                                                           \
    if ((DIR) == 1 || (DIR) == 2) {                                             \
      const orc_adj *a_ = &(T)->inc;                                            \
      for (uint64_t k_ = a_->offsets[U]; k_ < a_->offsets[(U) + 1]; k_++) {     \
        uint32_t V = a_->targets[k_];                                           \
        BODY;                                                                   \
      }                                                                         \
    }                                                                           \
  } while (0)

/* for_each_weighted_neighbor (topology.rs:410-430): weight gathered per slot
 * through edge_ids. */
#define FOR_EACH_WNEIGHBOR(T, W, DIR, U, V, WT, BODY)                           \
  do {                                                                          \
    if ((DIR) == 0 || (DIR) == 2) {                                             \
      const orc_adj *a_ = &(T)->out;                                            \
      for (uint64_t k_ = a_->offsets[U]; k_ < a_->offsets[(U) + 1]; k_++) {     \
        uint32_t V = a_->targets[k_];                                           \
        double WT = (W)[a_->edge_ids[k_]];                                      \
        BODY;                                                                   \
      }                                                                         \
    }                                                                           \
    if ((DIR) == 1 || (DIR) == 2) {                                             \
      const orc_adj *a_ = &(T)->inc;                                            \
      for (uint64_t k_ = a_->offsets[U]; k_ < a_->offsets[(U) + 1]; k_++) {     \
        uint32_t V = a_->targets[k_];                                           \
        double WT = (W)[a_->edge_ids[k_]];                                      \
        BODY;                                                                   \
      }                                                                         \
    }                                                                           \
  } while (0)

static void ensure_dir(orc_topo *t, int dir) {
  if (dir != 0) topo_incoming(t);
}

/* bfs_distances (bfs.rs:18-42). */
void orc_bfs_distances(orc_topo *t, uint32_t source, int dir, int32_t *dist) {
  uint64_t n = t->n;
  for (uint64_t i = 0; i < n; i++) dist[i] = -1;
  if ((uint64_t)source >= n) return;
  ensure_dir(t, dir);
  uint32_t *frontier = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint32_t *next = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint64_t fl = 0, nl;
  dist[source] = 0;
  frontier[fl++] = source;
  int32_t level = 1;
  while (fl > 0) {
    nl = 0;
    for (uint64_t i = 0; i < fl; i++) {
      uint32_t u = frontier[i];
      FOR_EACH_NEIGHBOR(t, dir, u, v, {
        if (dist[v] < 0) {
          dist[v] = level;
          next[nl++] = v;
        }
      });
    }
    level++;
    uint32_t *tmp = frontier;
    frontier = next;
    next = tmp;
    fl = nl;
  }
  free(frontier);
  free(next);
}

/* shortest_path (bfs.rs:48-102): parents, early exit after the frontier node
 * whose scan discovered the target, backtrack. */
int64_t orc_shortest_path(orc_topo *t, uint32_t source, uint32_t target,
                          int dir, uint32_t *path_out) {
  uint64_t n = t->n;
  if ((uint64_t)source >= n || (uint64_t)target >= n) return -1;
  if (source == target) {
    path_out[0] = source;
    return 1;
  }
  ensure_dir(t, dir);
  int64_t *parent = (int64_t *)malloc(n * sizeof(int64_t));
  for (uint64_t i = 0; i < n; i++) parent[i] = -1;
  parent[source] = source;
  uint32_t *frontier = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint32_t *next = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint64_t fl = 0, nl;
  frontier[fl++] = source;
  int found = 0;
  while (fl > 0 && !found) {
    nl = 0;
    for (uint64_t i = 0; i < fl; i++) {
      uint32_t u = frontier[i];
      int hit = 0;
      FOR_EACH_NEIGHBOR(t, dir, u, v, {
        if (parent[v] < 0) {
          parent[v] = u;
          if (v == target) hit = 1;
          next[nl++] = v;
        }
      });
      if (hit) {
        found = 1;
        break;
      }
    }
    uint32_t *tmp = frontier;
    frontier = next;
    next = tmp;
    fl = nl;
  }
  int64_t len = -1;
  if (found) {
    /* Backtrack target -> source, then reverse. */
    uint64_t l = 0;
    uint32_t cur = target;
    path_out[l++] = cur;
    while (cur != source) {
      cur = (uint32_t)parent[cur];
      path_out[l++] = cur;
    }
    for (uint64_t i = 0; i < l / 2; i++) {
      uint32_t x = path_out[i];
      path_out[i] = path_out[l - 1 - i];
      path_out[l - 1 - i] = x;
    }
    len = (int64_t)l;
  }
  free(parent);
  free(frontier);
  free(next);
  return len;
}

/* TotalF64 (bfs.rs:108-120): f64::total_cmp key. */
static int64_t total_key(double x) {
  int64_t k;
  memcpy(&k, &x, sizeof(k));
  k ^= (int64_t)(((uint64_t)(k >> 63)) >> 1);
  return k;
}

/* Min-heap on (TotalF64(dist), node): BinaryHeap<Reverse<(TotalF64, u32)>>.
 * Keys are pairwise distinct, so the pop order is fixed by the key order. */
typedef struct {
  int64_t key;
  double d;
  uint32_t v;
} heap_ent;

typedef struct {
  heap_ent *a;
  uint64_t len, cap;
} min_heap;

static int heap_less(const heap_ent *x, const heap_ent *y) {
  if (x->key != y->key) return x->key < y->key;
  return x->v < y->v;
}

static void heap_push(min_heap *h, double d, uint32_t v) {
  if (h->len == h->cap) {
    h->cap = h->cap ? h->cap * 2 : 64;
    h->a = (heap_ent *)realloc(h->a, h->cap * sizeof(heap_ent));
  }
  heap_ent e = {total_key(d), d, v};
  uint64_t i = h->len++;
  while (i > 0) {
    uint64_t p = (i - 1) / 2;
    if (!heap_less(&e, &h->a[p])) break;
    h->a[i] = h->a[p];
    i = p;
  }
  h->a[i] = e;
}

static int heap_pop(min_heap *h, double *d, uint32_t *v) {
  if (h->len == 0) return 0;
  *d = h->a[0].d;
  *v = h->a[0].v;
  heap_ent last = h->a[--h->len];
  uint64_t i = 0, n = h->len;
  while (1) {
    uint64_t l = 2 * i + 1, r = l + 1, s = i;
    const heap_ent *best = &last;
    if (l < n && heap_less(&h->a[l], best)) {
      s = l;
      best = &h->a[l];
    }
    if (r < n && heap_less(&h->a[r], best)) {
      s = r;
      best = &h->a[r];
    }
    if (s == i) break;
    h->a[i] = h->a[s];
    i = s;
  }
  if (n > 0) h->a[i] = last;
  return 1;
}

/* dijkstra_distances (bfs.rs:126-166). */
void orc_dijkstra_distances(orc_topo *t, const double *w, uint32_t source,
                            int dir, double *dist) {
  uint64_t n = t->n;
  for (uint64_t i = 0; i < n; i++) dist[i] = INFINITY;
  if ((uint64_t)source >= n) return;
  ensure_dir(t, dir);
  unsigned char *settled = (unsigned char *)calloc(n, 1);
  min_heap h = {0};
  dist[source] = 0.0;
  heap_push(&h, 0.0, source);
  double du;
  uint32_t u;
  while (heap_pop(&h, &du, &u)) {
    if (settled[u]) continue;
    settled[u] = 1;
    FOR_EACH_WNEIGHBOR(t, w, dir, u, v, wt, {
      if (!settled[v]) {
        double nd = du + wt;
        if (nd < dist[v]) {
          dist[v] = nd;
          heap_push(&h, nd, v);
        }
      }
    });
  }
  free(h.a);
  free(settled);
}

/* shortest_path_weighted_with_cost (bfs.rs:192-259). */
int64_t orc_shortest_path_weighted_with_cost(orc_topo *t, const double *w,
                                             uint32_t source, uint32_t target,
                                             int dir, uint32_t *path_out,
                                             double *cost_out) {
  uint64_t n = t->n;
  if ((uint64_t)source >= n || (uint64_t)target >= n) return -1;
  if (source == target) {
    path_out[0] = source;
    if (cost_out) cost_out[0] = 0.0;
    return 1;
  }
  ensure_dir(t, dir);
  double *dist = (double *)malloc(n * sizeof(double));
  int64_t *parent = (int64_t *)malloc(n * sizeof(int64_t));
  unsigned char *settled = (unsigned char *)calloc(n, 1);
  for (uint64_t i = 0; i < n; i++) {
    dist[i] = INFINITY;
    parent[i] = -1;
  }
  dist[source] = 0.0;
  parent[source] = source;
  min_heap h = {0};
  heap_push(&h, 0.0, source);
  double du;
  uint32_t u;
  while (heap_pop(&h, &du, &u)) {
    if (settled[u]) continue;
    settled[u] = 1;
    if (u == target) break;
    FOR_EACH_WNEIGHBOR(t, w, dir, u, v, wt, {
      if (!settled[v]) {
        double nd = du + wt;
        if (nd < dist[v]) {
          dist[v] = nd;
          parent[v] = u;
          heap_push(&h, nd, v);
        }
      }
    });
  }
  int64_t len = -1;
  if (settled[target]) {
    uint64_t l = 0;
    uint32_t cur = target;
    path_out[l++] = cur;
    while (cur != source) {
      cur = (uint32_t)parent[cur];
      path_out[l++] = cur;
    }
    for (uint64_t i = 0; i < l / 2; i++) {
      uint32_t x = path_out[i];
      path_out[i] = path_out[l - 1 - i];
      path_out[l - 1 - i] = x;
    }
    if (cost_out)
      for (uint64_t i = 0; i < l; i++) cost_out[i] = dist[path_out[i]];
    len = (int64_t)l;
  }
  free(h.a);
  free(dist);
  free(parent);
  free(settled);
  return len;
}

/* ------------------------------------------------------------------------ */
/* k_hop (algo/hop.rs:52-130)                                                 */
/* ------------------------------------------------------------------------ */

typedef struct {
  uint32_t *src, *dst;
  uint64_t len, cap;
} pair_buf;

static void pair_push(pair_buf *b, uint32_t s, uint32_t d) {
  if (b->len == b->cap) {
    b->cap = b->cap ? b->cap * 2 : 256;
    b->src = (uint32_t *)realloc(b->src, b->cap * sizeof(uint32_t));
    b->dst = (uint32_t *)realloc(b->dst, b->cap * sizeof(uint32_t));
  }
  b->src[b->len] = s;
  b->dst[b->len] = d;
  b->len++;
}

typedef struct {
  orc_topo *t;
  const uint32_t *seeds;
  uint32_t k;
  int dir;
  pair_buf *bufs; /* one per thread range, concatenated in order */
} khop_ctx;

/* bfs_seed (hop.rs:80-130) over a contiguous range of seeds. */
static void khop_range(void *p, uint64_t lo, uint64_t hi, int tid) {
  khop_ctx *c = (khop_ctx *)p;
  orc_topo *t = c->t;
  uint64_t n = t->n;
  unsigned char *visited = (unsigned char *)calloc(n, 1);
  uint32_t *frontier = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint32_t *next = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint32_t *touched = (uint32_t *)malloc(n * sizeof(uint32_t));
  pair_buf *out = &c->bufs[tid];
  for (uint64_t si = lo; si < hi; si++) {
    uint32_t seed = c->seeds[si];
    if ((uint64_t)seed >= n) continue;
    uint64_t fl = 0, nl, tl = 0;
    visited[seed] = 1;
    frontier[fl++] = seed;
    touched[tl++] = seed;
    int dir = c->dir;
    for (uint32_t level = 0; level < c->k; level++) {
      nl = 0;
      for (uint64_t i = 0; i < fl; i++) {
        uint32_t u = frontier[i];
        FOR_EACH_NEIGHBOR(t, dir, u, v, {
          if (!visited[v]) {
            visited[v] = 1;
            touched[tl++] = v;
            next[nl++] = v;
            pair_push(out, seed, v);
          }
        });
      }
      if (nl == 0) break;
      uint32_t *tmp = frontier;
      frontier = next;
      next = tmp;
      fl = nl;
    }
    for (uint64_t i = 0; i < tl; i++) visited[touched[i]] = 0;
  }
  free(visited);
  free(frontier);
  free(next);
  free(touched);
}

uint64_t orc_k_hop(orc_topo *t, const uint32_t *seeds, uint64_t n_seeds,
                   uint32_t k, int dir, uint32_t **src_out, uint32_t **dst_out) {
  *src_out = NULL;
  *dst_out = NULL;
  if (k == 0 || t->n == 0) return 0;
  ensure_dir(t, dir);
  int parts = g_threads;
  if ((uint64_t)parts > n_seeds) parts = n_seeds ? (int)n_seeds : 1;
  khop_ctx c = {t, seeds, k, dir, (pair_buf *)calloc(parts, sizeof(pair_buf))};
  par_ranges(n_seeds, parts, khop_range, &c);
  uint64_t total = 0;
  for (int i = 0; i < parts; i++) total += c.bufs[i].len;
  uint32_t *s = (uint32_t *)malloc((total ? total : 1) * sizeof(uint32_t));
  uint32_t *d = (uint32_t *)malloc((total ? total : 1) * sizeof(uint32_t));
  uint64_t o = 0;
  for (int i = 0; i < parts; i++) {
    memcpy(s + o, c.bufs[i].src, c.bufs[i].len * sizeof(uint32_t));
    memcpy(d + o, c.bufs[i].dst, c.bufs[i].len * sizeof(uint32_t));
    o += c.bufs[i].len;
    free(c.bufs[i].src);
    free(c.bufs[i].dst);
  }
  free(c.bufs);
  *src_out = s;
  *dst_out = d;
  return total;
}

void orc_free(void *p) { free(p); }

/* ------------------------------------------------------------------------ */
/* connected_components_weak (algo/components.rs:14-68)                      */
/* ------------------------------------------------------------------------ */

static uint32_t ds_find(uint32_t *parent, uint32_t x) {
  while (parent[x] != x) {
    uint32_t gp = parent[parent[x]];
    parent[x] = gp;
    x = gp;
  }
  return x;
}

void orc_connected_components_weak(orc_topo *t, uint32_t *out) {
  uint64_t n = t->n;
  uint32_t *parent = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
  unsigned char *rank = (unsigned char *)calloc(n ? n : 1, 1);
  for (uint64_t i = 0; i < n; i++) parent[i] = (uint32_t)i;
  for (uint64_t u = 0; u < n; u++) {
    for (uint64_t k = t->out.offsets[u]; k < t->out.offsets[u + 1]; k++) {
      uint32_t v = t->out.targets[k];
      uint32_t ra = ds_find(parent, (uint32_t)u), rb = ds_find(parent, v);
      if (ra == rb) continue;
      unsigned char rra = rank[ra], rrb = rank[rb];
      uint32_t small, big;
      if (rra < rrb) {
        small = ra;
        big = rb;
      } else {
        small = rb;
        big = ra;
      }
      parent[small] = big;
      if (rra == rrb) rank[big] += 1;
    }
  }
  for (uint64_t u = 0; u < n; u++) out[u] = ds_find(parent, (uint32_t)u);
  free(parent);
  free(rank);
}

/* ------------------------------------------------------------------------ */
/* triangle_count / clustering (algo/triangle.rs:23-62, clustering.rs:21-40)  */
/* ------------------------------------------------------------------------ */

static uint32_t intersection_count(const uint32_t *a, uint64_t na,
                                   const uint32_t *b, uint64_t nb) {
  uint64_t i = 0, j = 0;
  uint32_t count = 0;
  while (i < na && j < nb) {
    if (a[i] < b[j])
      i++;
    else if (a[i] > b[j])
      j++;
    else {
      count++;
      i++;
      j++;
    }
  }
  return count;
}

typedef struct {
  const uint64_t *off;
  const uint32_t *tg;
  uint32_t *out;
} tc_ctx;

static void tc_range(void *p, uint64_t lo, uint64_t hi, int tid) {
  tc_ctx *c = (tc_ctx *)p;
  (void)tid;
  for (uint64_t u = lo; u < hi; u++) {
    const uint32_t *nu = c->tg + c->off[u];
    uint64_t du = c->off[u + 1] - c->off[u];
    uint32_t count = 0;
    for (uint64_t i = 0; i < du; i++) {
      uint32_t a = nu[i];
      count += intersection_count(nu + i + 1, du - i - 1, c->tg + c->off[a],
                                  c->off[a + 1] - c->off[a]);
    }
    c->out[u] = count;
  }
}

void orc_triangle_count(orc_topo *t, uint32_t *out) {
  if (t->n == 0) return;
  topo_undirected(t);
  tc_ctx c = {t->u_offsets, t->u_targets, out};
  par_ranges(t->n, par_threads_for(t->n + t->m), tc_range, &c);
}

/* The same per-node count (triangle.rs:23-62: node u, every neighbour
 * a = N(u)[i], |N(u)[i+1..] & N(a)|) for the listed nodes only: the
 * reference computes each node's count independently, so this is the
 * reference's value for those nodes, at a cost a large graph can afford. */
typedef struct {
  const uint64_t *off;
  const uint32_t *tg;
  const uint32_t *nodes;
  uint32_t *out;
} tcn_ctx;

static void tcn_range(void *p, uint64_t lo, uint64_t hi, int tid) {
  tcn_ctx *c = (tcn_ctx *)p;
  (void)tid;
  for (uint64_t q = lo; q < hi; q++) {
    const uint32_t u = c->nodes[q];
    const uint32_t *nu = c->tg + c->off[u];
    uint64_t du = c->off[u + 1] - c->off[u];
    uint32_t count = 0;
    for (uint64_t i = 0; i < du; i++) {
      uint32_t a = nu[i];
      count += intersection_count(nu + i + 1, du - i - 1, c->tg + c->off[a],
                                  c->off[a + 1] - c->off[a]);
    }
    c->out[q] = count;
  }
}

void orc_triangle_count_nodes(orc_topo *t, const uint32_t *nodes, uint64_t k, uint32_t *out) {
  if (t->n == 0 || k == 0) return;
  topo_undirected(t);
  tcn_ctx c = {t->u_offsets, t->u_targets, nodes, out};
  par_ranges(k, par_threads_for(k * 1024), tcn_range, &c);
}

void orc_clustering_coefficient(orc_topo *t, double *out) {
  uint64_t n = t->n;
  if (n == 0) return;
  uint32_t *tri = (uint32_t *)malloc(n * sizeof(uint32_t));
  orc_triangle_count(t, tri);
  for (uint64_t u = 0; u < n; u++) {
    double k = (double)(t->u_offsets[u + 1] - t->u_offsets[u]);
    out[u] = k < 2.0 ? 0.0 : 2.0 * (double)tri[u] / (k * (k - 1.0));
  }
  free(tri);
}

/* ------------------------------------------------------------------------ */
/* rng (algo/rng.rs)                                                          */
/* ------------------------------------------------------------------------ */

#define DEFAULT_SEED 0x5EED5EED5EED5EEDull

static uint64_t sm_next(uint64_t *state) {
  *state += 0x9E3779B97F4A7C15ull;
  uint64_t z = *state;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

void orc_shuffled_order(uint64_t n, uint64_t seed, uint32_t *order) {
  for (uint64_t i = 0; i < n; i++) order[i] = (uint32_t)i;
  uint64_t st = seed ^ 0xD1B54A32D192ED03ull;
  for (uint64_t i = n; i-- > 1;) {
    uint64_t j = sm_next(&st) % (i + 1);
    uint32_t x = order[i];
    order[i] = order[j];
    order[j] = x;
  }
}

static int cmp_u64(const void *a, const void *b) {
  uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return (x > y) - (x < y);
}

uint64_t orc_sample_indices(uint64_t r, uint64_t k, int has_seed, uint64_t seed,
                            uint64_t *out) {
  if (k > r) k = r;
  uint64_t *pool = (uint64_t *)malloc((r ? r : 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < r; i++) pool[i] = i;
  uint64_t st = (has_seed ? seed : DEFAULT_SEED) ^ 0x2545F4914F6CDD1Dull;
  for (uint64_t i = 0; i < k; i++) {
    uint64_t j = i + sm_next(&st) % (r - i);
    uint64_t x = pool[i];
    pool[i] = pool[j];
    pool[j] = x;
  }
  memcpy(out, pool, k * sizeof(uint64_t));
  qsort(out, k, sizeof(uint64_t), cmp_u64);
  free(pool);
  return k;
}

/* sample_sources (betweenness.rs:349-362). */
uint64_t orc_sample_sources(uint64_t n, int has_sample, double frac,
                            int has_seed, uint64_t seed, uint32_t *out) {
  if (!has_sample) {
    for (uint64_t i = 0; i < n; i++) out[i] = (uint32_t)i;
    return n;
  }
  double f = frac;
  if (f < 0.0) f = 0.0;
  if (f > 1.0) f = 1.0;
  double kf = ceil((double)n * f);
  uint64_t k;
  if (isnan(kf) || kf <= 0.0)
    k = 0; /* Rust saturating float->usize cast */
  else if (kf >= 18446744073709551615.0)
    k = UINT64_MAX;
  else
    k = (uint64_t)kf;
  if (k < 1) k = 1;
  if (k > n) k = n;
  if (k == 0) return 0;
  uint32_t *order = (uint32_t *)malloc(n * sizeof(uint32_t));
  orc_shuffled_order(n, has_seed ? seed : DEFAULT_SEED, order);
  memcpy(out, order, k * sizeof(uint32_t));
  free(order);
  return k;
}

/* ------------------------------------------------------------------------ */
/* Betweenness (algo/betweenness.rs)                                          */
/* ------------------------------------------------------------------------ */

typedef struct {
  uint32_t *a;
  uint32_t len, cap;
} u32vec;

static void vpush(u32vec *v, uint32_t x) {
  if (v->len == v->cap) {
    v->cap = v->cap ? v->cap * 2 : 4;
    v->a = (uint32_t *)realloc(v->a, v->cap * sizeof(uint32_t));
  }
  v->a[v->len++] = x;
}

typedef struct {
  int64_t *dist_i;
  double *dist_f;
  double *sigma, *delta;
  u32vec *preds;
  uint32_t *order;
  uint64_t order_len;
  uint32_t *queue;
  unsigned char *settled;
  min_heap heap;
} bscratch;

static void bs_init(bscratch *s, uint64_t n, int weighted) {
  memset(s, 0, sizeof(*s));
  if (weighted) {
    s->dist_f = (double *)malloc(n * sizeof(double));
    for (uint64_t i = 0; i < n; i++) s->dist_f[i] = INFINITY;
    s->settled = (unsigned char *)calloc(n, 1);
  } else {
    s->dist_i = (int64_t *)malloc(n * sizeof(int64_t));
    for (uint64_t i = 0; i < n; i++) s->dist_i[i] = -1;
    s->queue = (uint32_t *)malloc(n * sizeof(uint32_t));
  }
  s->sigma = (double *)calloc(n, sizeof(double));
  s->delta = (double *)calloc(n, sizeof(double));
  s->preds = (u32vec *)calloc(n, sizeof(u32vec));
  s->order = (uint32_t *)malloc(n * sizeof(uint32_t));
}

static void bs_free(bscratch *s, uint64_t n) {
  for (uint64_t i = 0; i < n; i++) free(s->preds[i].a);
  free(s->preds);
  free(s->dist_i);
  free(s->dist_f);
  free(s->sigma);
  free(s->delta);
  free(s->order);
  free(s->queue);
  free(s->settled);
  free(s->heap.a);
}

/* reverse_accumulate (betweenness.rs:81-98). */
static void reverse_accumulate(uint32_t s, bscratch *sc, double *bc) {
  for (uint64_t i = sc->order_len; i-- > 0;) {
    uint32_t w = sc->order[i];
    double coeff = (1.0 + sc->delta[w]) / sc->sigma[w];
    u32vec *p = &sc->preds[w];
    for (uint32_t j = 0; j < p->len; j++) {
      uint32_t v = p->a[j];
      sc->delta[v] += sc->sigma[v] * coeff;
    }
    if (w != s) bc[w] += sc->delta[w];
  }
}

/* brandes_from (betweenness.rs:185-230). */
static void brandes_from(orc_topo *t, uint32_t s, double *bc, bscratch *sc) {
  const orc_adj *out = &t->out;
  uint64_t qh = 0, qt = 0;
  sc->order_len = 0;
  sc->dist_i[s] = 0;
  sc->sigma[s] = 1.0;
  sc->queue[qt++] = s;
  while (qh < qt) {
    uint32_t v = sc->queue[qh++];
    sc->order[sc->order_len++] = v;
    int64_t dv = sc->dist_i[v];
    for (uint64_t k = out->offsets[v]; k < out->offsets[v + 1]; k++) {
      uint32_t w = out->targets[k];
      if (sc->dist_i[w] < 0) {
        sc->dist_i[w] = dv + 1;
        sc->queue[qt++] = w;
      }
      if (sc->dist_i[w] == dv + 1) {
        sc->sigma[w] += sc->sigma[v];
        vpush(&sc->preds[w], v);
      }
    }
  }
  reverse_accumulate(s, sc, bc);
  for (uint64_t i = 0; i < sc->order_len; i++) {
    uint32_t w = sc->order[i];
    sc->dist_i[w] = -1;
    sc->sigma[w] = 0.0;
    sc->delta[w] = 0.0;
    sc->preds[w].len = 0;
  }
  sc->order_len = 0;
}

/* brandes_from_weighted (betweenness.rs:278-339). */
static void brandes_from_weighted(orc_topo *t, const double *weights, uint32_t s,
                                  double *bc, bscratch *sc) {
  const orc_adj *out = &t->out;
  sc->order_len = 0;
  sc->dist_f[s] = 0.0;
  sc->sigma[s] = 1.0;
  heap_push(&sc->heap, 0.0, s);
  double du;
  uint32_t u;
  while (heap_pop(&sc->heap, &du, &u)) {
    if (sc->settled[u]) continue;
    sc->settled[u] = 1;
    sc->order[sc->order_len++] = u;
    for (uint64_t k = out->offsets[u]; k < out->offsets[u + 1]; k++) {
      uint32_t w = out->targets[k];
      if (sc->settled[w]) continue;
      double nd = du + weights[out->edge_ids[k]];
      if (nd < sc->dist_f[w]) {
        sc->dist_f[w] = nd;
        sc->sigma[w] = sc->sigma[u];
        sc->preds[w].len = 0;
        vpush(&sc->preds[w], u);
        heap_push(&sc->heap, nd, w);
      } else if (nd == sc->dist_f[w]) {
        sc->sigma[w] += sc->sigma[u];
        vpush(&sc->preds[w], u);
      }
    }
  }
  reverse_accumulate(s, sc, bc);
  for (uint64_t i = 0; i < sc->order_len; i++) {
    uint32_t w = sc->order[i];
    sc->dist_f[w] = INFINITY;
    sc->sigma[w] = 0.0;
    sc->delta[w] = 0.0;
    sc->settled[w] = 0;
    sc->preds[w].len = 0;
  }
  sc->order_len = 0;
}

#define SRC_CHUNK 64u

typedef struct {
  orc_topo *t;
  const double *weights;
  const uint32_t *sources;
  uint64_t k;
  uint64_t chunk0;   /* first chunk of this wave */
  double **partials; /* one n-vector per thread slot */
  bscratch *scratch;
} bc_ctx;

static void bc_wave(void *p, uint64_t lo, uint64_t hi, int tid) {
  bc_ctx *c = (bc_ctx *)p;
  (void)tid;
  uint64_t n = c->t->n;
  for (uint64_t slot = lo; slot < hi; slot++) {
    uint64_t ch = c->chunk0 + slot;
    double *acc = c->partials[slot];
    memset(acc, 0, n * sizeof(double));
    uint64_t s0 = ch * SRC_CHUNK, s1 = s0 + SRC_CHUNK;
    if (s1 > c->k) s1 = c->k;
    for (uint64_t i = s0; i < s1; i++) {
      if (c->weights)
        brandes_from_weighted(c->t, c->weights, c->sources[i], acc, &c->scratch[slot]);
      else
        brandes_from(c->t, c->sources[i], acc, &c->scratch[slot]);
    }
  }
}

/* accumulate_sources (betweenness.rs:45-70): 64-source chunks, each summed
 * in source order; chunk partials added into bc in chunk order. */
static void accumulate_sources(orc_topo *t, const double *weights,
                               const uint32_t *sources, uint64_t k, double *bc) {
  uint64_t n = t->n;
  uint64_t nch = (k + SRC_CHUNK - 1) / SRC_CHUNK;
  int slots = g_threads;
  if ((uint64_t)slots > nch) slots = nch ? (int)nch : 1;
  bc_ctx c;
  c.t = t;
  c.weights = weights;
  c.sources = sources;
  c.k = k;
  c.partials = (double **)calloc(slots, sizeof(double *));
  c.scratch = (bscratch *)calloc(slots, sizeof(bscratch));
  for (int i = 0; i < slots; i++) {
    c.partials[i] = (double *)malloc(n * sizeof(double));
    bs_init(&c.scratch[i], n, weights != NULL);
  }
  for (uint64_t i = 0; i < n; i++) bc[i] = 0.0;
  for (uint64_t ch0 = 0; ch0 < nch; ch0 += slots) {
    uint64_t wave = nch - ch0 < (uint64_t)slots ? nch - ch0 : (uint64_t)slots;
    c.chunk0 = ch0;
    par_ranges(wave, (int)wave, bc_wave, &c);
    for (uint64_t s = 0; s < wave; s++)
      for (uint64_t i = 0; i < n; i++) bc[i] += c.partials[s][i];
  }
  for (int i = 0; i < slots; i++) {
    free(c.partials[i]);
    bs_free(&c.scratch[i], n);
  }
  free(c.partials);
  free(c.scratch);
}

static void betweenness_impl(orc_topo *t, const double *weights, int has_sample,
                             double sample, int has_seed, uint64_t seed,
                             double *out) {
  uint64_t n = t->n;
  if (n == 0) return;
  uint32_t *sources = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint64_t k = orc_sample_sources(n, has_sample, sample, has_seed, seed, sources);
  if (k == 0) {
    for (uint64_t i = 0; i < n; i++) out[i] = 0.0;
    free(sources);
    return;
  }
  accumulate_sources(t, weights, sources, k, out);
  if (has_sample) {
    double scale = (double)n / (double)k;
    for (uint64_t i = 0; i < n; i++) out[i] = out[i] * scale;
  }
  free(sources);
}

void orc_betweenness(orc_topo *t, int has_sample, double sample, int has_seed,
                     uint64_t seed, double *out) {
  betweenness_impl(t, NULL, has_sample, sample, has_seed, seed, out);
}

void orc_betweenness_weighted(orc_topo *t, const double *weights,
                              int has_sample, double sample, int has_seed,
                              uint64_t seed, double *out) {
  betweenness_impl(t, weights, has_sample, sample, has_seed, seed, out);
}

void orc_betweenness_sources(orc_topo *t, const double *weights,
                             const uint32_t *sources, uint64_t k, double *out) {
  if (t->n == 0) return;
  accumulate_sources(t, weights, sources, k, out);
}

/* ------------------------------------------------------------------------ */
/* IdMap::from_edge_batches for Int64 ids (id_map.rs:220-260, intern_i64     */
/* :294-320): edges are visited in chunk order and, per edge, src is interned */
/* before dst; an id's dense index is the number of distinct ids seen before  */
/* its first occurrence.  The reference uses an FxHashMap; the order of the   */
/* result depends only on first occurrences, so any exact map gives the same  */
/* output.  Here: open addressing over 2^k slots with linear probing.         */
/* ------------------------------------------------------------------------ */
static uint64_t idmap_mix(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return x;
}

uint64_t orc_idmap_build(const int64_t *src, const int64_t *dst, uint64_t n_edges,
                         uint32_t *dense_src, uint32_t *dense_dst, int64_t *to_user) {
  uint64_t cap = 16;
  while (cap < 4 * n_edges + 16) cap <<= 1;
  int64_t *keys = (int64_t *)malloc(cap * sizeof(int64_t));
  uint32_t *vals = (uint32_t *)malloc(cap * sizeof(uint32_t));
  unsigned char *used = (unsigned char *)calloc(cap, 1);
  uint64_t next = 0;
  for (uint64_t i = 0; i < 2 * n_edges; i++) {
    const int64_t key = (i & 1) ? dst[i >> 1] : src[i >> 1];
    uint64_t h = idmap_mix((uint64_t)key) & (cap - 1);
    while (used[h] && keys[h] != key) h = (h + 1) & (cap - 1);
    if (!used[h]) {
      used[h] = 1;
      keys[h] = key;
      vals[h] = (uint32_t)next;
      to_user[next++] = key;
    }
    if (i & 1)
      dense_dst[i >> 1] = vals[h];
    else
      dense_src[i >> 1] = vals[h];
  }
  free(keys);
  free(vals);
  free(used);
  return next;
}

/* ------------------------------------------------------------------------ */
/* closeness / closeness_weighted (algo/closeness.rs:69-224) and the path     */
/* statistics avg_path_length / diameter (ursa-plan/src/stats.rs:82-167).     */
/* Each source's traversal is independent: sources run in parallel ranges,   */
/* each writing its own slots; folds across sources happen in source order.   */
/* ------------------------------------------------------------------------ */
typedef struct {
  orc_topo *t;
  const double *w;
  const uint32_t *sources;
  double *out;          /* closeness per source */
  int64_t *sum, *cnt;   /* per-source hop-distance folds (stats) */
  int32_t *mx;
} clo_ctx;

static void clo_range(void *p, uint64_t lo, uint64_t hi, int tid) {
  (void)tid;
  clo_ctx *c = (clo_ctx *)p;
  uint64_t n = c->t->n;
  int32_t *dist = (int32_t *)malloc((n ? n : 1) * sizeof(int32_t));
  for (uint64_t i = lo; i < hi; i++) {
    uint32_t u = c->sources ? c->sources[i] : (uint32_t)i;
    orc_bfs_distances(c->t, u, 0, dist);
    int64_t sum = 0, reach = 0;
    int32_t mx = 0;
    for (uint64_t v = 0; v < n; v++)
      if (dist[v] >= 1) { /* closeness.rs:115-122, stats.rs:112-121 */
        sum += dist[v];
        reach++;
        if (dist[v] > mx) mx = dist[v];
      }
    if (c->out) c->out[i] = sum > 0 ? (double)reach / (double)sum : 0.0;
    if (c->sum) {
      c->sum[i] = sum;
      c->cnt[i] = reach;
      c->mx[i] = mx;
    }
  }
  free(dist);
}

void orc_closeness(orc_topo *t, double *out) {
  clo_ctx c = {t, NULL, NULL, out, NULL, NULL, NULL};
  par_ranges(t->n, par_threads_for(t->n * (t->n + t->m)), clo_range, &c);
}

/* closeness_one (closeness.rs:98-128) for the given sources only: out[i] is
 * the closeness of sources[i]. */
void orc_closeness_sources(orc_topo *t, const uint32_t *sources, uint64_t k, double *out) {
  clo_ctx c = {t, NULL, sources, out, NULL, NULL, NULL};
  par_ranges(k, par_threads_for(k * (t->n + t->m)), clo_range, &c);
}

static void clow_range(void *p, uint64_t lo, uint64_t hi, int tid) {
  (void)tid;
  clo_ctx *c = (clo_ctx *)p;
  uint64_t n = c->t->n;
  double *dist = (double *)malloc((n ? n : 1) * sizeof(double));
  for (uint64_t u = lo; u < hi; u++) {
    orc_dijkstra_distances(c->t, c->w, (uint32_t)u, 0, dist);
    double sum = 0.0; /* node-order fold (closeness.rs:196-217) */
    int64_t reach = 0;
    for (uint64_t v = 0; v < n; v++)
      if (v != u && isfinite(dist[v])) {
        sum += dist[v];
        reach++;
      }
    c->out[u] = sum > 0.0 ? (double)reach / sum : 0.0;
  }
  free(dist);
}

void orc_closeness_weighted(orc_topo *t, const double *w, double *out) {
  clo_ctx c = {t, w, NULL, out, NULL, NULL, NULL};
  par_ranges(t->n, par_threads_for(t->n * (t->n + t->m)), clow_range, &c);
}

/* stats.rs:82-101 sample_sources: None -> all; Some(frac) -> k evenly strided. */
static uint64_t stats_sources(uint64_t n, int has_frac, double frac, uint32_t *out) {
  if (!has_frac) {
    for (uint64_t i = 0; i < n; i++) out[i] = (uint32_t)i;
    return n;
  }
  double f = frac < 0.0 ? 0.0 : (frac > 1.0 ? 1.0 : frac);
  double kd = round((double)n * f);
  if (kd < 1.0) kd = 1.0;
  uint64_t k = (uint64_t)kd;
  if (k > n) k = n;
  double step = k ? (double)n / (double)k : 1.0;
  if (step < 1.0) step = 1.0;
  for (uint64_t i = 0; i < k; i++) {
    uint64_t v = (uint64_t)floor((double)i * step);
    out[i] = (uint32_t)(v < n - 1 ? v : n - 1);
  }
  return k;
}

/* bfs_source_scan (stats.rs:107-140): per-source f64 sums folded in source
 * order. */
static void stats_scan(orc_topo *t, const uint32_t *src, uint64_t k, double *sum, uint64_t *count,
                       int32_t *max) {
  int64_t *ps = (int64_t *)malloc((k ? k : 1) * sizeof(int64_t));
  int64_t *pc = (int64_t *)malloc((k ? k : 1) * sizeof(int64_t));
  int32_t *pm = (int32_t *)malloc((k ? k : 1) * sizeof(int32_t));
  clo_ctx c = {t, NULL, src, NULL, ps, pc, pm};
  par_ranges(k, par_threads_for(k * (t->n + t->m)), clo_range, &c);
  double s = 0.0;
  uint64_t cnt = 0;
  int32_t mx = 0;
  for (uint64_t i = 0; i < k; i++) {
    s += (double)ps[i]; /* a per-source f64 sum of integers: exact below 2^53 */
    cnt += (uint64_t)pc[i];
    if (pm[i] > mx) mx = pm[i];
  }
  *sum = s;
  *count = cnt;
  *max = mx;
  free(ps);
  free(pc);
  free(pm);
}

double orc_avg_path_length(orc_topo *t, int has_sample, double sample) {
  uint32_t *src = (uint32_t *)malloc((t->n ? t->n : 1) * sizeof(uint32_t));
  uint64_t k = stats_sources(t->n, has_sample, sample, src);
  double sum;
  uint64_t count;
  int32_t mx;
  stats_scan(t, src, k, &sum, &count, &mx);
  free(src);
  return count == 0 ? 0.0 : sum / (double)count;
}

int64_t orc_diameter(orc_topo *t, int approximate) {
  uint64_t n = t->n;
  uint32_t *src = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
  uint64_t k = approximate && n > 0
                   ? stats_sources(n, 1, fmin(128.0 / (double)n, 1.0), src)
                   : stats_sources(n, 0, 0.0, src);
  double sum;
  uint64_t count;
  int32_t mx;
  stats_scan(t, src, k, &sum, &count, &mx);
  free(src);
  return mx;
}
