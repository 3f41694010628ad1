/*
 * gen.c -- seeded, counter-based synthetic graph generators used by the
 * benchmark and the parity tests.  The reference ships no generator at these
 * shapes (its benchmark datasets are NetworkX ER/BA/grid/SBM), so these are
 * project-defined:
 *
 *  R-MAT(scale, edge_factor, a, b, c, seed): edge i recurses `scale` levels;
 *    level L draws r = U[0,1) from mix64(seed, i, L) and picks quadrant
 *    (0,0) if r<a, (0,1) if r<a+b, (1,0) if r<a+b+c, else (1,1); the row bit
 *    goes to src, the column bit to dst, most significant first.  No noise and
 *    no vertex relabelling.  Self-loops are dropped, then duplicate (u,v)
 *    pairs, keeping the first occurrence in generation order, so the row
 *    order stays unsorted.
 *  Poisson(n, mean, seed): node u draws out-degree ~ Poisson(mean) (Knuth's
 *    product-of-uniforms method) and uniform targets; rows are node-major;
 *    multiplicity and self-loops are kept.
 *  Weights: f32 uniform in [lo, hi) per edge row.
 *
 * Every draw is a pure function of (seed, index, lane), so the output does not
 * depend on the thread count.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define GOLDEN 0x9E3779B97F4A7C15ull

static inline uint64_t fmix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* One 64-bit draw for (seed, index, lane); lanes < 64. */
static inline uint64_t draw(uint64_t seed, uint64_t index, uint64_t lane) {
  uint64_t s = fmix(seed ^ 0xA0761D6478BD642Full);
  return fmix(s + (index * 64u + lane + 1u) * GOLDEN);
}

static inline double unit(uint64_t x) { return (double)(x >> 11) * (1.0 / 9007199254740992.0); }

typedef void (*range_fn)(void *ctx, uint64_t lo, uint64_t hi, int tid);
typedef struct {
  range_fn fn;
  void *ctx;
  uint64_t lo, hi;
  int tid;
} job;
static void *tramp(void *p) {
  job *j = (job *)p;
  j->fn(j->ctx, j->lo, j->hi, j->tid);
  return NULL;
}
static void par(uint64_t n, int parts, range_fn fn, void *ctx) {
  if (parts < 1) parts = 1;
  if (parts > 128) parts = 128;
  if ((uint64_t)parts > n) parts = n ? (int)n : 1;
  pthread_t th[128];
  job jobs[128];
  uint64_t step = (n + parts - 1) / parts;
  for (int t = 0; t < parts; t++) {
    uint64_t lo = step * t, hi = lo + step;
    if (lo > n) lo = n;
    if (hi > n) hi = n;
    jobs[t] = (job){fn, ctx, lo, hi, t};
  }
  for (int t = 1; t < parts; t++) pthread_create(&th[t], NULL, tramp, &jobs[t]);
  tramp(&jobs[0]);
  for (int t = 1; t < parts; t++) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------------ */
typedef struct {
  int scale;
  double t0, t1, t2;
  uint64_t seed;
  uint32_t *src, *dst;
} rmat_ctx;

static void rmat_range(void *p, uint64_t lo, uint64_t hi, int tid) {
  rmat_ctx *c = (rmat_ctx *)p;
  (void)tid;
  uint64_t s = fmix(c->seed ^ 0xA0761D6478BD642Full);
  for (uint64_t i = lo; i < hi; i++) {
    uint32_t u = 0, v = 0;
    for (int L = 0; L < c->scale; L++) {
      double r = unit(fmix(s + (i * 64u + (uint64_t)L + 1u) * GOLDEN));
      uint32_t bu, bv;
      if (r < c->t0) {
        bu = 0;
        bv = 0;
      } else if (r < c->t1) {
        bu = 0;
        bv = 1;
      } else if (r < c->t2) {
        bu = 1;
        bv = 0;
      } else {
        bu = 1;
        bv = 1;
      }
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    c->src[i] = u;
    c->dst[i] = v;
  }
}

/* Dedup keeping the first occurrence: rows are split by key hash into NP
 * partitions (stable within a partition), each partition runs an
 * open-addressing set in row order, then kept rows are compacted in order. */
#define NP 256
typedef struct {
  const uint32_t *src, *dst;
  uint64_t m;
  int threads;
  uint64_t (*cnt)[NP];   /* [thread][partition] */
  uint64_t *part_off;    /* NP + 1 */
  uint32_t *rows;        /* m, grouped by partition */
  unsigned char *keep;   /* m */
  uint64_t *kept_cnt;    /* per thread */
  uint32_t *out_src, *out_dst;
} dd_ctx;

static inline uint64_t ekey(const dd_ctx *c, uint64_t r) {
  return ((uint64_t)c->src[r] << 32) | c->dst[r];
}
static inline uint32_t part_of(uint64_t key) { return (uint32_t)(fmix(key + GOLDEN) >> 56); }

static void dd_count(void *p, uint64_t lo, uint64_t hi, int tid) {
  dd_ctx *c = (dd_ctx *)p;
  memset(c->cnt[tid], 0, sizeof(c->cnt[tid]));
  for (uint64_t r = lo; r < hi; r++) {
    if (c->src[r] == c->dst[r]) continue; /* self-loops dropped */
    c->cnt[tid][part_of(ekey(c, r))]++;
  }
}

static void dd_scatter(void *p, uint64_t lo, uint64_t hi, int tid) {
  dd_ctx *c = (dd_ctx *)p;
  uint64_t pos[NP];
  for (int q = 0; q < NP; q++) pos[q] = c->cnt[tid][q]; /* converted to bases */
  for (uint64_t r = lo; r < hi; r++) {
    if (c->src[r] == c->dst[r]) continue;
    c->rows[pos[part_of(ekey(c, r))]++] = (uint32_t)r;
  }
}

static void dd_parts(void *p, uint64_t lo, uint64_t hi, int tid) {
  dd_ctx *c = (dd_ctx *)p;
  (void)tid;
  for (uint64_t q = lo; q < hi; q++) {
    uint64_t s = c->part_off[q], e = c->part_off[q + 1], len = e - s;
    if (!len) continue;
    uint64_t cap = 16;
    while (cap < 2 * len) cap <<= 1;
    uint64_t *tab = (uint64_t *)malloc(cap * sizeof(uint64_t));
    memset(tab, 0xFF, cap * sizeof(uint64_t));
    for (uint64_t i = s; i < e; i++) {
      uint32_t r = c->rows[i];
      uint64_t k = ekey(c, r);
      uint64_t h = fmix(k ^ 0x5851F42D4C957F2Dull) & (cap - 1);
      for (;;) {
        if (tab[h] == UINT64_MAX) {
          tab[h] = k;
          c->keep[r] = 1;
          break;
        }
        if (tab[h] == k) break;
        h = (h + 1) & (cap - 1);
      }
    }
    free(tab);
  }
}

static void dd_kcount(void *p, uint64_t lo, uint64_t hi, int tid) {
  dd_ctx *c = (dd_ctx *)p;
  uint64_t k = 0;
  for (uint64_t r = lo; r < hi; r++) k += c->keep[r];
  c->kept_cnt[tid] = k;
}

static void dd_compact(void *p, uint64_t lo, uint64_t hi, int tid) {
  dd_ctx *c = (dd_ctx *)p;
  uint64_t o = c->kept_cnt[tid]; /* converted to bases */
  for (uint64_t r = lo; r < hi; r++)
    if (c->keep[r]) {
      c->out_src[o] = c->src[r];
      c->out_dst[o] = c->dst[r];
      o++;
    }
}

/* Drops self-loops and duplicate pairs (first occurrence kept) from
 * (src, dst)[0..m), writing the survivors in order to out_src/out_dst (may
 * alias the inputs only if distinct buffers are used by the caller). Returns
 * the kept count. */
uint64_t ug_dedup(const uint32_t *src, const uint32_t *dst, uint64_t m,
                  uint32_t *out_src, uint32_t *out_dst, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 128) threads = 128;
  if ((uint64_t)threads > m) threads = m ? (int)m : 1;
  dd_ctx c;
  memset(&c, 0, sizeof(c));
  c.src = src;
  c.dst = dst;
  c.m = m;
  c.threads = threads;
  c.cnt = (uint64_t(*)[NP])calloc(threads, sizeof(uint64_t[NP]));
  c.part_off = (uint64_t *)calloc(NP + 1, sizeof(uint64_t));
  c.rows = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
  c.keep = (unsigned char *)calloc(m ? m : 1, 1);
  c.kept_cnt = (uint64_t *)calloc(threads, sizeof(uint64_t));
  c.out_src = out_src;
  c.out_dst = out_dst;
  par(m, threads, dd_count, &c);
  /* Partition-major, thread-minor exclusive prefix keeps row order inside a
   * partition. */
  uint64_t run = 0;
  for (int q = 0; q < NP; q++) {
    c.part_off[q] = run;
    for (int t = 0; t < threads; t++) {
      uint64_t x = c.cnt[t][q];
      c.cnt[t][q] = run;
      run += x;
    }
  }
  c.part_off[NP] = run;
  par(m, threads, dd_scatter, &c);
  par(NP, threads, dd_parts, &c);
  par(m, threads, dd_kcount, &c);
  uint64_t total = 0;
  for (int t = 0; t < threads; t++) {
    uint64_t x = c.kept_cnt[t];
    c.kept_cnt[t] = total;
    total += x;
  }
  par(m, threads, dd_compact, &c);
  free(c.cnt);
  free(c.part_off);
  free(c.rows);
  free(c.keep);
  free(c.kept_cnt);
  return total;
}

/* R-MAT edges (before cleaning) into src/dst[0 .. edge_factor << scale). */
void ug_rmat_raw(int scale, uint64_t edge_factor, double a, double b, double c,
                 uint64_t seed, uint32_t *src, uint32_t *dst, int threads) {
  rmat_ctx x;
  x.scale = scale;
  x.t0 = a;
  x.t1 = a + b;
  x.t2 = a + b + c;
  x.seed = seed;
  x.src = src;
  x.dst = dst;
  par(edge_factor << scale, threads, rmat_range, &x);
}

/* R-MAT with self-loops and duplicates removed. src/dst must hold
 * edge_factor << scale entries; returns the kept count. */
uint64_t ug_rmat(int scale, uint64_t edge_factor, double a, double b, double c,
                 uint64_t seed, uint32_t *src, uint32_t *dst, int threads) {
  uint64_t m = edge_factor << scale;
  uint32_t *rs = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
  uint32_t *rd = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
  ug_rmat_raw(scale, edge_factor, a, b, c, seed, rs, rd, threads);
  uint64_t k = ug_dedup(rs, rd, m, src, dst, threads);
  free(rs);
  free(rd);
  return k;
}

/* ------------------------------------------------------------------------ */
/* Poisson out-degree graph.                                                  */
typedef struct {
  uint64_t n;
  double limit;
  uint64_t seed;
  uint32_t *deg;
  uint64_t *off;
  uint32_t *src, *dst;
} pois_ctx;

static uint32_t pois_deg(uint64_t seed, uint64_t u, double limit) {
  /* Knuth: count draws until the running product falls to <= e^-mean. */
  double prod = unit(draw(seed, u, 0));
  uint32_t k = 0;
  uint64_t lane = 1;
  while (prod > limit) {
    k++;
    prod *= unit(draw(seed ^ 0x632BE59BD9B4E019ull, u * 4096u + lane / 64u, lane % 64u));
    lane++;
  }
  return k;
}

static void pois_deg_range(void *p, uint64_t lo, uint64_t hi, int tid) {
  pois_ctx *c = (pois_ctx *)p;
  (void)tid;
  for (uint64_t u = lo; u < hi; u++) c->deg[u] = pois_deg(c->seed, u, c->limit);
}

static void pois_fill(void *p, uint64_t lo, uint64_t hi, int tid) {
  pois_ctx *c = (pois_ctx *)p;
  (void)tid;
  for (uint64_t u = lo; u < hi; u++) {
    uint64_t o = c->off[u];
    for (uint32_t j = 0; j < c->deg[u]; j++) {
      uint64_t x = draw(c->seed ^ 0x8CB92BA72F3D8DD7ull, u * 4096u + j / 64u, j % 64u);
      c->src[o + j] = (uint32_t)u;
      c->dst[o + j] = (uint32_t)(((x >> 32) * c->n) >> 32);
    }
  }
}

/* Out-degrees for the Poisson graph; returns the edge total. */
uint64_t ug_poisson_degrees(uint64_t n, double mean, uint64_t seed, uint32_t *deg,
                            int threads) {
  pois_ctx c;
  memset(&c, 0, sizeof(c));
  c.n = n;
  c.limit = exp(-mean);
  c.seed = seed;
  c.deg = deg;
  par(n, threads, pois_deg_range, &c);
  uint64_t m = 0;
  for (uint64_t u = 0; u < n; u++) m += deg[u];
  return m;
}

/* Fills node-major rows given the degrees from ug_poisson_degrees. n must be
 * < 2^32; targets are uniform in [0, n). */
void ug_poisson_fill(uint64_t n, uint64_t seed, const uint32_t *deg,
                     uint32_t *src, uint32_t *dst, int threads) {
  pois_ctx c;
  memset(&c, 0, sizeof(c));
  c.n = n;
  c.seed = seed;
  c.deg = (uint32_t *)deg;
  c.off = (uint64_t *)malloc((n + 1) * sizeof(uint64_t));
  c.off[0] = 0;
  for (uint64_t u = 0; u < n; u++) c.off[u + 1] = c.off[u] + deg[u];
  c.src = src;
  c.dst = dst;
  par(n, threads, pois_fill, &c);
  free(c.off);
}

/* f32 weights uniform in [lo, hi): lo + (hi-lo) * k/2^24 for a 24-bit k. */
typedef struct {
  float lo, span;
  uint64_t seed;
  float *out;
} w_ctx;
static void w_range(void *p, uint64_t a, uint64_t b, int tid) {
  w_ctx *c = (w_ctx *)p;
  (void)tid;
  for (uint64_t i = a; i < b; i++) {
    uint32_t k = (uint32_t)(draw(c->seed ^ 0x1D8E4E27C47D124Full, i, 0) >> 40);
    c->out[i] = c->lo + c->span * ((float)k * (1.0f / 16777216.0f));
  }
}
void ug_weights_f32(uint64_t m, float lo, float hi, uint64_t seed, float *out,
                    int threads) {
  w_ctx c = {lo, hi - lo, seed, out};
  par(m, threads, w_range, &c);
}

/* ------------------------------------------------------------------------ */
/* Batches of small R-MAT graphs.  Graph i has n_i nodes, R-MAT on scale      */
/* ceil(log2 n_i) with edge_factor_i * n_i draws and seed seed0 + i; draws    */
/* with an endpoint >= n_i are rejected, then self-loops and duplicates are   */
/* dropped (first occurrence kept).  Edges are written graph after graph with */
/* local node ids.                                                            */
typedef struct {
  const uint64_t *n, *ef, *edge_off;
  uint64_t seed0;
  double t0, t1, t2;
  uint32_t *src, *dst;
  uint64_t *kept;
} rbatch_ctx;

static int ceil_log2(uint64_t n) {
  int s = 0;
  while ((1ull << s) < n) s++;
  return s;
}

static void rbatch_range(void *p, uint64_t lo, uint64_t hi, int tid) {
  rbatch_ctx *c = (rbatch_ctx *)p;
  (void)tid;
  for (uint64_t g = lo; g < hi; g++) {
    uint64_t n = c->n[g], draws = c->ef[g] * n;
    int scale = ceil_log2(n);
    uint64_t seed = c->seed0 + g;
    uint64_t s = fmix(seed ^ 0xA0761D6478BD642Full);
    uint32_t *rs = (uint32_t *)malloc((draws ? draws : 1) * sizeof(uint32_t));
    uint32_t *rd = (uint32_t *)malloc((draws ? draws : 1) * sizeof(uint32_t));
    uint64_t k = 0;
    for (uint64_t i = 0; i < draws; i++) {
      uint32_t u = 0, v = 0;
      for (int L = 0; L < scale; L++) {
        double r = unit(fmix(s + (i * 64u + (uint64_t)L + 1u) * GOLDEN));
        uint32_t bu = r >= c->t1, bv = (r >= c->t0 && r < c->t1) || r >= c->t2;
        u = (u << 1) | bu;
        v = (v << 1) | bv;
      }
      if (u < n && v < n) {
        rs[k] = u;
        rd[k] = v;
        k++;
      }
    }
    uint64_t kept = ug_dedup(rs, rd, k, c->src + c->edge_off[g], c->dst + c->edge_off[g], 1);
    c->kept[g] = kept;
    free(rs);
    free(rd);
  }
}

/* Fills per-graph edges into src/dst at edge_off[g] (capacity ef*n each) and
 * writes the kept counts; the caller compacts. */
void ug_rmat_batch(uint64_t count, const uint64_t *n, const uint64_t *ef, uint64_t seed0,
                   double a, double b, double c, const uint64_t *edge_off, uint32_t *src,
                   uint32_t *dst, uint64_t *kept, int threads) {
  rbatch_ctx x;
  x.n = n;
  x.ef = ef;
  x.edge_off = edge_off;
  x.seed0 = seed0;
  x.t0 = a;
  x.t1 = a + b;
  x.t2 = a + b + c;
  x.src = src;
  x.dst = dst;
  x.kept = kept;
  par(count, threads, rbatch_range, &x);
}

/* Uniform 64-bit draws (used for seeded source/query streams). */
uint64_t ug_draw(uint64_t seed, uint64_t index, uint64_t lane) {
  return draw(seed, index, lane & 63u);
}
