// pagerank.cu -- pull PageRank (unweighted and weighted) as ONE persistent
// cooperative kernel per call.
//
// Reference semantics (ursa-core/src/algo/pagerank.rs):
//   rank_0 = 1/n; per iteration
//     dangling_mass = sum of rank over dangling nodes           (:78)
//     base = (1-d)/n + d*dangling_mass/n                        (:79)
//     next[u] = base + d * sum_{v in in(u)} rank[v]/outdeg[v]   (:81-83, :113-123)
//               (weighted: w_e * rank[v] / out_strength[v], :159-166)
//     delta = L1(next, rank); swap; stop if delta < tol         (:85-91)
//   returns the last `next`, no renormalisation.
//
// B200 design.
//  * Arithmetic: the per-edge share x[v] = rank[v]/divisor[v] is stored as
//    f32 and each row sums its shares with Kahan-compensated f32; the update,
//    L1 residual, dangling mass and the ranks are f64.
//  * Execution CSR (built once per topology, cached): a copy of the in-CSR
//    with node ids relabelled by in-degree, highest first.  Rows of similar
//    degree become contiguous, so each degree class gets a fixed group width
//    (1..32 lanes per row, about four edges per lane) and no warp diverges on
//    row lengths.  On R-MAT graphs in- and out-degree go together, so the
//    smallest ids are also the most-gathered shares: the first kHot of them
//    are copied into shared memory every iteration (about half of all gathers
//    at R-MAT-22), taking them off L2.  Ranks return to the caller's ids at
//    the end.
//  * Work units: a unit is 32/G consecutive rows of a class with group width
//    G, or a kHubChunk-edge chunk of a hub row (in-degree > kHubDeg).  Warps
//    take units round-robin and never wait for each other inside an
//    iteration; a hub's chunk sums are combined in chunk order by whichever
//    chunk arrives last (an arrival counter, no waiting).
//  * One bounded grid barrier per iteration.  Every reduction has a fixed
//    order, so runs are bit-reproducible.
#include <cmath>

#include "fixedpoint.cuh"
#include "primitives.cuh"
#include "topo.cuh"

namespace ug {

namespace {
constexpr int kPrBlock = 1024;
constexpr int kPrWarps = kPrBlock / 32;
constexpr uint32_t kHubDeg = 1024;    // in-degree above which a row is chunked
constexpr uint32_t kHubChunk = 2048;  // edges per hub chunk (64 per lane)
constexpr int kHot = 32768;           // shares cached in shared memory (128 KB)
constexpr int kClasses = 7;           // hub, G = 32, 16, 8, 4, 2, 1
constexpr int kBatchWide = 8;         // loads in flight per lane, 32-lane rows
constexpr int kBatchHub = 16;         // loads in flight per lane, hub chunks
constexpr int kUnitsPerGrab = 8;      // units a warp takes from its block's counter
constexpr uint64_t kBarrierLimitNs = 5000000000ull;  // 5 s per grid barrier wait
}  // namespace

struct PrClassTable {
  uint32_t lo[kClasses], hi[kClasses];   // row ranges (new ids)
  uint32_t unit_begin[kClasses + 1];     // first unit of each class
};

struct PrPlan {
  PrClassTable cls{};
  uint32_t iso_lo = 0;  // rows [iso_lo, n) are isolated: rank follows in closed form
  uint32_t zi_lo = 0;   // rows [zi_lo, n) have no in-edges: rank = base every iteration
  uint32_t n_units = 0, n_hub = 0, n_chunks = 0;
  DevArray<uint2> hub_unit;            // per hub chunk: {hub index, chunk}
  DevArray<uint32_t> hub_first, hub_nch;
  // execution CSR in relabelled ids
  DevArray<uint32_t> old_of_new, new_of_old;
  DevArray<uint32_t> off, src, eid;
  DevArray<uint32_t> outdeg;  // per new id
};

void pr_plan_free(PrPlan* p) { delete p; }
uint64_t pr_plan_bytes(const PrPlan* p) {
  if (!p) return 0;
  return (uint64_t)p->hub_unit.n * sizeof(uint2) +
         4ull * (p->hub_first.n + p->hub_nch.n + p->old_of_new.n + p->new_of_old.n + p->off.n +
                 p->src.n + p->eid.n + p->outdeg.n);
}

namespace {

// ------------------------------------------------------------ plan kernels
// Relabel key, ascending = execution order: in-degree high to low; among
// in-degree-0 nodes, sources (out-degree > 0) before isolated nodes, which
// end the order (their ranks follow in closed form).
__global__ void exec_order_key_k(const uint32_t* __restrict__ in_off,
                                 const uint32_t* __restrict__ out_off, uint64_t n,
                                 uint32_t* __restrict__ key) {
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t din = in_off[u + 1] - in_off[u];
    const uint64_t dout = out_off[u + 1] - out_off[u];
    uint64_t r = din ? 2 * din : (dout ? 1 : 0);
    if (r > 0xFFFFFFFEull) r = 0xFFFFFFFEull;
    key[u] = ~(uint32_t)r;
  }
}

__global__ void relabel_maps_k(const uint32_t* __restrict__ old_of_new, uint64_t n,
                               const uint32_t* __restrict__ in_off,
                               const uint32_t* __restrict__ out_off,
                               uint32_t* __restrict__ new_of_old, uint32_t* __restrict__ deg_new,
                               uint32_t* __restrict__ outdeg_new) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t u = old_of_new[i];
    new_of_old[u] = (uint32_t)i;
    deg_new[i] = in_off[u + 1] - in_off[u];
    outdeg_new[i] = out_off[u + 1] - out_off[u];
  }
}

// Copy row old_of_new[i] of the in-CSR into new row i, relabelling sources.
__global__ void relabel_copy_k(const uint32_t* __restrict__ off_new, uint64_t n, uint64_t m,
                               const uint32_t* __restrict__ old_of_new,
                               const uint32_t* __restrict__ new_of_old,
                               const uint32_t* __restrict__ in_off,
                               const uint32_t* __restrict__ in_src,
                               const uint32_t* __restrict__ in_eid, uint32_t* __restrict__ src_new,
                               uint32_t* __restrict__ eid_new) {
  for_each_slot_owner(off_new, n, m, [&](uint64_t k, uint32_t i) {
    uint32_t u = old_of_new[i];
    uint32_t slot = in_off[u] + (uint32_t)(k - off_new[i]);
    src_new[k] = new_of_old[in_src[slot]];
    eid_new[k] = in_eid[slot];
  });
}

// Class boundaries over the non-increasing degree sequence: bounds[t] =
// number of rows with degree > thr[t]; bounds[kClasses - 1] = first isolated
// row (in- and out-degree 0; they end the execution order); bounds[kClasses]
// = first row without in-edges.
__global__ void class_bounds_k(const uint32_t* __restrict__ deg, const uint32_t* __restrict__ outdeg,
                               uint64_t n, uint32_t* __restrict__ bounds) {
  const uint32_t thr[kClasses - 1] = {kHubDeg, 64u, 32u, 16u, 8u, 4u};
  for (int t = 0; t < kClasses - 1; t++) {
    uint64_t lo = 0, hi = n;  // first index with deg <= thr
    while (lo < hi) {
      uint64_t mid = (lo + hi) >> 1;
      if (deg[mid] > thr[t])
        lo = mid + 1;
      else
        hi = mid;
    }
    bounds[t] = (uint32_t)lo;
  }
  uint64_t lo = 0, hi = n;  // first isolated row
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (deg[mid] != 0 || outdeg[mid] != 0)
      lo = mid + 1;
    else
      hi = mid;
  }
  bounds[kClasses - 1] = (uint32_t)lo;
  lo = 0;
  hi = n;  // first row without in-edges
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (deg[mid] != 0)
      lo = mid + 1;
    else
      hi = mid;
  }
  bounds[kClasses] = (uint32_t)lo;
}

__global__ void hub_nch_k(const uint32_t* __restrict__ deg, uint32_t n_hub,
                          uint32_t* __restrict__ nch) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_hub; i += gridDim.x * blockDim.x)
    nch[i] = (deg[i] + kHubChunk - 1) / kHubChunk;
}

__global__ void hub_units_k(const uint32_t* __restrict__ first, const uint32_t* __restrict__ nch,
                            uint32_t n_hub, uint2* __restrict__ units) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_hub; i += gridDim.x * blockDim.x)
    for (uint32_t c = 0; c < nch[i]; c++) units[first[i] + c] = make_uint2(i, c);
}

// ---------------------------------------------------------- iteration kernel
struct PrArgs {
  uint64_t n;
  uint32_t hot;                        // shares cached in shared memory (<= kHot)
  PrClassTable cls;
  uint32_t n_units;
  const uint32_t* __restrict__ off;    // execution CSR offsets (new ids)
  const uint32_t* __restrict__ src;    // execution CSR sources (new ids)
  const float* __restrict__ w;         // weighted: f32 weight per slot, else null
  const uint32_t* __restrict__ outdeg;   // unweighted divisor (new ids)
  const double* __restrict__ out_str;    // weighted divisor (new ids), else null
  double* rank[2];
  float* x[2];
  const uint2* __restrict__ hub_unit;
  const uint32_t* __restrict__ hub_first;
  const uint32_t* __restrict__ hub_nch;
  uint32_t n_hub;
  F2* chunk_part;            // per hub chunk
  unsigned* hub_cnt;         // per hub: chunk arrivals this iteration
  ulonglong2* hub_contrib[2];  // per hub: (|next-rank|, dangling next), fixed point
  ulonglong2* block_part[2];   // per block, fixed point
  double2* totals;           // [2]: (delta, dangling) published by the barrier
  uint32_t iso_lo;           // first isolated row
  uint32_t zi_lo;            // first row without in-edges (<= iso_lo)
  unsigned* bar_count;
  unsigned* bar_gen;
  int* err;
  double damping;
  double tol;
  uint32_t max_iter;
  uint32_t* out_iters;
  double* out_delta;
  uint32_t* out_buf;
};

struct Fin {
  double delta, dang;
};

// Per-thread fixed-point accumulators of |next - rank| and of the dangling
// rows' next ranks (64-bit, scale 2^-58: order-independent; every partial
// sum is below its total, and the totals are at most 2 and 1).
struct Fx {
  unsigned long long delta, dang;
};

struct PrSmem {
  float hot[kHot];
  ulonglong2 red[kPrWarps];
  unsigned gen;
  int last;
  unsigned next;  // work counter of the block (dynamic unit scheduling)
};

__device__ __forceinline__ double row_divisor(const PrArgs& a, uint64_t u) {
  return a.out_str ? a.out_str[u] : (double)a.outdeg[u];
}

__device__ __forceinline__ void finish_row(const PrArgs& a, uint64_t u, double sum, double old,
                                           double div, double base, int cur, Fx& f) {
  // next[u] = base + d * contrib(u)   (pagerank.rs:81-83)
  double nx = __dadd_rn(base, __dmul_rn(a.damping, sum));
  f.delta += fx64_of(fabs(__dsub_rn(nx, old)));
  a.rank[cur ^ 1][u] = nx;
  bool dangling = !(div > 0.0);
  a.x[cur ^ 1][u] = dangling ? 0.f : (float)(nx / div);
  if (dangling) f.dang += fx64_of(nx);
}

__device__ __forceinline__ void init_row(const PrArgs& a, uint64_t u, double r0, Fx& f) {
  a.rank[0][u] = r0;
  double div = row_divisor(a, u);
  bool dangling = !(div > 0.0);
  a.x[0][u] = dangling ? 0.f : (float)(r0 / div);
  if (dangling) f.dang += fx64_of(r0);
}

__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
  float y = __fsub_rn(v, c);
  float t = __fadd_rn(s, y);
  c = __fsub_rn(__fsub_rn(t, s), y);
  s = t;
}

// Share of source v: shared-memory copy for the hottest ids, else global.
__device__ __forceinline__ float share(const PrArgs& a, const PrSmem& sm, const float* x,
                                      uint32_t v) {
  return v < a.hot ? sm.hot[v] : x[v];
}

// Sums the shares of edges [b + sub, e) with stride G; B source loads (and
// then B gathers) in flight per lane.
template <int G, bool kW, int B>
__device__ __forceinline__ F2 row_sum(const PrArgs& a, const PrSmem& sm, const float* x, uint32_t b,
                                      uint32_t e, int sub) {
  float s = 0.f, c = 0.f;
  for (uint32_t j = b + sub; j < e; j += B * G) {
    uint32_t v[B];
#pragma unroll
    for (int k = 0; k < B; k++) {
      uint32_t jj = j + k * G;
      v[k] = jj < e ? __ldcs(a.src + jj) : 0u;
    }
    float sv[B];
#pragma unroll
    for (int k = 0; k < B; k++) {
      uint32_t jj = j + k * G;
      sv[k] = 0.f;
      if (jj < e) {
        sv[k] = share(a, sm, x, v[k]);
        if (kW) sv[k] = __fmul_rn(sv[k], __ldcs(a.w + jj));
      }
    }
#pragma unroll
    for (int k = 0; k < B; k++)
      if (j + k * G < e) kahan_add(s, c, sv[k]);
  }
  return F2{s, -c};
}

// Fixed-order reduction over the G lanes of a group; valid in sub == 0.
template <int G>
__device__ __forceinline__ F2 group_sum(F2 v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    F2 t{__shfl_down_sync(0xffffffffu, v.hi, o, G), __shfl_down_sync(0xffffffffu, v.lo, o, G)};
    v = f2_combine(v, t);
  }
  return v;
}

// One unit of a row class: 32/G consecutive rows, G lanes per row.
template <int G, bool kW>
__device__ __forceinline__ void class_unit(const PrArgs& a, const PrSmem& sm, uint32_t lo,
                                           uint32_t hi, uint32_t unit, int cur, double base,
                                           Fx& f) {
  const int lane = threadIdx.x & 31;
  const int sub = lane % G;
  const uint32_t r = lo + unit * (32u / G) + (uint32_t)(lane / G);
  const bool valid = r < hi;
  uint32_t b = 0, e = 0;
  double old = 0.0, div = 0.0;
  if (valid) {
    b = a.off[r];
    e = a.off[r + 1];
    if (sub == 0) {
      old = a.rank[cur][r];
      div = row_divisor(a, r);
    }
  }
  F2 acc = row_sum<G, kW, (G >= 32 ? kBatchWide : 4)>(a, sm, a.x[cur], b, e, sub);
  acc = group_sum<G>(acc);
  if (valid && sub == 0) finish_row(a, r, f2_value(acc), old, div, base, cur, f);
}

template <bool kW>
__device__ __forceinline__ void hub_unit(const PrArgs& a, const PrSmem& sm, uint32_t unit, int cur,
                                         int parity, double base) {
  const int lane = threadIdx.x & 31;
  const uint2 hu = a.hub_unit[unit];
  const uint32_t r = a.cls.lo[0] + hu.x;  // hub rows are the first rows
  const uint32_t rb = a.off[r], re = a.off[r + 1];
  const uint32_t eb = rb + hu.y * kHubChunk;
  const uint32_t ee = eb + kHubChunk < re ? eb + kHubChunk : re;
  F2 acc = row_sum<32, kW, kBatchHub>(a, sm, a.x[cur], eb, ee, lane);
  acc = group_sum<32>(acc);
  if (lane == 0) {
    const uint32_t nch = a.hub_nch[hu.x];
    bool finish = nch == 1;
    F2 row = acc;
    if (!finish) {
      a.chunk_part[unit] = acc;
      __threadfence();
      unsigned arrived = atomicAdd(&a.hub_cnt[hu.x], 1u);
      if (arrived == nch - 1) {
        __threadfence();
        finish = true;
        const uint32_t first = a.hub_first[hu.x];
        row = f2_zero();
        for (uint32_t k = 0; k < nch; k++) {
          F2 pk;
          pk.hi = __ldcg(&a.chunk_part[first + k].hi);
          pk.lo = __ldcg(&a.chunk_part[first + k].lo);
          row = f2_combine(row, pk);
        }
        a.hub_cnt[hu.x] = 0u;
      }
    }
    if (finish) {
      Fx g{0, 0};
      finish_row(a, r, f2_value(row), a.rank[cur][r], row_divisor(a, r), base, cur, g);
      a.hub_contrib[parity][hu.x] = make_ulonglong2(g.delta, g.dang);
    }
  }
}

template <bool kW>
__device__ __forceinline__ void run_unit(const PrArgs& a, const PrSmem& sm, uint32_t u, int cur,
                                         int parity, double base, Fx& f) {
  int c = 0;
#pragma unroll
  for (int k = 1; k < kClasses; k++)
    if (u >= a.cls.unit_begin[k]) c = k;
  const uint32_t unit = u - a.cls.unit_begin[c];
  const uint32_t lo = a.cls.lo[c], hi = a.cls.hi[c];
  switch (c) {
    case 0: hub_unit<kW>(a, sm, unit, cur, parity, base); break;
    case 1: class_unit<32, kW>(a, sm, lo, hi, unit, cur, base, f); break;
    case 2: class_unit<16, kW>(a, sm, lo, hi, unit, cur, base, f); break;
    case 3: class_unit<8, kW>(a, sm, lo, hi, unit, cur, base, f); break;
    case 4: class_unit<4, kW>(a, sm, lo, hi, unit, cur, base, f); break;
    case 5: class_unit<2, kW>(a, sm, lo, hi, unit, cur, base, f); break;
    default: class_unit<1, kW>(a, sm, lo, hi, unit, cur, base, f); break;
  }
}

// Block sum of the fixed-point accumulators; result valid in thread 0.
__device__ __forceinline__ Fx block_sum_fx(Fx v, ulonglong2* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.delta += __shfl_down_sync(0xffffffffu, v.delta, o);
    v.dang += __shfl_down_sync(0xffffffffu, v.dang, o);
  }
  __syncthreads();
  if (lane == 0) sh[w] = make_ulonglong2(v.delta, v.dang);
  __syncthreads();
  Fx r{0, 0};
  if (threadIdx.x == 0)
    for (int i = 0; i < kPrWarps; i++) {
      r.delta += sh[i].x;
      r.dang += sh[i].y;
    }
  return r;
}

// Bounded grid barrier whose last-arriving block sums the fixed-point
// partials of parity p (block partials and hub contributions; exact, so the
// result does not depend on which block arrives last or which warp did which
// unit), adds `extra` (the closed-form terms of the rows without in-edges)
// and publishes the totals; every block returns them.  A wait longer than
// kBarrierLimitNs sets the error flag and returns.
__device__ __forceinline__ Fin barrier_totals(const PrArgs& a, int p, PrSmem& sm, Fin extra) {
  __syncthreads();
  if (threadIdx.x == 0) {
    sm.gen = *(volatile unsigned*)a.bar_gen;
    __threadfence();
    sm.last = atomicAdd(a.bar_count, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (sm.last) {
    __threadfence();
    Fx acc{0, 0};
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kPrBlock) {
      const ulonglong2 v = __ldcg(&a.block_part[p][i]);
      acc.delta += v.x;
      acc.dang += v.y;
    }
    for (uint32_t i = threadIdx.x; i < a.n_hub; i += kPrBlock) {
      const ulonglong2 v = __ldcg(&a.hub_contrib[p][i]);
      acc.delta += v.x;
      acc.dang += v.y;
    }
    const Fx r = block_sum_fx(acc, sm.red);
    if (threadIdx.x == 0) {
      a.totals[p] = make_double2(__dadd_rn(fx64_value(r.delta), extra.delta),
                                 __dadd_rn(fx64_value(r.dang), extra.dang));
      __threadfence();
      atomicExch(a.bar_count, 0u);
      __threadfence();
      atomicAdd(a.bar_gen, 1u);
    }
  } else if (threadIdx.x == 0) {
    const uint64_t t0 = global_ns();
    while (*(volatile unsigned*)a.bar_gen == sm.gen) {
      __nanosleep(32);
      if (global_ns() - t0 > kBarrierLimitNs) {
        atomicExch(a.err, 1);
        break;
      }
      if (*(volatile int*)a.err) break;
    }
    __threadfence();
  }
  __syncthreads();
  const double2 t = __ldcg(&a.totals[p]);
  return Fin{t.x, t.y};
}

__device__ __forceinline__ void load_hot(const PrArgs& a, PrSmem& sm, int cur) {
  const float* __restrict__ x = a.x[cur];
  const uint32_t n4 = a.hot / 4;
  const float4* x4 = reinterpret_cast<const float4*>(x);
  float4* h4 = reinterpret_cast<float4*>(sm.hot);
#pragma unroll 4
  for (uint32_t i = threadIdx.x; i < n4; i += kPrBlock) h4[i] = __ldcg(x4 + i);
  for (uint32_t i = n4 * 4 + threadIdx.x; i < a.hot; i += kPrBlock) sm.hot[i] = __ldcg(x + i);
  __syncthreads();
}

// Sources without in-edges (rows [zi_lo, iso_lo)): their rank is `rank`
// (closed form, not stored per iteration); only the share they pass on is
// written, and a dangling one (weighted, all out-weights 0) adds its rank to
// the dangling mass.  A coalesced pass over all threads of the grid.
__device__ __forceinline__ void sources_without_in_edges(const PrArgs& a, double rank, int buf,
                                                         Fx& f) {
  for (uint64_t u = a.zi_lo + (uint64_t)blockIdx.x * kPrBlock + threadIdx.x; u < a.iso_lo;
       u += (uint64_t)gridDim.x * kPrBlock) {
    const double div = row_divisor(a, u);
    const bool dangling = !(div > 0.0);
    a.x[buf][u] = dangling ? 0.f : (float)(rank / div);
    if (dangling) f.dang += fx64_of(rank);
  }
}

template <bool kW>
__global__ void __launch_bounds__(kPrBlock, 1) pr_persistent_k(PrArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PrSmem& sm = *reinterpret_cast<PrSmem*>(smem_raw);
  const double nf = (double)a.n;
  const uint32_t gwarp = blockIdx.x * kPrWarps + (threadIdx.x >> 5);
  const uint32_t nwarps = gridDim.x * kPrWarps;
  const int lane = threadIdx.x & 31;
  // ---- prologue: rank_0 = 1/n, shares, dangling mass of rank_0
  {
    Fx f{0, 0};
    const double r0 = 1.0 / nf;
    for (uint32_t u = gwarp; u < a.n_units; u += nwarps) {
      int c = 0;
#pragma unroll
      for (int k = 1; k < kClasses; k++)
        if (u >= a.cls.unit_begin[k]) c = k;
      const uint32_t unit = u - a.cls.unit_begin[c];
      if (c == 0) {
        const uint2 hu = a.hub_unit[unit];
        if (hu.y == 0 && lane == 0) {
          Fx g{0, 0};
          init_row(a, a.cls.lo[0] + hu.x, r0, g);
          a.hub_contrib[0][hu.x] = make_ulonglong2(0ull, g.dang);
        }
      } else {
        const int G = 32 >> (c - 1);
        const uint32_t r = a.cls.lo[c] + unit * (32u / G) + (uint32_t)(lane / G);
        if (r < a.cls.hi[c] && lane % G == 0) init_row(a, r, r0, f);
      }
    }
    sources_without_in_edges(a, r0, 0, f);
    const Fx b = block_sum_fx(f, sm.red);
    if (threadIdx.x == 0) a.block_part[0][blockIdx.x] = make_ulonglong2(0ull, b.dang);
  }
  // rows without in-edges: next = base + d * 0 = base on every iteration
  // (1/n before the first), so their ranks follow in closed form; isolated
  // rows (no out-edges either) are dangling and are never gathered
  const double n_zi = (double)(a.n - a.zi_lo);
  const double n_iso = (double)(a.n - a.iso_lo);
  const double r0 = 1.0 / nf;
  Fin tot = barrier_totals(a, 0, sm, Fin{0.0, n_iso * r0});
  double dm = tot.dang;
  double prev_iso = r0;
  int cur = 0;
  uint32_t iters = 0;
  double delta = 0.0;
  for (uint32_t it = 0; it < a.max_iter; it++) {
    if (*(volatile int*)a.err) break;
    const int parity = (int)((it + 1) & 1u);
    // base = (1-d)/n + d*dangling_mass/n   (pagerank.rs:79)
    const double base = __dadd_rn(__ddiv_rn(1.0 - a.damping, nf),
                                  __ddiv_rn(__dmul_rn(a.damping, dm), nf));
    if (threadIdx.x == 0) sm.next = 0;
    load_hot(a, sm, cur);  // ends with a block barrier
    Fx f{0, 0};
    // blocks own interleaved units (u = block + k * grid); warps of a block
    // take kUnitsPerGrab of them at a time from the block's counter
    for (bool done = false; !done;) {
      uint32_t k = 0;
      if (lane == 0) k = atomicAdd(&sm.next, (unsigned)kUnitsPerGrab);
      k = __shfl_sync(0xffffffffu, k, 0);
      for (uint32_t q = 0; q < (uint32_t)kUnitsPerGrab; q++) {
        const uint32_t u = blockIdx.x + (k + q) * gridDim.x;
        if (u >= a.n_units) {
          done = true;
          break;
        }
        run_unit<kW>(a, sm, u, cur, parity, base, f);
      }
    }
    sources_without_in_edges(a, base, cur ^ 1, f);
    const Fx b = block_sum_fx(f, sm.red);
    if (threadIdx.x == 0) a.block_part[parity][blockIdx.x] = make_ulonglong2(b.delta, b.dang);
    tot = barrier_totals(a, parity, sm, Fin{n_zi * fabs(base - prev_iso), n_iso * base});
    prev_iso = base;
    delta = tot.delta;
    dm = tot.dang;
    cur ^= 1;
    iters++;
    if (delta < a.tol) break;  // every block sees the same delta
  }
  // rows without in-edges: the last iteration's base (1/n if none ran)
  for (uint64_t u = a.zi_lo + (uint64_t)blockIdx.x * kPrBlock + threadIdx.x; u < a.n;
       u += (uint64_t)gridDim.x * kPrBlock)
    a.rank[cur][u] = prev_iso;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *a.out_iters = iters;
    *a.out_delta = delta;
    *a.out_buf = (uint32_t)cur;
  }
}

// Weighted helpers: out-strength in out-CSR slot order (pagerank.rs:148-150,
// the same sequential order, so the f64 sums are bit-identical), relabelled,
// and the f32 weight of every execution-CSR slot.
__global__ void out_strength_new_k(const uint32_t* __restrict__ off,
                                   const uint32_t* __restrict__ eid, const double* __restrict__ w,
                                   const uint32_t* __restrict__ old_of_new, uint64_t n,
                                   double* __restrict__ out_str) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t u = old_of_new[i];
    double s = 0.0;
    for (uint32_t k = off[u]; k < off[u + 1]; k++) s += w[eid[k]];
    out_str[i] = s;
  }
}

__global__ void permute_w_f32_k(const uint32_t* __restrict__ eid, const double* __restrict__ w,
                                uint64_t m, float* __restrict__ out) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m;
       k += (uint64_t)gridDim.x * blockDim.x)
    out[k] = (float)w[eid[k]];
}

__global__ void unpermute_k(const double* __restrict__ rank_new,
                            const uint32_t* __restrict__ new_of_old, uint64_t n,
                            double* __restrict__ out) {
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x)
    out[u] = rank_new[new_of_old[u]];
}

size_t pr_smem_bytes() { return sizeof(PrSmem); }

}  // namespace

static PrPlan* build_pr_plan(TopoImpl* t, cudaStream_t s) {
  const uint64_t n = t->n, m = t->m;
  auto* plan = new PrPlan();
  // ---- relabel by in-degree, highest first (stable: ties keep id order)
  {
    Scratch<uint32_t> key(n, s), key_sorted(n, s);
    exec_order_key_k<<<grid_for(n), kBlock, 0, s>>>(t->in.off.get(), t->out.off.get(), n, key.get());
    UG_LAUNCH_CHECK();
    plan->old_of_new.alloc(n, s);
    radix_sort_pairs(key.get(), nullptr, n, 32, key_sorted.get(), plan->old_of_new.get(), nullptr,
                     nullptr, s);
  }
  plan->new_of_old.alloc(n, s);
  plan->outdeg.alloc(n, s);
  plan->off.alloc(n + 1, s);
  Scratch<uint32_t> deg(n + 1, s);
  relabel_maps_k<<<grid_for(n), kBlock, 0, s>>>(plan->old_of_new.get(), n, t->in.off.get(),
                                                 t->out.off.get(), plan->new_of_old.get(),
                                                 deg.get(), plan->outdeg.get());
  UG_LAUNCH_CHECK();
  UG_CUDA(cudaMemsetAsync(deg.get() + n, 0, sizeof(uint32_t), s));
  exclusive_scan_u32(deg.get(), plan->off.get(), n + 1, nullptr, s);
  plan->src.alloc(m ? m : 1, s);
  plan->eid.alloc(m ? m : 1, s);
  if (m) {
    relabel_copy_k<<<grid_for(m), kBlock, 0, s>>>(plan->off.get(), n, m, plan->old_of_new.get(),
                                                   plan->new_of_old.get(), t->in.off.get(),
                                                   t->in.tgt.get(), t->in.eid.get(),
                                                   plan->src.get(), plan->eid.get());
    UG_LAUNCH_CHECK();
  }
  // ---- degree classes (rows are sorted by degree, so each is a range)
  uint32_t bounds[kClasses + 1];
  {
    Scratch<uint32_t> db(kClasses + 1, s);
    class_bounds_k<<<1, 1, 0, s>>>(deg.get(), plan->outdeg.get(), n, db.get());
    UG_LAUNCH_CHECK();
    UG_CUDA(cudaMemcpyAsync(bounds, db.get(), sizeof(bounds), cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  }
  PrClassTable& c = plan->cls;
  c.lo[0] = 0;
  c.hi[0] = bounds[0];
  for (int k = 1; k < kClasses; k++) {
    c.lo[k] = bounds[k - 1];
    c.hi[k] = k < kClasses - 1 ? bounds[k] : bounds[kClasses];  // up to the rows without in-edges
  }
  plan->iso_lo = bounds[kClasses - 1];
  plan->zi_lo = bounds[kClasses];
  plan->n_hub = c.hi[0];
  // hub chunks
  plan->hub_nch.alloc(plan->n_hub ? plan->n_hub : 1, s);
  plan->hub_first.alloc(plan->n_hub ? plan->n_hub : 1, s);
  uint32_t n_chunks = 0;
  if (plan->n_hub) {
    Scratch<uint32_t> tot(1, s);
    hub_nch_k<<<grid_for(plan->n_hub), kBlock, 0, s>>>(deg.get(), plan->n_hub, plan->hub_nch.get());
    UG_LAUNCH_CHECK();
    exclusive_scan_u32(plan->hub_nch.get(), plan->hub_first.get(), plan->n_hub, tot.get(), s);
    UG_CUDA(cudaMemcpyAsync(&n_chunks, tot.get(), 4, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  }
  plan->n_chunks = n_chunks;
  plan->hub_unit.alloc(n_chunks ? n_chunks : 1, s);
  if (n_chunks) {
    hub_units_k<<<grid_for(plan->n_hub), kBlock, 0, s>>>(plan->hub_first.get(), plan->hub_nch.get(),
                                                         plan->n_hub, plan->hub_unit.get());
    UG_LAUNCH_CHECK();
  }
  c.unit_begin[0] = 0;
  c.unit_begin[1] = n_chunks;
  for (int k = 1; k < kClasses; k++) {
    const uint32_t G = 32u >> (k - 1), rpu = 32u / G;
    c.unit_begin[k + 1] = c.unit_begin[k] + (c.hi[k] - c.lo[k] + rpu - 1) / rpu;
  }
  plan->n_units = c.unit_begin[kClasses];
  UG_CUDA(cudaStreamSynchronize(s));
  return plan;
}

static PrPlan* ensure_pr_plan(TopoImpl* t, cudaStream_t s) {
  ensure_in(t, s);
  std::lock_guard<std::mutex> g(t->mu);
  if (!t->pr_plan) t->pr_plan = build_pr_plan(t, s);
  return t->pr_plan;
}

template <bool kW>
static int pr_grid(int device) {
  static std::mutex mu;
  static int cached[64] = {0};
  std::lock_guard<std::mutex> g(mu);
  if (device < 0 || device >= 64) device = 0;
  if (!cached[device]) {
    const int smem = (int)pr_smem_bytes();
    UG_CUDA(cudaFuncSetAttribute(pr_persistent_k<kW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smem));
    int per_sm = 0;
    UG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pr_persistent_k<kW>, kPrBlock,
                                                          smem));
    UG_CHECK(per_sm > 0, URSA_GPU_ECUDA, "pagerank kernel cannot be resident");
    cached[device] = per_sm * sm_count(device);
  }
  return cached[device];
}

// Runs the iteration; the final ranks (caller's ids) are left in d_out
// (device).  d_weights (device, by edge row) selects the weighted variant.
void pagerank_run(TopoImpl* t, const ursa_gpu_pagerank_params& p, const double* d_weights,
                  double* d_out, cudaStream_t s, ursa_gpu_pagerank_stats* stats) {
  const uint64_t n = t->n, m = t->m;
  if (stats) *stats = ursa_gpu_pagerank_stats{0, 0.0, 0.0};
  if (n == 0) return;
  PrPlan* plan = ensure_pr_plan(t, s);
  const bool weighted = d_weights != nullptr;
  const int G = weighted ? pr_grid<true>(t->device) : pr_grid<false>(t->device);
  const size_t smem = pr_smem_bytes();
  const uint32_t nh = plan->n_hub ? plan->n_hub : 1;

  Scratch<double> rank(2 * n, s);
  const uint64_t n_pad = (n + 3) & ~3ull;  // both share buffers 16-byte aligned
  Scratch<float> x(2 * n_pad, s);
  Scratch<F2> chunk_part(plan->n_chunks ? plan->n_chunks : 1, s);
  Scratch<unsigned> hub_cnt(nh, s);
  Scratch<ulonglong2> hub_contrib(2 * (size_t)nh, s);
  Scratch<ulonglong2> block_part(2 * (size_t)G, s);
  Scratch<double2> totals(2, s);
  Scratch<unsigned> ctl(8, s);  // bar_count, bar_gen, err, iters, buf
  Scratch<double> ctl_d(1, s);
  UG_CUDA(cudaMemsetAsync(hub_cnt.get(), 0, nh * sizeof(unsigned), s));
  UG_CUDA(cudaMemsetAsync(hub_contrib.get(), 0, 2 * (size_t)nh * sizeof(ulonglong2), s));
  UG_CUDA(cudaMemsetAsync(ctl.get(), 0, 8 * sizeof(unsigned), s));

  Scratch<double> out_str;
  Scratch<float> w_new;
  if (weighted) {
    out_str.alloc(n, s);
    out_strength_new_k<<<grid_for(n), kBlock, 0, s>>>(t->out.off.get(), t->out.eid.get(),
                                                       d_weights, plan->old_of_new.get(), n,
                                                       out_str.get());
    UG_LAUNCH_CHECK();
    w_new.alloc(m ? m : 1, s);
    if (m) {
      permute_w_f32_k<<<grid_for(m), kBlock, 0, s>>>(plan->eid.get(), d_weights, m, w_new.get());
      UG_LAUNCH_CHECK();
    }
  }

  PrArgs a;
  a.n = n;
  a.hot = (uint32_t)(n < (uint64_t)kHot ? n : (uint64_t)kHot);
  a.cls = plan->cls;
  a.n_units = plan->n_units;
  a.off = plan->off.get();
  a.src = plan->src.get();
  a.w = weighted ? w_new.get() : nullptr;
  a.outdeg = plan->outdeg.get();
  a.out_str = weighted ? out_str.get() : nullptr;
  a.rank[0] = rank.get();
  a.rank[1] = rank.get() + n;
  a.x[0] = x.get();
  a.x[1] = x.get() + n_pad;
  a.hub_unit = plan->hub_unit.get();
  a.hub_first = plan->hub_first.get();
  a.hub_nch = plan->hub_nch.get();
  a.n_hub = plan->n_hub;
  a.chunk_part = chunk_part.get();
  a.hub_cnt = hub_cnt.get();
  a.hub_contrib[0] = hub_contrib.get();
  a.hub_contrib[1] = hub_contrib.get() + nh;
  a.block_part[0] = block_part.get();
  a.block_part[1] = block_part.get() + G;
  a.totals = totals.get();
  a.iso_lo = plan->iso_lo;
  a.zi_lo = plan->zi_lo;
  a.bar_count = ctl.get() + 0;
  a.bar_gen = ctl.get() + 1;
  a.err = (int*)(ctl.get() + 2);
  a.out_iters = ctl.get() + 3;
  a.out_buf = ctl.get() + 4;
  a.out_delta = ctl_d.get();
  a.damping = p.damping;
  a.tol = p.tol;
  a.max_iter = p.max_iter;

  cudaEvent_t e0, e1;
  UG_CUDA(cudaEventCreate(&e0));
  UG_CUDA(cudaEventCreate(&e1));
  UG_CUDA(cudaEventRecord(e0, s));
  void* args[] = {&a};
  void* fn = weighted ? (void*)pr_persistent_k<true> : (void*)pr_persistent_k<false>;
  UG_CUDA(cudaLaunchCooperativeKernel(fn, dim3(G), dim3(kPrBlock), args, smem, s));
  count_launch();
  UG_CUDA(cudaEventRecord(e1, s));
  unsigned h[8];
  double hd;
  UG_CUDA(cudaMemcpyAsync(h, ctl.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaMemcpyAsync(&hd, ctl_d.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  UG_CHECK(h[2] == 0, URSA_GPU_ETIMEOUT, "pagerank: a grid barrier wait expired");
  const uint32_t buf = p.max_iter == 0 ? 0u : h[4];
  unpermute_k<<<grid_for(n), kBlock, 0, s>>>(rank.get() + (size_t)buf * n, plan->new_of_old.get(),
                                             n, d_out);
  UG_LAUNCH_CHECK();
  if (stats) {
    stats->iterations = h[3];
    stats->last_delta = hd;
    stats->device_ms = ms;
  }
}

}  // namespace ug
