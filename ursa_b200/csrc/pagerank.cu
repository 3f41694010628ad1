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
// B200 design.  The in-CSR streams from HBM once per iteration; everything
// else is per-node.  The per-edge share x[v] = rank[v]/outdeg[v] is stored as
// f32 (4n bytes, L2-resident at R-MAT-22 scale) and gathered per in-edge; each
// row is summed with compensated f32 (TwoSum) accumulation, then the update,
// residual and dangling mass are computed in f64.
//
// Work partition (built once per topology and cached): rows with in-degree
// <= kLong are grouped into row-aligned tiles of about kTile merge items
// (edges + rows); rows above kLong ("hubs") are split into kChunk-edge chunks.
// Inside a tile, the tile's shares are staged in shared memory and each
// thread walks an equal slice of the (row-end, edge) merge path; rows that
// cross thread slices are stitched by a block segmented scan.  A hub's chunk
// partials are combined in chunk order by whichever chunk arrives last (an
// arrival counter, no waiting).  One bounded grid barrier per iteration; all
// reductions use fixed orders, so a run is bit-reproducible.
#include <cmath>

#include "primitives.cuh"
#include "topo.cuh"

namespace ug {

namespace {
constexpr int kTile = 2048;   // merge items per short-row tile (before the last row)
constexpr int kLong = 1024;   // in-degree above which a row is a hub
constexpr int kChunk = 2048;  // edges per hub chunk
constexpr int kECap = kTile + kLong;
constexpr int kRCap = kTile;
constexpr uint32_t kLongFlag = 0x80000000u;
constexpr int kPrBlock = 256;
constexpr int kPrWarps = kPrBlock / 32;
constexpr uint64_t kBarrierLimitNs = 5000000000ull;  // 5 s per grid barrier wait
}  // namespace

struct PrPlan {
  uint32_t n_work = 0, n_long = 0;
  DevArray<uint2> work;  // short tile: {r0, r1}; hub chunk: {long index, chunk | kLongFlag}
  DevArray<uint32_t> long_row, long_first, long_nch;
};

void pr_plan_free(PrPlan* p) { delete p; }
uint64_t pr_plan_bytes(const PrPlan* p) {
  return p ? (uint64_t)p->work.n * sizeof(uint2) + 3ull * p->long_row.n * sizeof(uint32_t) : 0;
}

namespace {

// ------------------------------------------------------------ plan kernels
__global__ void plan_w_k(const uint32_t* __restrict__ off, uint64_t n, uint64_t* __restrict__ w) {
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t deg = off[u + 1] - off[u];
    w[u] = deg > (uint32_t)kLong ? 0ull : (uint64_t)deg + 1ull;
  }
}

__global__ void plan_flags_k(const uint32_t* __restrict__ off, uint64_t n,
                             const uint64_t* __restrict__ W, uint32_t* __restrict__ brk,
                             uint32_t* __restrict__ cnt, uint32_t* __restrict__ lng) {
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t deg = off[u + 1] - off[u];
    bool is_long = deg > (uint32_t)kLong;
    bool prev_long = u > 0 && (off[u] - off[u - 1]) > (uint32_t)kLong;
    bool start = !is_long && (u == 0 || prev_long || (W[u] / kTile) != (W[u - 1] / kTile));
    brk[u] = (start || is_long) ? 1u : 0u;
    cnt[u] = start ? 1u : (is_long ? (deg + kChunk - 1) / kChunk : 0u);
    lng[u] = is_long ? 1u : 0u;
  }
}

__global__ void plan_breaks_k(uint64_t n, const uint32_t* __restrict__ brk,
                              const uint32_t* __restrict__ bpos, uint32_t* __restrict__ B) {
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x)
    if (brk[u]) B[bpos[u]] = (uint32_t)u;
}

__global__ void plan_fill_k(uint64_t n, const uint32_t* __restrict__ brk,
                            const uint32_t* __restrict__ bpos, const uint32_t* __restrict__ B,
                            const uint32_t* __restrict__ cnt, const uint32_t* __restrict__ wpos,
                            const uint32_t* __restrict__ lng, const uint32_t* __restrict__ lpos,
                            uint2* __restrict__ work, uint32_t* __restrict__ long_row,
                            uint32_t* __restrict__ long_first, uint32_t* __restrict__ long_nch) {
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    if (!brk[u]) continue;
    uint32_t wp = wpos[u];
    if (lng[u]) {
      uint32_t li = lpos[u], nch = cnt[u];
      long_row[li] = (uint32_t)u;
      long_first[li] = wp;
      long_nch[li] = nch;
      for (uint32_t c = 0; c < nch; c++) work[wp + c] = make_uint2(li, c | kLongFlag);
    } else {
      work[wp] = make_uint2((uint32_t)u, B[bpos[u] + 1]);
    }
  }
}

__global__ void set_u32_k(uint32_t* p, uint32_t v) { *p = v; }

// ---------------------------------------------------------- iteration kernel
struct PrArgs {
  uint64_t n;
  const uint32_t* __restrict__ off;  // in-CSR offsets
  const uint32_t* __restrict__ src;  // in-CSR neighbours (edge sources)
  const uint32_t* __restrict__ outdeg;   // unweighted
  const double* __restrict__ out_str;    // weighted (nullptr if unweighted)
  const float* __restrict__ w_in;        // weighted: f32 weight per in-CSR slot
  double* rank[2];
  float* x[2];
  const uint2* __restrict__ work;
  uint32_t n_work;
  const uint32_t* __restrict__ long_row;
  const uint32_t* __restrict__ long_first;
  const uint32_t* __restrict__ long_nch;
  uint32_t n_long;
  F2* chunk_part;         // per work item (hub chunks)
  unsigned* long_cnt;     // per hub: chunk arrivals this iteration
  double2* long_contrib[2];  // per hub: (|next-rank|, dangling next)
  double2* block_part[2];    // per block
  unsigned* bar_count;
  unsigned* bar_gen;
  int* err;
  double damping;
  double tol;
  uint32_t max_iter;
  // outputs
  uint32_t* out_iters;
  double* out_delta;
  uint32_t* out_buf;
};

struct Fin {
  double delta, dang;
};

__device__ __forceinline__ void finalize_row(const PrArgs& a, uint64_t u, double sum, double base,
                                             int cur, Fin& f) {
  // next[u] = base + d * contrib(u)   (pagerank.rs:81-83)
  double nx = __dadd_rn(base, __dmul_rn(a.damping, sum));
  double old = a.rank[cur][u];
  f.delta += fabs(nx - old);
  a.rank[cur ^ 1][u] = nx;
  bool dangling;
  float share;
  if (a.out_str) {
    double os = a.out_str[u];
    dangling = !(os > 0.0);
    share = dangling ? 0.f : (float)(nx / os);
  } else {
    uint32_t od = a.outdeg[u];
    dangling = od == 0;
    share = dangling ? 0.f : (float)(nx / (double)od);
  }
  a.x[cur ^ 1][u] = share;
  if (dangling) f.dang += nx;
}

__device__ __forceinline__ void init_row(const PrArgs& a, uint64_t u, double r0, Fin& f) {
  a.rank[0][u] = r0;
  bool dangling;
  float share;
  if (a.out_str) {
    double os = a.out_str[u];
    dangling = !(os > 0.0);
    share = dangling ? 0.f : (float)(r0 / os);
  } else {
    uint32_t od = a.outdeg[u];
    dangling = od == 0;
    share = dangling ? 0.f : (float)(r0 / (double)od);
  }
  a.x[0][u] = share;
  if (dangling) f.dang += r0;
}

// Fixed-order block reduction of two doubles; result valid in thread 0.
__device__ __forceinline__ Fin block_sum_fin(Fin v, double2* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.delta += __shfl_down_sync(0xffffffffu, v.delta, o);
    v.dang += __shfl_down_sync(0xffffffffu, v.dang, o);
  }
  __syncthreads();
  if (lane == 0) sh[w] = make_double2(v.delta, v.dang);
  __syncthreads();
  Fin r{0.0, 0.0};
  if (threadIdx.x == 0)
    for (int i = 0; i < kPrWarps; i++) {
      r.delta += sh[i].x;
      r.dang += sh[i].y;
    }
  return r;
}

// Fixed-order block reduction of an F2; result valid in thread 0.
__device__ __forceinline__ F2 block_sum_f2(F2 v, F2* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    F2 o2{__shfl_down_sync(0xffffffffu, v.hi, o), __shfl_down_sync(0xffffffffu, v.lo, o)};
    v = f2_combine(v, o2);
  }
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  F2 r = f2_zero();
  if (threadIdx.x == 0)
    for (int i = 0; i < kPrWarps; i++) r = f2_combine(r, sh[i]);
  return r;
}

// Every block computes the same totals from the same partials in the same
// order (warp 0, lane-strided, then a fixed shuffle tree).
__device__ __forceinline__ Fin global_totals(const PrArgs& a, int p, double2* sh) {
  if (threadIdx.x < 32) {
    double d = 0.0, g = 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += 32) {
      double2 v = __ldcg(&a.block_part[p][i]);
      d += v.x;
      g += v.y;
    }
    for (uint32_t i = threadIdx.x; i < a.n_long; i += 32) {
      double2 v = __ldcg(&a.long_contrib[p][i]);
      d += v.x;
      g += v.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      d += __shfl_down_sync(0xffffffffu, d, o);
      g += __shfl_down_sync(0xffffffffu, g, o);
    }
    if (threadIdx.x == 0) sh[0] = make_double2(d, g);
  }
  __syncthreads();
  Fin r{sh[0].x, sh[0].y};
  __syncthreads();
  return r;
}

__device__ __forceinline__ void merge_path(int diag, const uint32_t* s_end, int R, int E, int& i,
                                           int& j) {
  int lo = diag - E > 0 ? diag - E : 0;
  int hi = diag < R ? diag : R;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if ((int)s_end[mid] <= diag - mid - 1)
      lo = mid + 1;
    else
      hi = mid;
  }
  i = lo;
  j = diag - lo;
}

struct TileSmem {
  float val[kECap];
  uint32_t end[kRCap];
  uint32_t wkey[kPrWarps];
  F2 wval[kPrWarps];
  F2 f2sh[kPrWarps];
  double2 dsh[kPrWarps];
};

__device__ void short_tile(const PrArgs& a, uint32_t r0, uint32_t r1, int cur, double base,
                           TileSmem& sm, Fin& f) {
  const uint32_t e0 = a.off[r0];
  const int R = (int)(r1 - r0);
  const int E = (int)(a.off[r1] - e0);
  const float* __restrict__ x = a.x[cur];
  // stage the tile's shares and row ends
  for (int j = threadIdx.x; j < E; j += kPrBlock) {
    uint32_t v = a.src[e0 + j];
    float s = x[v];
    if (a.w_in) s = __fmul_rn(s, a.w_in[e0 + j]);
    sm.val[j] = s;
  }
  for (int i = threadIdx.x; i < R; i += kPrBlock) sm.end[i] = a.off[r0 + i + 1] - e0;
  __syncthreads();
  const int items = R + E;
  const int ipt = (items + kPrBlock - 1) / kPrBlock;
  int d0 = threadIdx.x * ipt;
  if (d0 > items) d0 = items;
  int d1 = d0 + ipt;
  if (d1 > items) d1 = items;
  int i, j;
  merge_path(d0, sm.end, R, E, i, j);
  const int first_row = i;
  bool ended_first = false;
  F2 first_acc = f2_zero();
  F2 acc = f2_zero();
  for (int d = d0; d < d1; d++) {
    if (j < (int)sm.end[i]) {  // i < R whenever d < items
      acc = f2_add(acc, sm.val[j]);
      j++;
    } else {
      if (!ended_first) {
        ended_first = true;
        first_acc = acc;
      } else {
        finalize_row(a, (uint64_t)r0 + i, f2_value(acc), base, cur, f);
      }
      acc = f2_zero();
      i++;
    }
  }
  // Segmented inclusive scan of (open row, partial) over threads.
  uint32_t key = (uint32_t)i;  // row still open at the end of the slice (R = none)
  F2 val = acc;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t k2 = __shfl_up_sync(0xffffffffu, key, o);
    F2 v2{__shfl_up_sync(0xffffffffu, val.hi, o), __shfl_up_sync(0xffffffffu, val.lo, o)};
    if (lane >= o && k2 == key) val = f2_combine(v2, val);
  }
  if (lane == 31) {
    sm.wkey[w] = key;
    sm.wval[w] = val;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int ww = 1; ww < kPrWarps; ww++)
      if (sm.wkey[ww] == sm.wkey[ww - 1]) sm.wval[ww] = f2_combine(sm.wval[ww - 1], sm.wval[ww]);
  }
  __syncthreads();
  if (w > 0 && sm.wkey[w - 1] == key) val = f2_combine(sm.wval[w - 1], val);
  // carry into this thread = inclusive value of thread t-1 (same key by construction)
  uint32_t pk = __shfl_up_sync(0xffffffffu, key, 1);
  F2 pv{__shfl_up_sync(0xffffffffu, val.hi, 1), __shfl_up_sync(0xffffffffu, val.lo, 1)};
  if (lane == 0) {
    if (w > 0) {
      pk = sm.wkey[w - 1];
      pv = sm.wval[w - 1];
    } else {
      pk = 0xffffffffu;
    }
  }
  if (ended_first) {
    F2 tot = first_acc;
    if (threadIdx.x > 0 && pk == (uint32_t)first_row) tot = f2_combine(pv, first_acc);
    finalize_row(a, (uint64_t)r0 + first_row, f2_value(tot), base, cur, f);
  }
  __syncthreads();  // smem reuse by the next tile
}

__device__ void hub_chunk(const PrArgs& a, uint32_t li, uint32_t c, uint32_t work_id, int cur,
                          int parity, double base, TileSmem& sm) {
  const uint32_t u = a.long_row[li];
  const uint32_t rb = a.off[u], re = a.off[u + 1];
  const uint32_t eb = rb + c * (uint32_t)kChunk;
  const uint32_t ee = eb + (uint32_t)kChunk < re ? eb + (uint32_t)kChunk : re;
  const float* __restrict__ x = a.x[cur];
  F2 acc = f2_zero();
  for (uint32_t e = eb + threadIdx.x; e < ee; e += kPrBlock) {
    float s = x[a.src[e]];
    if (a.w_in) s = __fmul_rn(s, a.w_in[e]);
    acc = f2_add(acc, s);
  }
  F2 tot = block_sum_f2(acc, sm.f2sh);
  if (threadIdx.x == 0) {
    a.chunk_part[work_id] = tot;
    __threadfence();
    unsigned arrived = atomicAdd(&a.long_cnt[li], 1u);
    if (arrived == a.long_nch[li] - 1) {
      __threadfence();
      uint32_t first = a.long_first[li], nch = a.long_nch[li];
      F2 row = f2_zero();
      for (uint32_t k = 0; k < nch; k++) {
        F2 pk;
        pk.hi = __ldcg(&a.chunk_part[first + k].hi);
        pk.lo = __ldcg(&a.chunk_part[first + k].lo);
        row = f2_combine(row, pk);
      }
      Fin f{0.0, 0.0};
      finalize_row(a, u, f2_value(row), base, cur, f);
      a.long_contrib[parity][li] = make_double2(f.delta, f.dang);
      a.long_cnt[li] = 0u;
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kPrBlock, 2) pr_persistent_k(PrArgs a) {
  __shared__ TileSmem sm;
  const double nf = (double)a.n;
  // ---- prologue: rank_0 = 1/n, shares, dangling mass of rank_0
  {
    Fin f{0.0, 0.0};
    const double r0 = 1.0 / nf;
    for (uint32_t wi = blockIdx.x; wi < a.n_work; wi += gridDim.x) {
      uint2 it = a.work[wi];
      if (it.y & kLongFlag) {
        if ((it.y & ~kLongFlag) == 0 && threadIdx.x == 0) {
          Fin g{0.0, 0.0};
          init_row(a, a.long_row[it.x], r0, g);
          a.long_contrib[0][it.x] = make_double2(0.0, g.dang);
        }
      } else {
        for (uint32_t u = it.x + threadIdx.x; u < it.y; u += kPrBlock) init_row(a, u, r0, f);
      }
    }
    Fin b = block_sum_fin(f, sm.dsh);
    if (threadIdx.x == 0) a.block_part[0][blockIdx.x] = make_double2(0.0, b.dang);
  }
  grid_barrier(a.bar_count, a.bar_gen, gridDim.x, a.err, kBarrierLimitNs);
  Fin tot = global_totals(a, 0, sm.dsh);
  double dm = tot.dang;
  int cur = 0;
  uint32_t iters = 0;
  double delta = 0.0;
  for (uint32_t it = 0; it < a.max_iter; it++) {
    if (*(volatile int*)a.err) break;
    const int parity = (int)((it + 1) & 1u);
    // base = (1-d)/n + d*dangling_mass/n   (pagerank.rs:79)
    const double base = __dadd_rn(__ddiv_rn(1.0 - a.damping, nf),
                                  __ddiv_rn(__dmul_rn(a.damping, dm), nf));
    Fin f{0.0, 0.0};
    for (uint32_t wi = blockIdx.x; wi < a.n_work; wi += gridDim.x) {
      uint2 w = a.work[wi];
      if (w.y & kLongFlag)
        hub_chunk(a, w.x, w.y & ~kLongFlag, wi, cur, parity, base, sm);
      else
        short_tile(a, w.x, w.y, cur, base, sm, f);
    }
    Fin b = block_sum_fin(f, sm.dsh);
    if (threadIdx.x == 0) a.block_part[parity][blockIdx.x] = make_double2(b.delta, b.dang);
    grid_barrier(a.bar_count, a.bar_gen, gridDim.x, a.err, kBarrierLimitNs);
    tot = global_totals(a, parity, sm.dsh);
    delta = tot.delta;
    dm = tot.dang;
    cur ^= 1;
    iters++;
    if (delta < a.tol) break;  // every block sees the same delta
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *a.out_iters = iters;
    *a.out_delta = delta;
    *a.out_buf = (uint32_t)cur;
  }
}

// Weighted helpers: out-strength in out-CSR slot order (pagerank.rs:148-150,
// the same sequential order, so the f64 sums are bit-identical), and the
// f32 weight of every in-CSR slot.
__global__ void out_strength_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ eid,
                               const double* __restrict__ w, uint64_t n,
                               double* __restrict__ out_str) {
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (uint32_t k = off[u]; k < off[u + 1]; k++) s += w[eid[k]];
    out_str[u] = s;
  }
}

__global__ void permute_w_f32_k(const uint32_t* __restrict__ eid, const double* __restrict__ w,
                                uint64_t m, float* __restrict__ out) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m;
       k += (uint64_t)gridDim.x * blockDim.x)
    out[k] = (float)w[eid[k]];
}

}  // namespace

static PrPlan* build_pr_plan(TopoImpl* t, cudaStream_t s) {
  const uint64_t n = t->n;
  const uint32_t* off = t->in.off.get();
  auto* plan = new PrPlan();
  Scratch<uint64_t> W(n, s);
  Scratch<uint32_t> brk(n, s), cnt(n, s), lng(n, s), bpos(n, s), wpos(n, s), lpos(n, s);
  Scratch<uint32_t> tots(3, s);
  plan_w_k<<<grid_for(n), kBlock, 0, s>>>(off, n, W.get());
  UG_LAUNCH_CHECK();
  exclusive_scan_u64(W.get(), W.get(), n, nullptr, s);
  plan_flags_k<<<grid_for(n), kBlock, 0, s>>>(off, n, W.get(), brk.get(), cnt.get(), lng.get());
  UG_LAUNCH_CHECK();
  exclusive_scan_u32(brk.get(), bpos.get(), n, tots.get() + 0, s);
  exclusive_scan_u32(cnt.get(), wpos.get(), n, tots.get() + 1, s);
  exclusive_scan_u32(lng.get(), lpos.get(), n, tots.get() + 2, s);
  uint32_t h[3];
  UG_CUDA(cudaMemcpyAsync(h, tots.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  const uint32_t nb = h[0];
  plan->n_work = h[1];
  plan->n_long = h[2];
  Scratch<uint32_t> B((size_t)nb + 1, s);
  plan_breaks_k<<<grid_for(n), kBlock, 0, s>>>(n, brk.get(), bpos.get(), B.get());
  UG_LAUNCH_CHECK();
  set_u32_k<<<1, 1, 0, s>>>(B.get() + nb, (uint32_t)n);
  UG_LAUNCH_CHECK();
  plan->work.alloc(plan->n_work);
  plan->long_row.alloc(plan->n_long);
  plan->long_first.alloc(plan->n_long);
  plan->long_nch.alloc(plan->n_long);
  plan_fill_k<<<grid_for(n), kBlock, 0, s>>>(n, brk.get(), bpos.get(), B.get(), cnt.get(),
                                             wpos.get(), lng.get(), lpos.get(), plan->work.get(),
                                             plan->long_row.get(), plan->long_first.get(),
                                             plan->long_nch.get());
  UG_LAUNCH_CHECK();
  UG_CUDA(cudaStreamSynchronize(s));
  return plan;
}

static PrPlan* ensure_pr_plan(TopoImpl* t, cudaStream_t s) {
  ensure_in(t, s);
  ensure_outdeg(t, s);
  std::lock_guard<std::mutex> g(t->mu);
  if (!t->pr_plan) t->pr_plan = build_pr_plan(t, s);
  return t->pr_plan;
}

static int pr_grid(int device) {
  static std::mutex mu;
  static int cached[64] = {0};
  std::lock_guard<std::mutex> g(mu);
  if (device < 0 || device >= 64) device = 0;
  if (!cached[device]) {
    int per_sm = 0;
    UG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pr_persistent_k, kPrBlock, 0));
    UG_CHECK(per_sm > 0, URSA_GPU_ECUDA, "pagerank kernel cannot be resident");
    cached[device] = per_sm * sm_count(device);
  }
  return cached[device];
}

// Runs the iteration; the final ranks are left in d_out (device). Returns
// stats. `weights` (device, by edge row) selects the weighted variant.
void pagerank_run(TopoImpl* t, const ursa_gpu_pagerank_params& p, const double* d_weights,
                  double* d_out, cudaStream_t s, ursa_gpu_pagerank_stats* stats) {
  const uint64_t n = t->n;
  if (stats) *stats = ursa_gpu_pagerank_stats{0, 0.0, 0.0};
  if (n == 0) return;
  PrPlan* plan = ensure_pr_plan(t, s);
  const int G = pr_grid(t->device);

  Scratch<double> rank(2 * n, s);
  Scratch<float> x(2 * n, s);
  Scratch<F2> chunk_part(plan->n_work ? plan->n_work : 1, s);
  Scratch<unsigned> long_cnt(plan->n_long ? plan->n_long : 1, s);
  Scratch<double2> long_contrib(2 * (size_t)(plan->n_long ? plan->n_long : 1), s);
  Scratch<double2> block_part(2 * (size_t)G, s);
  // control block: bar_count, bar_gen, err, iters, buf | delta
  Scratch<unsigned> ctl(8, s);
  Scratch<double> ctl_d(1, s);
  UG_CUDA(cudaMemsetAsync(long_cnt.get(), 0, long_cnt.n * sizeof(unsigned), s));
  UG_CUDA(cudaMemsetAsync(long_contrib.get(), 0, long_contrib.n * sizeof(double2), s));
  UG_CUDA(cudaMemsetAsync(ctl.get(), 0, 8 * sizeof(unsigned), s));

  Scratch<double> out_str;
  Scratch<float> w_in;
  if (d_weights) {
    out_str.alloc(n, s);
    out_strength_k<<<grid_for(n), kBlock, 0, s>>>(t->out.off.get(), t->out.eid.get(), d_weights,
                                                   n, out_str.get());
    UG_LAUNCH_CHECK();
    w_in.alloc(t->m ? t->m : 1, s);
    if (t->m) {
      permute_w_f32_k<<<grid_for(t->m), kBlock, 0, s>>>(t->in.eid.get(), d_weights, t->m,
                                                         w_in.get());
      UG_LAUNCH_CHECK();
    }
  }

  PrArgs a;
  a.n = n;
  a.off = t->in.off.get();
  a.src = t->in.tgt.get();
  a.outdeg = t->outdeg.get();
  a.out_str = d_weights ? out_str.get() : nullptr;
  a.w_in = d_weights ? w_in.get() : nullptr;
  a.rank[0] = rank.get();
  a.rank[1] = rank.get() + n;
  a.x[0] = x.get();
  a.x[1] = x.get() + n;
  a.work = plan->work.get();
  a.n_work = plan->n_work;
  a.long_row = plan->long_row.get();
  a.long_first = plan->long_first.get();
  a.long_nch = plan->long_nch.get();
  a.n_long = plan->n_long;
  a.chunk_part = chunk_part.get();
  a.long_cnt = long_cnt.get();
  a.long_contrib[0] = long_contrib.get();
  a.long_contrib[1] = long_contrib.get() + (plan->n_long ? plan->n_long : 1);
  a.block_part[0] = block_part.get();
  a.block_part[1] = block_part.get() + G;
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
  UG_CUDA(cudaLaunchCooperativeKernel((void*)pr_persistent_k, dim3(G), dim3(kPrBlock), args, 0, s));
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
  UG_CUDA(cudaMemcpyAsync(d_out, rank.get() + (size_t)buf * n, n * sizeof(double),
                          cudaMemcpyDeviceToDevice, s));
  if (stats) {
    stats->iterations = h[3];
    stats->last_delta = hd;
    stats->device_ms = ms;
  }
}

}  // namespace ug
