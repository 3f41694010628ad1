// bc.cu -- Brandes betweenness (ursa-core/src/algo/betweenness.rs, rng.rs).
//
// Sources: all nodes, or the reference's seeded sample -- the first
// ceil(frac * n) entries of a SplitMix64 Fisher-Yates shuffle
// (betweenness.rs:349-362, rng.rs:12-72) -- computed on the host, so the
// device uses exactly the reference's source set for a given seed.
//
// Per source, on the device:
//  * unweighted (brandes_from, :185-230): level-synchronous BFS over the
//    out-CSR; sigma[w] += sigma[v] for every CSR slot v->w with
//    dist[w] = dist[v] + 1 (parallel edges count, as in the reference), as f64
//    atomics -- shortest-path counts are integers, exact below 2^53, so the
//    order of those additions does not matter;
//  * weighted (brandes_from_weighted, :278-339): Dijkstra-equivalent f64
//    distances (frontier Bellman-Ford), then the tight-edge DAG
//    (fl(dist[u] + w) == dist[v], exact equality as the reference's tie rule)
//    is walked in Kahn order to accumulate sigma;
//  * reverse accumulation (reverse_accumulate, :81-98): levels in reverse,
//    one warp per node sums sigma[v] * ((1 + delta[w]) / sigma[w]) over its
//    DAG successors with a fixed-order reduction, then bc += delta (source
//    excluded).
// Sources go in 64-source chunks whose partial vectors are added in chunk
// order, and sampled results are scaled by n / k (accumulate_sources,
// :45-70; :171-176).  The dependency sums run in a different order than the
// reference's predecessor lists, so results agree to f64 rounding.
#include <algorithm>
#include <cmath>
#include <vector>

#include "frontier.cuh"

namespace ug {

void sssp_run(const DirView& d, const double* w0, const double* w1, uint64_t n, uint32_t source,
              unsigned long long* dist, cudaStream_t s);

namespace {

constexpr unsigned long long kInfBits = 0x7FF0000000000000ull;
constexpr uint32_t kSrcChunk = 64;  // betweenness.rs:51
constexpr bool kBatchedWeighted = true;  // weighted sources 64 at a time (else one by one)

// ---------------------------------------------------------------- rng.rs
constexpr uint64_t kDefaultSeed = 0x5EED5EED5EED5EEDull;  // rng.rs:9

uint64_t splitmix_next(uint64_t& state) {
  state += 0x9E3779B97F4A7C15ull;
  uint64_t z = state;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// sample_sources (betweenness.rs:349-362) with shuffled_order (rng.rs:64-72).
std::vector<uint32_t> sample_sources(uint64_t n, bool has_sample, double frac, bool has_seed,
                                     uint64_t seed) {
  std::vector<uint32_t> out;
  if (!has_sample) {
    out.resize(n);
    for (uint64_t i = 0; i < n; i++) out[i] = (uint32_t)i;
    return out;
  }
  double f = frac;
  if (f < 0.0) f = 0.0;
  if (f > 1.0) f = 1.0;
  double kf = std::ceil((double)n * f);
  uint64_t k = (std::isnan(kf) || kf <= 0.0) ? 0 : (kf >= 1.8446744073709552e19 ? UINT64_MAX : (uint64_t)kf);
  if (k < 1) k = 1;
  if (k > n) k = n;
  if (k == 0) return out;
  std::vector<uint32_t> order(n);
  for (uint64_t i = 0; i < n; i++) order[i] = (uint32_t)i;
  uint64_t st = (has_seed ? seed : kDefaultSeed) ^ 0xD1B54A32D192ED03ull;
  for (uint64_t i = n; i-- > 1;) {
    uint64_t j = splitmix_next(st) % (i + 1);
    std::swap(order[i], order[j]);
  }
  out.assign(order.begin(), order.begin() + k);
  return out;
}

// ------------------------------------------------------------ kernels
__device__ __forceinline__ void append_bc(uint32_t* Q, uint32_t* cnt, bool take, uint32_t v) {
  uint32_t mask = __ballot_sync(0xffffffffu, take);
  if (!take) return;
  int lane = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(cnt, (uint32_t)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  Q[base + __popc(mask & ((1u << lane) - 1u))] = v;
}

__global__ void bfs_discover_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                               const uint32_t* __restrict__ F, uint64_t f,
                               const uint64_t* __restrict__ pos, uint64_t T, int32_t* dist,
                               int32_t level, uint32_t* __restrict__ N, uint32_t* __restrict__ cnt) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t span = ((T + stride - 1) / stride) * stride;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < span; e += stride) {
    bool take = false;
    uint32_t v = 0;
    if (e < T) {
      uint64_t i = owner_in_pos(pos, f, e);
      v = tgt[off[F[i]] + (uint32_t)(e - pos[i])];
      if (dist[v] < 0) take = atomicCAS(&dist[v], -1, level + 1) == -1;
    }
    append_bc(N, cnt, take, v);
  }
}

__global__ void bfs_sigma_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                            const uint32_t* __restrict__ F, uint64_t f,
                            const uint64_t* __restrict__ pos, uint64_t T,
                            const int32_t* __restrict__ dist, int32_t level, double* sigma) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < T;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t i = owner_in_pos(pos, f, e);
    uint32_t u = F[i];
    uint32_t v = tgt[off[u] + (uint32_t)(e - pos[i])];
    if (dist[v] == level + 1) atomicAdd(&sigma[v], sigma[u]);
  }
}

__device__ __forceinline__ bool tight(const unsigned long long* __restrict__ dist, uint32_t u,
                                      uint32_t v, double w) {
  unsigned long long du = dist[u], dv = dist[v];
  if (du == kInfBits || u == v) return false;
  double nd = __dadd_rn(__longlong_as_double((long long)du), w);
  if ((unsigned long long)__double_as_longlong(nd) != dv) return false;
  return du < dv || (du == dv && u < v);  // zero weights: keep the DAG acyclic
}

// tight in-slot counts over every out-slot
__global__ void tight_indeg_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                              const double* __restrict__ w, uint64_t n, uint64_t m,
                              const unsigned long long* __restrict__ dist,
                              uint32_t* __restrict__ indeg) {
  for_each_slot_owner(off, n, m, [&](uint64_t k, uint32_t u) {
    uint32_t v = tgt[k];
    if (tight(dist, u, v, w[k])) atomicAdd(&indeg[v], 1u);
  });
}

__global__ void kahn_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                       const double* __restrict__ w, const uint32_t* __restrict__ F, uint64_t f,
                       const uint64_t* __restrict__ pos, uint64_t T,
                       const unsigned long long* __restrict__ dist, uint32_t* indeg, double* sigma,
                       uint32_t* __restrict__ N, uint32_t* __restrict__ cnt) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t span = ((T + stride - 1) / stride) * stride;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < span; e += stride) {
    bool take = false;
    uint32_t v = 0;
    if (e < T) {
      uint64_t i = owner_in_pos(pos, f, e);
      uint32_t u = F[i];
      uint32_t k = off[u] + (uint32_t)(e - pos[i]);
      v = tgt[k];
      if (tight(dist, u, v, w[k])) {
        atomicAdd(&sigma[v], sigma[u]);
        take = atomicSub(&indeg[v], 1u) == 1u;
      }
    }
    append_bc(N, cnt, take, v);
  }
}

// One warp per node of the level: delta[v] = sum over DAG successors of
// sigma[v] * ((1 + delta[w]) / sigma[w]); bc[v] += delta[v] unless v == s.
template <bool kWeighted>
__global__ void dependency_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                             const double* __restrict__ w, const uint32_t* __restrict__ L,
                             uint64_t cnt, const int32_t* __restrict__ hop,
                             const unsigned long long* __restrict__ dist,
                             const double* __restrict__ sigma, double* delta, double* bc,
                             uint32_t source) {
  const int lane = threadIdx.x & 31;
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i = warp; i < cnt; i += nwarps) {
    const uint32_t v = L[i];
    const double sv = sigma[v];
    double acc = 0.0;
    for (uint32_t k = off[v] + lane; k < off[v + 1]; k += 32) {
      const uint32_t x = tgt[k];
      bool succ = kWeighted ? tight(dist, v, x, w[k]) : (hop[x] == hop[v] + 1);
      if (succ) acc += __dmul_rn(sv, __ddiv_rn(__dadd_rn(1.0, delta[x]), sigma[x]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) {
      delta[v] = acc;
      if (v != source) bc[v] += acc;
    }
  }
}

__global__ void add_into_k(double* __restrict__ dst, const double* __restrict__ src, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = __dadd_rn(dst[i], src[i]);
}

__global__ void scale_k(double* __restrict__ x, uint64_t n, double s) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    x[i] = __dmul_rn(x[i], s);
}

__global__ void seed_source_k(int32_t* hop, double* sigma, uint32_t* L, uint32_t s) {
  if (hop) hop[s] = 0;
  sigma[s] = 1.0;
  L[0] = s;
}

__global__ void fdeg_out_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ F,
                           uint64_t f, uint64_t* __restrict__ pos) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= f;
       i += (uint64_t)gridDim.x * blockDim.x)
    pos[i] = i < f ? (uint64_t)(off[F[i] + 1] - off[F[i]]) : 0ull;
}

// ---- 64 sources at once (unweighted) -------------------------------------
// Batch b holds sources [64 b, 64 b + 64) of the source list, the
// reference's accumulation chunk (betweenness.rs:45-70).  Per node v the
// batch keeps a row of 64 values per quantity (hop i32, sigma f64, delta
// f64; node-major, so lane j of a warp reads entries j and j + 32 of a row
// in one coalesced access), a visited mask and a frontier mask (bit q =
// source q).
//  forward level L: one warp per node v still missing some sources; it walks
//    v's in-edges u -> v in CSR order (eight in flight); the sources in
//    front[u] & need reach v at level L, sigma_q[v] += sigma_q[u] for each
//    (per slot, as brandes_from counts parallel edges), and the slot of the
//    out-CSR holding u -> v records those sources (dag[], the shortest-path
//    DAG per source);
//  backward level L (deepest first): one warp per node v with some source at
//    level L; over v's out-edges in CSR order, for each source q of dag[k]
//    at level L, delta_q[v] += sigma_q[v] * ((1 + delta_q[w]) / sigma_q[w])
//    (reverse_accumulate, :81-98, summed per successor instead of per
//    predecessor list);
//  fold: per node, the batch's partial = sum over q in source order of
//    delta_q[v] (v != source q), added to the result in batch order.
constexpr int kBcB = 64;

struct BcBatchArgs {
  const uint32_t* in_off;
  const uint32_t* in_src;
  const uint32_t* in_to_out;  // in-CSR slot -> out-CSR slot of the same edge
  const uint32_t* out_off;
  const uint32_t* out_tgt;
  uint64_t n;
  uint64_t qmask;
  uint64_t* vis;
  const uint64_t* front;
  uint64_t* next;
  int32_t* hop;      // n x 64
  double* sigma;     // n x 64
  double* delta;     // n x 64
  uint64_t* dag;     // per out-CSR slot
  int32_t level;
  unsigned* found;
};

__global__ void bc_seed_k(const uint32_t* __restrict__ src, uint32_t nq, uint64_t* vis, uint64_t* front,
                          int32_t* hop, double* sigma) {
  const uint32_t q = threadIdx.x;
  if (q >= nq) return;
  const uint32_t s = src[q];
  atomicOr((unsigned long long*)(vis + s), 1ull << q);
  atomicOr((unsigned long long*)(front + s), 1ull << q);
  hop[(uint64_t)s * kBcB + q] = 0;
  sigma[(uint64_t)s * kBcB + q] = 1.0;
}

__global__ void bc_forward_k(BcBatchArgs A) {
  const int lane = threadIdx.x & 31;
  const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  bool any = false;
  for (uint64_t v = gw; v < A.n; v += nw) {
    const uint64_t need = A.qmask & ~A.vis[v];
    if (need == 0) {
      if (lane == 0) A.next[v] = 0;
      continue;
    }
    const uint32_t b = A.in_off[v], e = A.in_off[v + 1];
    double s0 = 0.0, s1 = 0.0;
    uint64_t reached = 0;
    for (uint32_t k0 = b; k0 < e; k0 += 8) {
      uint32_t u = 0;
      uint64_t f = 0;
      if (lane < 8 && k0 + lane < e) {
        u = A.in_src[k0 + lane];
        f = A.front[u] & need;
        // an edge can be on several sources' DAGs at different levels; the
        // warp owning v is the only writer of v's in-slots within a level
        if (f) A.dag[A.in_to_out[k0 + lane]] |= f;
      }
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const uint64_t fj = __shfl_sync(0xffffffffu, f, j);
        const uint32_t uj = __shfl_sync(0xffffffffu, u, j);
        if (fj) {
          reached |= fj;
          const double* row = A.sigma + (uint64_t)uj * kBcB;
          if ((fj >> lane) & 1ull) s0 += row[lane];
          if ((fj >> (lane + 32)) & 1ull) s1 += row[lane + 32];
        }
      }
    }
    if (lane == 0) A.next[v] = reached;
    if (reached) {
      any = true;
      if (lane == 0) A.vis[v] |= reached;
      if ((reached >> lane) & 1ull) {
        A.sigma[v * kBcB + lane] = s0;
        A.hop[v * kBcB + lane] = A.level;
      }
      if ((reached >> (lane + 32)) & 1ull) {
        A.sigma[v * kBcB + lane + 32] = s1;
        A.hop[v * kBcB + lane + 32] = A.level;
      }
    }
  }
  if (lane == 0 && any) atomicOr(A.found, 1u);
}

__global__ void bc_backward_k(BcBatchArgs A) {
  const int lane = threadIdx.x & 31;
  const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t v = gw; v < A.n; v += nw) {
    const bool h0 = A.hop[v * kBcB + lane] == A.level;
    const bool h1 = A.hop[v * kBcB + lane + 32] == A.level;
    const uint64_t mL = (uint64_t)__ballot_sync(0xffffffffu, h0) |
                        ((uint64_t)__ballot_sync(0xffffffffu, h1) << 32);
    if (mL == 0) continue;
    const double sv0 = h0 ? A.sigma[v * kBcB + lane] : 0.0;
    const double sv1 = h1 ? A.sigma[v * kBcB + lane + 32] : 0.0;
    double d0 = 0.0, d1 = 0.0;
    const uint32_t b = A.out_off[v], e = A.out_off[v + 1];
    for (uint32_t k0 = b; k0 < e; k0 += 8) {
      uint32_t w = 0;
      uint64_t dm = 0;
      if (lane < 8 && k0 + lane < e) {
        dm = A.dag[k0 + lane] & mL;
        if (dm) w = A.out_tgt[k0 + lane];
      }
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const uint64_t dj = __shfl_sync(0xffffffffu, dm, j);
        const uint32_t wj = __shfl_sync(0xffffffffu, w, j);
        if (dj) {
          const uint64_t r = (uint64_t)wj * kBcB;
          if ((dj >> lane) & 1ull)  // coeff = (1 + delta[w]) / sigma[w]; delta[v] += sigma[v] * coeff
            d0 += __dmul_rn(sv0, __ddiv_rn(__dadd_rn(1.0, A.delta[r + lane]), A.sigma[r + lane]));
          if ((dj >> (lane + 32)) & 1ull)
            d1 += __dmul_rn(sv1, __ddiv_rn(__dadd_rn(1.0, A.delta[r + lane + 32]), A.sigma[r + lane + 32]));
        }
      }
    }
    if (h0) A.delta[v * kBcB + lane] = d0;
    if (h1) A.delta[v * kBcB + lane + 32] = d1;
  }
}

// The batch's partial (sources in order, each source's own node excluded),
// added to out in batch order.
__global__ void bc_fold_k(const double* __restrict__ delta, const uint32_t* __restrict__ src,
                          uint32_t nq, uint64_t n, double* __restrict__ out) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    double p = 0.0;
    for (uint32_t q = 0; q < nq; q++)
      if (src[q] != v) p = __dadd_rn(p, delta[v * kBcB + q]);
    out[v] = __dadd_rn(out[v], p);
  }
}

// ---- weighted, 64 sources at once -----------------------------------------
// brandes_from_weighted (:278-339) for the batch: distances by a multi-source
// frontier Bellman-Ford (lanes are sources; atomicMin on the bit patterns of
// non-negative f64, whose fixpoint is Dijkstra's distances); then the tight
// DAG per source (fl(dist[u] + w) == dist[v] exactly, the reference's tie
// rule; zero-weight ties ordered by id) as a mask per out-CSR slot; then
// sigma in rounds over that DAG -- a (node, source) is settled once every
// tight predecessor was settled in an earlier round, and sigma is the sum
// over them -- with the round as the node's level for the backward pass.
struct BcwArgs {
  const uint32_t* out_off;
  const uint32_t* out_tgt;
  const double* w_out;        // per out-CSR slot
  const uint32_t* in_off;
  const uint32_t* in_src;
  const uint32_t* in_to_out;
  uint64_t n;
  uint64_t qmask;
  unsigned long long* dist;   // n x 64 bit patterns
  const uint64_t* flag_cur;   // sources whose distance at v fell last round
  uint64_t* flag_next;
  uint64_t* dag;              // per out-CSR slot: sources for which the edge is tight
  uint64_t* reach;            // per node: sources that reach it
  const uint64_t* done_prev;
  uint64_t* done_next;
  double* sigma;
  int32_t* round;             // n x 64: the round a (node, source) settled, -1 = never
  int32_t r;
  unsigned* found;
};

__global__ void bcw_seed_k(const uint32_t* __restrict__ src, uint32_t nq, unsigned long long* dist,
                           uint64_t* flag, uint64_t* done, int32_t* round, double* sigma) {
  const uint32_t q = threadIdx.x;
  if (q >= nq) return;
  const uint32_t s = src[q];
  dist[(uint64_t)s * kBcB + q] = 0ull;  // +0.0
  atomicOr((unsigned long long*)(flag + s), 1ull << q);
  atomicOr((unsigned long long*)(done + s), 1ull << q);
  round[(uint64_t)s * kBcB + q] = 0;
  sigma[(uint64_t)s * kBcB + q] = 1.0;
}

// One Bellman-Ford round: every (v, source) whose distance fell last round
// relaxes v's out-edges.
__global__ void bcw_relax_k(BcwArgs A) {
  const int lane = threadIdx.x & 31;
  const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  bool any = false;
  for (uint64_t v = gw; v < A.n; v += nw) {
    const uint64_t fl = A.flag_cur[v];
    if (!fl) continue;
    const bool f0 = (fl >> lane) & 1ull, f1 = (fl >> (lane + 32)) & 1ull;
    const double d0 = f0 ? __longlong_as_double((long long)A.dist[v * kBcB + lane]) : 0.0;
    const double d1 = f1 ? __longlong_as_double((long long)A.dist[v * kBcB + lane + 32]) : 0.0;
    const uint32_t b = A.out_off[v], e = A.out_off[v + 1];
    for (uint32_t k0 = b; k0 < e; k0 += 8) {
      uint32_t wl = 0;
      double xl = 0.0;
      if (lane < 8 && k0 + lane < e) {
        wl = A.out_tgt[k0 + lane];
        xl = A.w_out[k0 + lane];
      }
#pragma unroll
      for (int j = 0; j < 8; j++) {
        if (k0 + j >= e) break;
        const uint32_t w = __shfl_sync(0xffffffffu, wl, j);
        const double x = __shfl_sync(0xffffffffu, xl, j);
        bool low0 = false, low1 = false;
        if (f0) {
          const unsigned long long nd = (unsigned long long)__double_as_longlong(__dadd_rn(d0, x));
          low0 = nd < atomicMin(&A.dist[(uint64_t)w * kBcB + lane], nd);
        }
        if (f1) {
          const unsigned long long nd = (unsigned long long)__double_as_longlong(__dadd_rn(d1, x));
          low1 = nd < atomicMin(&A.dist[(uint64_t)w * kBcB + lane + 32], nd);
        }
        const uint64_t lowered = (uint64_t)__ballot_sync(0xffffffffu, low0) |
                                 ((uint64_t)__ballot_sync(0xffffffffu, low1) << 32);
        if (lowered) {
          any = true;
          if (lane == 0) atomicOr((unsigned long long*)(A.flag_next + w), lowered);
        }
      }
    }
  }
  if (lane == 0 && any) atomicOr(A.found, 1u);
}

__device__ __forceinline__ bool tight_bits(unsigned long long du, unsigned long long dv, double x,
                                           uint32_t u, uint32_t v) {
  if (du == kInfBits || u == v) return false;
  const unsigned long long nd = (unsigned long long)__double_as_longlong(
      __dadd_rn(__longlong_as_double((long long)du), x));
  if (nd != dv) return false;
  return du < dv || (du == dv && u < v);  // zero weights: keep the DAG acyclic
}

// Tight mask of every out-slot, and the sources that reach each node.
__global__ void bcw_tight_k(BcwArgs A) {
  const int lane = threadIdx.x & 31;
  const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t u = gw; u < A.n; u += nw) {
    const unsigned long long du0 = A.dist[u * kBcB + lane], du1 = A.dist[u * kBcB + lane + 32];
    const uint64_t reach = ((uint64_t)__ballot_sync(0xffffffffu, du0 != kInfBits) |
                            ((uint64_t)__ballot_sync(0xffffffffu, du1 != kInfBits) << 32)) & A.qmask;
    if (lane == 0) A.reach[u] = reach;
    if (!reach) continue;
    const uint32_t b = A.out_off[u], e = A.out_off[u + 1];
    for (uint32_t k = b; k < e; k++) {
      const uint32_t v = A.out_tgt[k];
      const double x = A.w_out[k];
      const bool t0 = tight_bits(du0, A.dist[(uint64_t)v * kBcB + lane], x, (uint32_t)u, v);
      const bool t1 = tight_bits(du1, A.dist[(uint64_t)v * kBcB + lane + 32], x, (uint32_t)u, v);
      const uint64_t m = ((uint64_t)__ballot_sync(0xffffffffu, t0) |
                          ((uint64_t)__ballot_sync(0xffffffffu, t1) << 32)) & A.qmask;
      if (lane == 0) A.dag[k] = m;
    }
  }
}

// Round r of sigma: (w, source) settles when no tight predecessor is still
// unsettled (as of the round's start); sigma = the sum over its tight
// predecessors, in in-CSR order.
__global__ void bcw_sigma_k(BcwArgs A) {
  const int lane = threadIdx.x & 31;
  const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  bool any = false;
  for (uint64_t w = gw; w < A.n; w += nw) {
    const uint64_t dp = A.done_prev[w];
    const uint64_t pend = A.reach[w] & ~dp;
    if (!pend) {
      if (lane == 0) A.done_next[w] = dp;
      continue;
    }
    const uint32_t b = A.in_off[w], e = A.in_off[w + 1];
    uint64_t notready = 0;
    for (uint32_t k = b + lane; k < e; k += 32) {
      const uint64_t tm = A.dag[A.in_to_out[k]] & pend;
      if (tm) notready |= tm & ~A.done_prev[A.in_src[k]];
    }
    notready = ((uint64_t)__reduce_or_sync(0xffffffffu, (unsigned)(notready >> 32)) << 32) |
               __reduce_or_sync(0xffffffffu, (unsigned)notready);
    const uint64_t ready = pend & ~notready;
    if (lane == 0) A.done_next[w] = dp | ready;
    if (!ready) continue;
    any = true;
    double s0 = 0.0, s1 = 0.0;
    for (uint32_t k0 = b; k0 < e; k0 += 8) {
      uint32_t ul = 0;
      uint64_t tl = 0;
      if (lane < 8 && k0 + lane < e) {
        tl = A.dag[A.in_to_out[k0 + lane]] & ready;
        if (tl) ul = A.in_src[k0 + lane];
      }
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const uint64_t tj = __shfl_sync(0xffffffffu, tl, j);
        const uint32_t uj = __shfl_sync(0xffffffffu, ul, j);
        if (tj) {
          if ((tj >> lane) & 1ull) s0 += A.sigma[(uint64_t)uj * kBcB + lane];
          if ((tj >> (lane + 32)) & 1ull) s1 += A.sigma[(uint64_t)uj * kBcB + lane + 32];
        }
      }
    }
    if ((ready >> lane) & 1ull) {
      A.sigma[w * kBcB + lane] = s0;
      A.round[w * kBcB + lane] = A.r;
    }
    if ((ready >> (lane + 32)) & 1ull) {
      A.sigma[w * kBcB + lane + 32] = s1;
      A.round[w * kBcB + lane + 32] = A.r;
    }
  }
  if (lane == 0 && any) atomicOr(A.found, 1u);
}

__global__ void fill_u64_bc_k(unsigned long long* p, uint64_t n, unsigned long long v) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

__global__ void inv_perm_k(const uint32_t* __restrict__ eid, uint64_t m, uint32_t* __restrict__ inv) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m;
       k += (uint64_t)gridDim.x * blockDim.x)
    inv[eid[k]] = (uint32_t)k;
}

__global__ void compose_k(const uint32_t* __restrict__ a, const uint32_t* __restrict__ inv, uint64_t m,
                          uint32_t* __restrict__ out) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m;
       k += (uint64_t)gridDim.x * blockDim.x)
    out[k] = inv[a[k]];
}

}  // namespace

// Unweighted betweenness over `sources`, 64 at a time, added into d_out.
static void betweenness_batched(TopoImpl* t, const std::vector<uint32_t>& sources, double* d_out,
                                cudaStream_t s) {
  const uint64_t n = t->n, m = t->m;
  ensure_in(t, s);
  Scratch<uint32_t> in_to_out(m ? m : 1, s);
  if (m) {
    Scratch<uint32_t> inv(m, s);
    inv_perm_k<<<grid_for(m), kBlock, 0, s>>>(t->out.eid.get(), m, inv.get());
    UG_LAUNCH_CHECK();
    compose_k<<<grid_for(m), kBlock, 0, s>>>(t->in.eid.get(), inv.get(), m, in_to_out.get());
    UG_LAUNCH_CHECK();
  }
  Scratch<uint64_t> vis(n, s), fa(n, s), fb(n, s), dag(m ? m : 1, s);
  Scratch<int32_t> hop(n * kBcB, s);
  Scratch<double> sigma(n * kBcB, s), delta(n * kBcB, s);
  Scratch<uint32_t> d_src(kBcB, s);
  Scratch<unsigned> found(1, s);
  BcBatchArgs a;
  a.in_off = t->in.off.get();
  a.in_src = t->in.tgt.get();
  a.in_to_out = in_to_out.get();
  a.out_off = t->out.off.get();
  a.out_tgt = t->out.tgt.get();
  a.n = n;
  a.vis = vis.get();
  a.hop = hop.get();
  a.sigma = sigma.get();
  a.delta = delta.get();
  a.dag = dag.get();
  a.found = found.get();
  const unsigned gw = grid_for(n * 32, kBlock, 148u * 8u);
  for (size_t c0 = 0; c0 < sources.size(); c0 += kBcB) {
    const uint32_t nq = (uint32_t)std::min<size_t>(kBcB, sources.size() - c0);
    a.qmask = nq == 64 ? ~0ull : ((1ull << nq) - 1ull);
    UG_CUDA(cudaMemcpyAsync(d_src.get(), sources.data() + c0, nq * 4, cudaMemcpyHostToDevice, s));
    UG_CUDA(cudaMemsetAsync(vis.get(), 0, n * 8, s));
    UG_CUDA(cudaMemsetAsync(fa.get(), 0, n * 8, s));
    UG_CUDA(cudaMemsetAsync(hop.get(), 0xFF, n * kBcB * 4, s));
    UG_CUDA(cudaMemsetAsync(sigma.get(), 0, n * kBcB * 8, s));
    UG_CUDA(cudaMemsetAsync(delta.get(), 0, n * kBcB * 8, s));
    if (m) UG_CUDA(cudaMemsetAsync(dag.get(), 0, m * 8, s));
    bc_seed_k<<<1, kBcB, 0, s>>>(d_src.get(), nq, vis.get(), fa.get(), hop.get(), sigma.get());
    UG_LAUNCH_CHECK();
    int32_t L = 0;
    uint64_t* cur = fa.get();
    uint64_t* nxt = fb.get();
    while (true) {
      a.level = L + 1;
      a.front = cur;
      a.next = nxt;
      UG_CUDA(cudaMemsetAsync(found.get(), 0, 4, s));
      bc_forward_k<<<gw, kBlock, 0, s>>>(a);
      UG_LAUNCH_CHECK();
      unsigned f = 0;
      UG_CUDA(cudaMemcpyAsync(&f, found.get(), 4, cudaMemcpyDeviceToHost, s));
      UG_CUDA(cudaStreamSynchronize(s));
      if (!f) break;
      L++;
      std::swap(cur, nxt);
    }
    // nodes of the deepest level L have no successors (delta 0)
    for (int32_t lvl = L - 1; lvl >= 0; lvl--) {
      a.level = lvl;
      bc_backward_k<<<gw, kBlock, 0, s>>>(a);
      UG_LAUNCH_CHECK();
    }
    bc_fold_k<<<grid_for(n), kBlock, 0, s>>>(delta.get(), d_src.get(), nq, n, d_out);
    UG_LAUNCH_CHECK();
  }
}

// Weighted betweenness over `sources`, 64 at a time, added into d_out;
// w_out: the weights in out-CSR slot order.
static void betweenness_weighted_batched(TopoImpl* t, const double* w_out,
                                         const std::vector<uint32_t>& sources, double* d_out,
                                         cudaStream_t s) {
  const uint64_t n = t->n, m = t->m;
  ensure_in(t, s);
  Scratch<uint32_t> in_to_out(m ? m : 1, s);
  if (m) {
    Scratch<uint32_t> inv(m, s);
    inv_perm_k<<<grid_for(m), kBlock, 0, s>>>(t->out.eid.get(), m, inv.get());
    UG_LAUNCH_CHECK();
    compose_k<<<grid_for(m), kBlock, 0, s>>>(t->in.eid.get(), inv.get(), m, in_to_out.get());
    UG_LAUNCH_CHECK();
  }
  Scratch<unsigned long long> dist(n * kBcB, s);
  Scratch<uint64_t> fl0(n, s), fl1(n, s), reach(n, s), dn0(n, s), dn1(n, s), dag(m ? m : 1, s);
  Scratch<int32_t> round(n * kBcB, s);
  Scratch<double> sigma(n * kBcB, s), delta(n * kBcB, s);
  Scratch<uint32_t> d_src(kBcB, s);
  Scratch<unsigned> found(1, s);
  BcwArgs a;
  a.out_off = t->out.off.get();
  a.out_tgt = t->out.tgt.get();
  a.w_out = w_out;
  a.in_off = t->in.off.get();
  a.in_src = t->in.tgt.get();
  a.in_to_out = in_to_out.get();
  a.n = n;
  a.dist = dist.get();
  a.dag = dag.get();
  a.reach = reach.get();
  a.sigma = sigma.get();
  a.round = round.get();
  a.found = found.get();
  BcBatchArgs bk{};  // the backward pass of the unweighted batch, on rounds and the tight DAG
  bk.out_off = t->out.off.get();
  bk.out_tgt = t->out.tgt.get();
  bk.n = n;
  bk.hop = round.get();
  bk.sigma = sigma.get();
  bk.delta = delta.get();
  bk.dag = dag.get();
  const unsigned gw = grid_for(n * 32, kBlock, 148u * 8u);
  auto read_found = [&]() {
    unsigned f = 0;
    UG_CUDA(cudaMemcpyAsync(&f, found.get(), 4, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
    return f;
  };
  for (size_t c0 = 0; c0 < sources.size(); c0 += kBcB) {
    const uint32_t nq = (uint32_t)std::min<size_t>(kBcB, sources.size() - c0);
    a.qmask = nq == 64 ? ~0ull : ((1ull << nq) - 1ull);
    UG_CUDA(cudaMemcpyAsync(d_src.get(), sources.data() + c0, nq * 4, cudaMemcpyHostToDevice, s));
    fill_u64_bc_k<<<grid_for(n * kBcB), kBlock, 0, s>>>(dist.get(), n * kBcB, kInfBits);
    UG_LAUNCH_CHECK();
    UG_CUDA(cudaMemsetAsync(fl0.get(), 0, n * 8, s));
    UG_CUDA(cudaMemsetAsync(fl1.get(), 0, n * 8, s));
    UG_CUDA(cudaMemsetAsync(dn0.get(), 0, n * 8, s));
    UG_CUDA(cudaMemsetAsync(round.get(), 0xFF, n * kBcB * 4, s));
    UG_CUDA(cudaMemsetAsync(sigma.get(), 0, n * kBcB * 8, s));
    UG_CUDA(cudaMemsetAsync(delta.get(), 0, n * kBcB * 8, s));
    if (m) UG_CUDA(cudaMemsetAsync(dag.get(), 0, m * 8, s));  // unreached nodes' slots stay 0
    bcw_seed_k<<<1, kBcB, 0, s>>>(d_src.get(), nq, dist.get(), fl0.get(), dn0.get(), round.get(),
                                  sigma.get());
    UG_LAUNCH_CHECK();
    // distances
    uint64_t* cur = fl0.get();
    uint64_t* nxt = fl1.get();
    while (true) {
      a.flag_cur = cur;
      a.flag_next = nxt;
      UG_CUDA(cudaMemsetAsync(found.get(), 0, 4, s));
      bcw_relax_k<<<gw, kBlock, 0, s>>>(a);
      UG_LAUNCH_CHECK();
      UG_CUDA(cudaMemsetAsync(cur, 0, n * 8, s));  // consumed
      if (!read_found()) break;
      std::swap(cur, nxt);
    }
    // tight DAG, then sigma by rounds
    bcw_tight_k<<<gw, kBlock, 0, s>>>(a);
    UG_LAUNCH_CHECK();
    uint64_t* dprev = dn0.get();
    uint64_t* dnext = dn1.get();
    int32_t r = 0;
    while (true) {
      a.r = r + 1;
      a.done_prev = dprev;
      a.done_next = dnext;
      UG_CUDA(cudaMemsetAsync(found.get(), 0, 4, s));
      bcw_sigma_k<<<gw, kBlock, 0, s>>>(a);
      UG_LAUNCH_CHECK();
      if (!read_found()) break;
      r++;
      std::swap(dprev, dnext);
    }
    // backward over rounds, deepest first (round r's nodes have no successors)
    for (int32_t lvl = r - 1; lvl >= 0; lvl--) {
      bk.level = lvl;
      bc_backward_k<<<gw, kBlock, 0, s>>>(bk);
      UG_LAUNCH_CHECK();
    }
    bc_fold_k<<<grid_for(n), kBlock, 0, s>>>(delta.get(), d_src.get(), nq, n, d_out);
    UG_LAUNCH_CHECK();
  }
}

struct BcState {
  Scratch<int32_t> hop;                 // unweighted BFS level (-1 = unreached)
  Scratch<unsigned long long> dist;     // weighted distance bits
  Scratch<uint32_t> indeg;              // weighted: tight in-slots left
  Scratch<double> sigma, delta;
  Scratch<uint32_t> L;                  // nodes in discovery order, by level
  Scratch<uint64_t> pos;
  Scratch<uint32_t> cnt;
};

static uint64_t out_scan(const uint32_t* off, const uint32_t* F, uint64_t f, uint64_t* pos,
                         cudaStream_t s) {
  fdeg_out_k<<<grid_for(f + 1), kBlock, 0, s>>>(off, F, f, pos);
  UG_LAUNCH_CHECK();
  exclusive_scan_u64(pos, pos, f + 1, nullptr, s);
  uint64_t total = 0;
  UG_CUDA(cudaMemcpyAsync(&total, pos + f, 8, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  return total;
}

// One source's dependencies added into acc.
static void brandes_source(TopoImpl* t, const double* w_out, uint32_t src, BcState& st,
                           double* acc, cudaStream_t s) {
  const uint64_t n = t->n, m = t->m;
  const uint32_t* off = t->out.off.get();
  const uint32_t* tgt = t->out.tgt.get();
  const bool weighted = w_out != nullptr;
  UG_CUDA(cudaMemsetAsync(st.sigma.get(), 0, n * 8, s));
  UG_CUDA(cudaMemsetAsync(st.delta.get(), 0, n * 8, s));
  if (weighted) {
    DirView dv{};
    dv.off0 = off;
    dv.tgt0 = tgt;
    dv.eid0 = t->out.eid.get();
    sssp_run(dv, w_out, nullptr, n, src, st.dist.get(), s);
    UG_CUDA(cudaMemsetAsync(st.indeg.get(), 0, n * 4, s));
    if (m) {
      tight_indeg_k<<<grid_for(m, kBlock, 148u * 64u), kBlock, 0, s>>>(off, tgt, w_out, n, m,
                                                                        st.dist.get(),
                                                                        st.indeg.get());
      UG_LAUNCH_CHECK();
    }
  } else {
    UG_CUDA(cudaMemsetAsync(st.hop.get(), 0xFF, n * 4, s));
  }
  seed_source_k<<<1, 1, 0, s>>>(weighted ? nullptr : st.hop.get(), st.sigma.get(), st.L.get(), src);
  UG_LAUNCH_CHECK();
  std::vector<uint64_t> lev = {0, 1};  // level l = L[lev[l] .. lev[l+1])
  int32_t level = 0;
  while (true) {
    const uint64_t lo = lev[lev.size() - 2], hi = lev.back();
    const uint64_t f = hi - lo;
    if (f == 0) break;
    const uint32_t* F = st.L.get() + lo;
    uint64_t T = out_scan(off, F, f, st.pos.get(), s);
    if (T == 0) {
      lev.push_back(hi);
      break;
    }
    UG_CUDA(cudaMemsetAsync(st.cnt.get(), 0, 4, s));
    unsigned g = grid_for(T, kBlock, 148u * 64u);
    if (weighted) {
      kahn_k<<<g, kBlock, 0, s>>>(off, tgt, w_out, F, f, st.pos.get(), T, st.dist.get(),
                                  st.indeg.get(), st.sigma.get(), st.L.get() + hi, st.cnt.get());
      UG_LAUNCH_CHECK();
    } else {
      bfs_discover_k<<<g, kBlock, 0, s>>>(off, tgt, F, f, st.pos.get(), T, st.hop.get(), level,
                                          st.L.get() + hi, st.cnt.get());
      UG_LAUNCH_CHECK();
      bfs_sigma_k<<<g, kBlock, 0, s>>>(off, tgt, F, f, st.pos.get(), T, st.hop.get(), level,
                                       st.sigma.get());
      UG_LAUNCH_CHECK();
    }
    uint32_t next = read_u32(st.cnt.get(), s);
    lev.push_back(hi + next);
    level++;
  }
  // reverse accumulation, deepest level first
  for (size_t l = lev.size() - 1; l-- > 0;) {
    const uint64_t lo = lev[l], hi = lev[l + 1];
    if (hi <= lo) continue;
    const uint64_t cnt = hi - lo;
    unsigned g = grid_for(cnt * 32, kBlock, 148u * 64u);
    if (weighted)
      dependency_k<true><<<g, kBlock, 0, s>>>(off, tgt, w_out, st.L.get() + lo, cnt, nullptr,
                                              st.dist.get(), st.sigma.get(), st.delta.get(), acc,
                                              src);
    else
      dependency_k<false><<<g, kBlock, 0, s>>>(off, tgt, nullptr, st.L.get() + lo, cnt,
                                               st.hop.get(), nullptr, st.sigma.get(),
                                               st.delta.get(), acc, src);
    UG_LAUNCH_CHECK();
  }
}

void betweenness_run(TopoImpl* t, const double* d_weights, bool has_sample, double sample,
                     bool has_seed, uint64_t seed, double* d_out, cudaStream_t s) {
  const uint64_t n = t->n, m = t->m;
  if (n == 0) return;
  std::vector<uint32_t> sources = sample_sources(n, has_sample, sample, has_seed, seed);
  UG_CUDA(cudaMemsetAsync(d_out, 0, n * 8, s));
  if (sources.empty()) return;
  BcState st;
  st.sigma.alloc(n, s);
  st.delta.alloc(n, s);
  st.L.alloc(n, s);
  st.pos.alloc(n + 1, s);
  st.cnt.alloc(1, s);
  Scratch<double> w_out;
  if (d_weights) {
    st.dist.alloc(n, s);
    st.indeg.alloc(n, s);
    w_out.alloc(m ? m : 1, s);
    DirView dv{};
    dv.off0 = t->out.off.get();
    dv.tgt0 = t->out.tgt.get();
    dv.eid0 = t->out.eid.get();
    DirWeights dw;
    gather_dir_weights(t, dv, d_weights, dw, s);
    swap(w_out, dw.w0);
  } else {
    st.hop.alloc(n, s);
  }
  if (!d_weights) {
    betweenness_batched(t, sources, d_out, s);
  } else if (kBatchedWeighted) {
    betweenness_weighted_batched(t, w_out.get(), sources, d_out, s);
  } else {
  Scratch<double> acc(n, s);
  for (size_t c0 = 0; c0 < sources.size(); c0 += kSrcChunk) {
    UG_CUDA(cudaMemsetAsync(acc.get(), 0, n * 8, s));
    size_t c1 = c0 + kSrcChunk < sources.size() ? c0 + kSrcChunk : sources.size();
    for (size_t i = c0; i < c1; i++)
      brandes_source(t, d_weights ? w_out.get() : nullptr, sources[i], st, acc.get(), s);
    add_into_k<<<grid_for(n), kBlock, 0, s>>>(d_out, acc.get(), n);
    UG_LAUNCH_CHECK();
  }
  }
  if (has_sample) {
    scale_k<<<grid_for(n), kBlock, 0, s>>>(d_out, n, (double)n / (double)sources.size());
    UG_LAUNCH_CHECK();
  }
}

}  // namespace ug

using namespace ug;

extern "C" {

int ursa_gpu_betweenness(ursa_gpu_topo* t, int has_sample, double sample, int has_seed,
                         uint64_t seed, double* out) {
  return guard([&] {
    UG_CHECK(t, URSA_GPU_EINVAL, "topology is NULL");
    TopoImpl* ti = &t->impl;
    if (ti->n == 0) return;  // betweenness.rs:155-157
    UG_CHECK(out, URSA_GPU_EINVAL, "out is NULL");
    cudaStream_t s = thread_stream(ti->device);
    Scratch<double> d(ti->n, s);
    betweenness_run(ti, nullptr, has_sample != 0, sample, has_seed != 0, seed, d.get(), s);
    UG_CUDA(cudaMemcpyAsync(out, d.get(), ti->n * 8, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_betweenness_weighted(ursa_gpu_topo* t, const double* weights, uint64_t n_weights,
                                  int has_sample, double sample, int has_seed, uint64_t seed,
                                  double* out) {
  return guard([&] {
    UG_CHECK(t, URSA_GPU_EINVAL, "topology is NULL");
    TopoImpl* ti = &t->impl;
    UG_CHECK(n_weights == ti->m, URSA_GPU_EINVAL, "weights length must equal the edge count");
    UG_CHECK(ti->m == 0 || weights, URSA_GPU_EINVAL, "weights is NULL");
    if (ti->n == 0) return;  // betweenness.rs:248-250
    UG_CHECK(out, URSA_GPU_EINVAL, "out is NULL");
    cudaStream_t s = thread_stream(ti->device);
    Scratch<double> dw(ti->m ? ti->m : 1, s), d(ti->n, s);
    if (ti->m) UG_CUDA(cudaMemcpyAsync(dw.get(), weights, ti->m * 8, cudaMemcpyHostToDevice, s));
    check_sssp_weights_device(dw.get(), ti->m, s);
    betweenness_run(ti, dw.get(), has_sample != 0, sample, has_seed != 0, seed, d.get(), s);
    UG_CUDA(cudaMemcpyAsync(out, d.get(), ti->n * 8, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

}  // extern "C"
