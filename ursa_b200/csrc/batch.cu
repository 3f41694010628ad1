// batch.cu -- many small independent graphs in one CUDA-graph launch:
// pagerank (ursa-core/src/algo/pagerank.rs:63-124), connected_components_weak
// (components.rs:14-68) and triangle_count (triangle.rs:23-62) for every
// graph of a batch.  The reference runs these per Topology; here the batch is
// one device-resident block-diagonal union (graph g owns the node range
// [N_g, N_g + n_g)), described per graph by a GraphDesc.
//
// Execution.  Graphs are sorted into buckets by node count.  Each bucket is a
// persistent kernel whose CTAs take whole graphs from a work list (largest
// first) and run all three algorithms for that graph before taking the next:
//  * pagerank: the f32 shares of the graph live in shared memory (one f32 per
//    node), so every per-edge gather is a shared-memory load; each iteration
//    writes the next shares to a global staging row (L2-resident) and
//    reloads them after the CTA barrier.  Graphs larger than the bucket's
//    capacity keep their shares in global memory.  Rows are visited by
//    degree class (rows of each graph grouped by in-degree at build time)
//    with 32/16/8/4/2/1 lanes per row, each lane summing its strided edges
//    with Kahan-compensated f32 and the group combining in a fixed tree.
//    The lane count depends on the row's in-degree only, and the L1 residual
//    and dangling mass are summed as 128-bit fixed-point integers (each term
//    truncated at 2^-96, order-independent), so the results do not depend on
//    the bucket, the CTA size or the other graphs of the batch.
//  * weak components: lock-free union-find over the graph's oriented
//    undirected edges with the parent array in shared memory; labels are
//    each component's minimum local id.
//  * triangle counts: per oriented edge (u, v) the sorted oriented lists of u
//    and v are merged; counts are integer atomics in shared memory.
// The bucket kernels run on parallel branches of one captured CUDA graph.
// A project-written autotuner picks the bucket capacities, CTA sizes and the
// triangle-count tile by timing the captured graph; results are identical
// for every configuration.
#include <algorithm>
#include <cstring>
#include <vector>

#include "frontier.cuh"
#include "primitives.cuh"
#include "batch.cuh"
#include "fixedpoint.cuh"
#include "unionfind.cuh"

namespace ug {

namespace {

constexpr int kBkMaxBuckets = 3;
// Shared-memory budget of one CTA for per-node state (f32 shares, u32
// parents or counts), leaving room for the static reduction area.
constexpr uint32_t kBkSmemBytesMax = 224u * 1024u;

struct BkShared {
  GraphDesc g;
  unsigned long long red[4 * 32];
  double tot[2];
  uint32_t unit_begin[8];
  uint32_t range[2];
  uint32_t item;
};

// Block sum of two fixed-point accumulators; every thread gets the f64
// values.  Integer addition is exact, so the order does not matter.
template <int NT>
__device__ __forceinline__ void block_sum2(u128 a, u128 b, BkShared& sh, double& va, double& vb) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += shfl_down_u128(a, o);
    b += shfl_down_u128(b, o);
  }
  if (lane == 0) {
    sh.red[4 * w + 0] = (unsigned long long)a;
    sh.red[4 * w + 1] = (unsigned long long)(a >> 64);
    sh.red[4 * w + 2] = (unsigned long long)b;
    sh.red[4 * w + 3] = (unsigned long long)(b >> 64);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    u128 ta = 0, tb = 0;
    for (int i = 0; i < NT / 32; i++) {
      ta += ((u128)sh.red[4 * i + 1] << 64) | sh.red[4 * i + 0];
      tb += ((u128)sh.red[4 * i + 3] << 64) | sh.red[4 * i + 2];
    }
    sh.tot[0] = fx_value(ta);
    sh.tot[1] = fx_value(tb);
  }
  __syncthreads();
  va = sh.tot[0];
  vb = sh.tot[1];
}

__device__ __forceinline__ void bk_kahan_add(float& s, float& c, float v) {
  float y = __fsub_rn(v, c);
  float t = __fadd_rn(s, y);
  c = __fsub_rn(__fsub_rn(t, s), y);
  s = t;
}

// Shares of edges [b + sub, e) with stride G, B loads in flight per lane; the
// per-lane addition order is the edge order whatever B is.
template <int G, int B>
__device__ __forceinline__ F2 bk_row_sum(const uint32_t* __restrict__ src, const float* x,
                                         uint32_t idb, uint32_t b, uint32_t e, int sub) {
  float s = 0.f, c = 0.f;
  for (uint32_t j = b + sub; j < e; j += B * G) {
    uint32_t v[B];
#pragma unroll
    for (int k = 0; k < B; k++) {
      const uint32_t jj = j + k * G;
      v[k] = jj < e ? __ldg(src + jj) - idb : 0u;
    }
    float sv[B];
#pragma unroll
    for (int k = 0; k < B; k++) sv[k] = (j + k * G < e) ? x[v[k]] : 0.f;
#pragma unroll
    for (int k = 0; k < B; k++)
      if (j + k * G < e) bk_kahan_add(s, c, sv[k]);
  }
  return F2{s, -c};
}

template <int G>
__device__ __forceinline__ F2 bk_group_sum(F2 v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    F2 t{__shfl_down_sync(0xffffffffu, v.hi, o, G), __shfl_down_sync(0xffffffffu, v.lo, o, G)};
    v = f2_combine(v, t);
  }
  return v;
}

struct PrIter {
  const float* xr;  // current shares (shared or global), local ids
  float* xw;        // next shares (global)
  double base, damping;
  u128 delta, dang;
};

template <int G>
__device__ __forceinline__ void bk_class_unit(const GraphDesc& g, uint32_t lo, uint32_t hi,
                                              uint32_t unit, PrIter& it) {
  const int lane = threadIdx.x & 31;
  const int sub = lane % G;
  const uint32_t idx = lo + unit * (32u / G) + (uint32_t)(lane / G);
  const bool valid = idx < hi;
  uint32_t r = 0, b = 0, e = 0;
  if (valid) {
    r = g.rows[idx];
    b = g.in_off[r];
    e = g.in_off[r + 1];
  }
  F2 acc = bk_row_sum<G, (G >= 32 ? 8 : 4)>(g.in_src, it.xr, g.id_base, b, e, sub);
  acc = bk_group_sum<G>(acc);
  if (valid && sub == 0) {
    // next[u] = base + d * contrib(u)   (pagerank.rs:81-83)
    const double old = g.rank[r];
    const double nx = __dadd_rn(it.base, __dmul_rn(it.damping, f2_value(acc)));
    it.delta += fx_of(fabs(__dsub_rn(nx, old)));
    g.rank[r] = nx;
    const uint32_t od = g.out_off[r + 1] - g.out_off[r];
    it.xw[r] = od ? __double2float_rn(__ddiv_rn(nx, (double)od)) : 0.f;
    if (!od) it.dang += fx_of(nx);
  }
}

template <int NT>
__device__ void bk_pagerank(const BucketArgs& A, BkShared& sh, float* sx, uint32_t gi) {
  const GraphDesc& g = sh.g;
  const uint32_t n = g.n;
  const bool in_smem = n <= A.cap;
  const double nf = (double)n;
  const double r0 = __ddiv_rn(1.0, nf);
  if (threadIdx.x == 0) {
    uint32_t u = 0;
    sh.unit_begin[0] = 0;
    for (int c = 0; c < 6; c++) {
      const uint32_t rpu = 1u << c;  // rows per unit: 32 / G with G = 32 >> c
      u += (g.cls[c + 1] - g.cls[c] + rpu - 1) >> c;
      sh.unit_begin[c + 1] = u;
    }
  }
  // rank_0 = 1/n, shares and dangling mass of rank_0
  u128 dang = 0;
  for (uint32_t u = threadIdx.x; u < n; u += NT) {
    g.rank[u] = r0;
    const uint32_t od = g.out_off[u + 1] - g.out_off[u];
    const float xv = od ? __double2float_rn(__ddiv_rn(r0, (double)od)) : 0.f;
    if (in_smem)
      sx[u] = xv;
    else
      g.x0[u] = xv;
    if (!od) dang += fx_of(r0);
  }
  double dm, unused;
  block_sum2<NT>(0, dang, sh, unused, dm);
  const uint32_t n_units = sh.unit_begin[6];
  const uint32_t warp = threadIdx.x >> 5;
  int cur = 0;
  uint32_t iters = 0;
  double delta = 0.0;
  for (uint32_t itn = 0; itn < A.max_iter; itn++) {
    PrIter it;
    it.xr = in_smem ? sx : (cur ? g.x1 : g.x0);
    it.xw = cur ? g.x0 : g.x1;
    // base = (1-d)/n + d*dangling_mass/n   (pagerank.rs:79)
    it.base = __dadd_rn(__ddiv_rn(1.0 - A.damping, nf), __ddiv_rn(__dmul_rn(A.damping, dm), nf));
    it.damping = A.damping;
    it.delta = 0;
    it.dang = 0;
    for (uint32_t u = warp; u < n_units; u += NT / 32) {
      int c = 0;
#pragma unroll
      for (int k = 1; k < 6; k++)
        if (u >= sh.unit_begin[k]) c = k;
      const uint32_t unit = u - sh.unit_begin[c];
      const uint32_t lo = g.cls[c], hi = g.cls[c + 1];
      switch (c) {
        case 0: bk_class_unit<32>(g, lo, hi, unit, it); break;
        case 1: bk_class_unit<16>(g, lo, hi, unit, it); break;
        case 2: bk_class_unit<8>(g, lo, hi, unit, it); break;
        case 3: bk_class_unit<4>(g, lo, hi, unit, it); break;
        case 4: bk_class_unit<2>(g, lo, hi, unit, it); break;
        default: bk_class_unit<1>(g, lo, hi, unit, it); break;
      }
    }
    block_sum2<NT>(it.delta, it.dang, sh, delta, dm);
    if (in_smem) {
      for (uint32_t u = threadIdx.x; u < n; u += NT) sx[u] = __ldcg(it.xw + u);
      __syncthreads();
    }
    cur ^= 1;
    iters++;
    if (delta < A.tol) break;  // every thread holds the same delta
  }
  if (threadIdx.x == 0) {
    A.iters[gi] = iters;
    A.delta[gi] = delta;
  }
  __syncthreads();
}

// Owner rows of the slots [first, last] of o_off (rows [0, n)).
__device__ __forceinline__ uint32_t bk_owner_between(const uint32_t* __restrict__ off, uint32_t lo,
                                                     uint32_t hi, uint32_t k) {
  while (lo < hi) {
    const uint32_t mid = lo + ((hi - lo + 1) >> 1);
    if (off[mid] <= k)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

template <int NT>
__device__ void bk_components(BkShared& sh, uint32_t* par) {
  const GraphDesc& g = sh.g;
  const uint32_t n = g.n;
  for (uint32_t u = threadIdx.x; u < n; u += NT) par[u] = u;
  __syncthreads();
  const uint32_t ob = g.o_off[0], oe = g.o_off[n];
  for (uint32_t base = ob; base < oe; base += NT) {
    if (threadIdx.x == 0) {
      const uint32_t last = base + NT - 1 < oe ? base + NT - 1 : oe - 1;
      sh.range[0] = owner_of(g.o_off, n, base);
      sh.range[1] = owner_of(g.o_off, n, last);
    }
    __syncthreads();
    const uint32_t k = base + threadIdx.x;
    if (k < oe) {
      const uint32_t u = bk_owner_between(g.o_off, sh.range[0], sh.range[1], k);
      uf_unite(par, u, g.o_tgt[k] - g.id_base);
    }
    __syncthreads();
  }
  // final roots; when par is the output itself, writing a root into par[u]
  // is a valid compression for concurrent walks
  for (uint32_t u = threadIdx.x; u < n; u += NT) g.cc[u] = uf_root(par, u);
  __syncthreads();
}

// ------------------------------------------------------- triangle counting
// Batch-wide: warps take units of `unit_len` consecutive vertices of one
// graph from a shared counter.  For a vertex u with oriented list N+(u), the
// warp marks N+(u) in its shared-memory bitmap (local ids), then streams the
// concatenation of N+(v) for all v in N+(u) -- lane p takes element p of the
// concatenation, located by a warp scan of the list lengths -- and every w
// found in the bitmap closes the triangle {u, v, w}, counted once (u < v < w
// in the orientation's rank order) and credited to all three vertices: u's
// credit once per vertex, v's once per run of lanes on the same v, w's per
// hit.  A 32-element chunk inside one or two lists (the common case) needs
// no per-lane search.  Graphs above kTcBitCap nodes use a per-lane sorted merge.
constexpr uint32_t kTcBitCap = 65536;  // nodes per graph on the bitmap path

struct TcArgs {
  const GraphDesc* desc;
  const uint2* units;  // {graph, first local vertex}
  uint32_t n_units;
  uint32_t unit_len;
  uint32_t words;      // bitmap words per warp (largest bitmap graph)
  uint32_t* next;
};

template <int NT>
__global__ void __launch_bounds__(NT) tc_batch_k(TcArgs A) {
  extern __shared__ __align__(16) uint32_t tc_smem[];
  const uint32_t FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  uint32_t* bm = tc_smem + (threadIdx.x >> 5) * A.words;
  // every vertex clears the bits it sets, so the bitmap is zeroed once
  for (uint32_t i = lane; i < A.words; i += 32) bm[i] = 0u;
  __syncwarp();
  while (true) {
    uint32_t unit = 0;
    if (lane == 0) unit = atomicAdd(A.next, 1u);
    unit = __shfl_sync(FULL, unit, 0);
    if (unit >= A.n_units) break;
    const uint2 un = A.units[unit];
    const GraphDesc* gd = A.desc + un.x;
    const uint32_t* __restrict__ off = gd->o_off;
    const uint32_t* __restrict__ tgt = gd->o_tgt;
    uint32_t* tri = gd->tri;
    const uint32_t n = gd->n, idb = gd->id_base;
    const uint32_t last = un.y + A.unit_len < n ? un.y + A.unit_len : n;
    const bool bitmap = n <= A.words * 32u;
    for (uint32_t u = un.y; u < last; u++) {
      const uint32_t ob = off[u], oe = off[u + 1];
      if (oe - ob < 2) continue;  // u is the lowest vertex of no triangle
      uint32_t cu = 0;
      if (bitmap) {
        for (uint32_t i = ob + lane; i < oe; i += 32) {
          const uint32_t w = tgt[i] - idb;
          atomicOr(&bm[w >> 5], 1u << (w & 31));
        }
        __syncwarp();
        for (uint32_t vb = ob; vb < oe; vb += 32) {
          const uint32_t i = vb + lane;
          uint32_t v = 0, st = 0, len = 0;
          if (i < oe) {
            v = tgt[i] - idb;
            st = off[v];
            len = off[v + 1] - st;
          }
          uint32_t incl = len;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += t;
          }
          const uint32_t total = __shfl_sync(FULL, incl, 31);
          const uint32_t excl = incl - len;
          const uint32_t nonempty = __ballot_sync(FULL, len > 0);
          for (uint32_t pb = 0; pb < total; pb += 32) {
            const uint32_t p = pb + lane;
            const uint32_t lim = pb + 32 < total ? pb + 32 : total;
            // first list still live at pb (non-empty: its end exceeds pb)
            const uint32_t j0 = __popc(__ballot_sync(FULL, incl <= pb));
            const uint32_t end0 = __shfl_sync(FULL, incl, j0);
            const bool one_list = end0 >= lim;
            uint32_t j = j0;
            if (!one_list) {
              const uint32_t after = j0 < 31 ? nonempty & (0xfffffffeu << j0) : 0u;
              const uint32_t j1 = after ? (uint32_t)(__ffs(after) - 1) : 31u;
              if (__shfl_sync(FULL, incl, j1) >= lim) {
                j = p < end0 ? j0 : j1;  // the chunk spans two lists
              } else {
                j = 0;  // first lane whose inclusive end exceeds p
#pragma unroll
                for (int step = 16; step >= 1; step >>= 1) {
                  const uint32_t t = __shfl_sync(FULL, incl, j + step - 1);
                  if (t <= p) j += step;
                }
              }
            }
            const uint32_t vj = __shfl_sync(FULL, v, j);
            const uint32_t sj = __shfl_sync(FULL, st, j);
            const uint32_t ej = __shfl_sync(FULL, excl, j);
            bool hit = false;
            if (p < total) {
              const uint32_t w = tgt[sj + (p - ej)] - idb;
              hit = (bm[w >> 5] >> (w & 31)) & 1u;
              if (hit) atomicAdd(&tri[w], 1u);
            }
            const uint32_t hits = __ballot_sync(FULL, hit);
            if (hits) {
              cu += hit ? 1u : 0u;
              // v's credit: one atomic per run of lanes on the same v
              const uint32_t run = one_list ? FULL : __match_any_sync(FULL, j);
              const uint32_t c = __popc(run & hits);
              if (c && lane == __ffs(run) - 1) atomicAdd(&tri[vj], c);
            }
          }
        }
        __syncwarp();
        for (uint32_t i = ob + lane; i < oe; i += 32) bm[(tgt[i] - idb) >> 5] = 0u;
        __syncwarp();
      } else {
        for (uint32_t q = ob + lane; q < oe; q += 32) {
          const uint32_t v = tgt[q] - idb;
          uint32_t i = ob, j = off[v];
          const uint32_t je = off[v + 1];
          uint32_t c = 0;
          if (j < je) {
            uint32_t a = tgt[i], b = tgt[j];
            while (true) {
              if (a < b) {
                if (++i == oe) break;
                a = tgt[i];
              } else if (a > b) {
                if (++j == je) break;
                b = tgt[j];
              } else {
                c++;
                atomicAdd(&tri[a - idb], 1u);
                if (++i == oe || ++j == je) break;
                a = tgt[i];
                b = tgt[j];
              }
            }
          }
          if (c) atomicAdd(&tri[v], c);
          cu += c;
        }
      }
      cu = __reduce_add_sync(FULL, cu);
      if (lane == 0 && cu) atomicAdd(&tri[u], cu);
    }
  }
}

template <int NT>
__global__ void __launch_bounds__(NT, (NT >= 1024 ? 1 : 1024 / NT)) batch_k(BucketArgs A) {
  extern __shared__ __align__(16) unsigned char bk_dyn[];
  __shared__ BkShared sh;
  float* sx = reinterpret_cast<float*>(bk_dyn);
  while (true) {
    if (threadIdx.x == 0) sh.item = atomicAdd(A.next, 1u);
    __syncthreads();
    const uint32_t item = sh.item;
    if (item >= A.n_work) break;
    const uint32_t gi = A.work[item];
    if (threadIdx.x < sizeof(GraphDesc) / 4)
      reinterpret_cast<uint32_t*>(&sh.g)[threadIdx.x] =
          reinterpret_cast<const uint32_t*>(A.desc + gi)[threadIdx.x];
    __syncthreads();
    const uint32_t n = sh.g.n;
    if (n) {
      const bool in_smem = n <= A.cap;
      if (A.what & kBkWhatPr) bk_pagerank<NT>(A, sh, sx, gi);
      if (A.what & kBkWhatCc) bk_components<NT>(sh, in_smem ? reinterpret_cast<uint32_t*>(sx) : sh.g.cc);
    } else if (threadIdx.x == 0 && (A.what & kBkWhatPr)) {
      A.iters[gi] = 0;
      A.delta[gi] = 0.0;
    }
    __syncthreads();  // sh.item and sh.g are rewritten for the next graph
  }
}

// ------------------------------------------------------------ build kernels
// Adds each graph's node offset to its local endpoint ids and flags ids that
// are not below the graph's node count.
__global__ void bk_offset_ids_k(const uint32_t* __restrict__ edge_off, uint64_t n_graphs,
                                uint64_t m, const uint32_t* __restrict__ node_off,
                                uint32_t* __restrict__ src, uint32_t* __restrict__ dst,
                                unsigned* __restrict__ bad) {
  for_each_slot_owner(edge_off, n_graphs, m, [&](uint64_t k, uint32_t g) {
    const uint32_t b = node_off[g], ng = node_off[g + 1] - b;
    const uint32_t s = src[k], d = dst[k];
    if (s >= ng || d >= ng) atomicOr(bad, 1u);
    src[k] = b + (s < ng ? s : 0u);
    dst[k] = b + (d < ng ? d : 0u);
  });
}

// Degree class of each row (the plain kernel's classes: in-degree > 64, 32,
// 16, 8, 4, else), keyed by graph: key = graph * 8 + class.
__global__ void bk_class_keys_k(const uint32_t* __restrict__ node_off, uint64_t n_graphs,
                                uint64_t n, const uint32_t* __restrict__ in_off,
                                uint32_t* __restrict__ key) {
  for_each_slot_owner(node_off, n_graphs, n, [&](uint64_t r, uint32_t g) {
    const uint32_t d = in_off[r + 1] - in_off[r];
    const uint32_t c = d > 64u ? 0u : d > 32u ? 1u : d > 16u ? 2u : d > 8u ? 3u : d > 4u ? 4u : 5u;
    key[r] = g * 8u + c;
  });
}

__global__ void bk_local_rows_k(const uint32_t* __restrict__ key, const uint32_t* __restrict__ node_off,
                                uint64_t n, uint32_t* __restrict__ rows) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    rows[i] -= node_off[key[i] >> 3];
}

template <int NT>
void* batch_fn() {
  return (void*)batch_k<NT>;
}

void* batch_fn_for(uint32_t threads) {
  switch (threads) {
    case 128: return batch_fn<128>();
    case 256: return batch_fn<256>();
    case 512: return batch_fn<512>();
    case 1024: return batch_fn<1024>();
    default: return nullptr;
  }
}

void* tc_fn_for(uint32_t threads) {
  switch (threads) {
    case 128: return (void*)tc_batch_k<128>;
    case 256: return (void*)tc_batch_k<256>;
    case 512: return (void*)tc_batch_k<512>;
    default: return nullptr;
  }
}

}  // namespace

}  // namespace ug

using namespace ug;

struct ursa_gpu_batch {
  int device = 0;
  uint64_t n_graphs = 0, n_nodes = 0, n_edges = 0;
  std::vector<uint64_t> h_n, h_m;  // per graph
  std::vector<uint64_t> h_mo;      // oriented undirected edges per graph
  ursa_gpu_topo* topo = nullptr;   // the union (out offsets + in-CSR kept)
  OrientedCsr orient;
  DevArray<uint32_t> rows;
  DevArray<GraphDesc> desc;
  std::vector<GraphDesc> h_desc;  // host copy of desc
  DevArray<double> rank, delta;
  DevArray<float> x;
  DevArray<uint32_t> cc, tri, iters;
  DevArray<uint32_t> work, counters;
  DevArray<uint2> tc_units;
  ursa_gpu_batch_config cfg{};
  bool cfg_set = false;
  // captured launch
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool captured = false;
  ursa_gpu_pagerank_params cap_params{};
  uint32_t cap_what = 0;
  uint32_t n_kernels = 0;
  cudaStream_t side[kBkMaxBuckets + 1] = {};  // [0] is the capture origin
  cudaEvent_t ev[kBkMaxBuckets + 2] = {};     // per branch join, [last] fork
  cudaEvent_t done = nullptr;  // recorded after every launch
  std::mutex mu;

  ~ursa_gpu_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto& s : side)
      if (s) cudaStreamDestroy(s);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (done) cudaEventDestroy(done);
    if (topo) ursa_gpu_topo_free(topo);
  }
};

namespace ug {
namespace {

uint32_t smem_cap_nodes() { return kBkSmemBytesMax / 4u; }

void check_config(const ursa_gpu_batch_config& c) {
  UG_CHECK(c.n_buckets >= 1 && c.n_buckets <= kBkMaxBuckets, URSA_GPU_EINVAL,
           "batch config: n_buckets must be 1..3");
  for (uint32_t b = 0; b < c.n_buckets; b++) {
    UG_CHECK(batch_fn_for(c.threads[b]) != nullptr, URSA_GPU_EINVAL,
             "batch config: threads must be 128, 256, 512 or 1024");
    UG_CHECK(c.cap[b] <= smem_cap_nodes(), URSA_GPU_EINVAL,
             "batch config: a bucket capacity exceeds the shared-memory limit (57,344 nodes)");
    UG_CHECK(b == 0 || c.cap[b] > c.cap[b - 1], URSA_GPU_EINVAL,
             "batch config: bucket capacities must increase");
  }
  UG_CHECK(c.tc_tile >= 1 && c.tc_tile <= 4096, URSA_GPU_EINVAL,
           "batch config: tc_tile must be in [1, 4096] vertices");
  UG_CHECK(tc_fn_for(c.tc_threads) != nullptr, URSA_GPU_EINVAL,
           "batch config: tc_threads must be 128, 256 or 512");
}

ursa_gpu_batch_config default_config() {
  ursa_gpu_batch_config c{};
  c.n_buckets = 3;
  c.cap[0] = 4096;
  c.cap[1] = 16384;
  c.cap[2] = smem_cap_nodes();
  c.threads[0] = 256;
  c.threads[1] = 512;
  c.threads[2] = 1024;
  c.tc_tile = 32;
  c.tc_threads = 256;
  return c;
}

// Work lists: graph g goes to the first bucket whose capacity holds n_g
// (graphs above the last capacity run in the last bucket with global shares);
// inside a bucket, largest edge count first.
void build_work(ursa_gpu_batch* b, const ursa_gpu_batch_config& c, std::vector<uint32_t>& work,
                uint32_t begin[kBkMaxBuckets + 1]) {
  std::vector<std::vector<uint32_t>> lists(c.n_buckets);
  for (uint64_t g = 0; g < b->n_graphs; g++) {
    uint32_t k = c.n_buckets - 1;
    for (uint32_t j = 0; j < c.n_buckets; j++)
      if (b->h_n[g] <= c.cap[j]) {
        k = j;
        break;
      }
    lists[k].push_back((uint32_t)g);
  }
  work.clear();
  for (uint32_t k = 0; k < c.n_buckets; k++) {
    auto& L = lists[k];
    std::stable_sort(L.begin(), L.end(), [&](uint32_t a, uint32_t bb) {
      const uint64_t ca = b->h_m[a] + b->h_mo[a] + b->h_n[a];
      const uint64_t cb = b->h_m[bb] + b->h_mo[bb] + b->h_n[bb];
      return ca > cb;
    });
    begin[k] = (uint32_t)work.size();
    work.insert(work.end(), L.begin(), L.end());
  }
  for (uint32_t k = c.n_buckets; k <= kBkMaxBuckets; k++) begin[k] = (uint32_t)work.size();
}

int resident_ctas(void* fn, uint32_t threads, size_t smem, int device) {
  UG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  UG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, (int)threads, smem));
  UG_CHECK(per_sm > 0, URSA_GPU_ECUDA, "batch kernel cannot be resident with this configuration");
  return per_sm * sm_count(device);
}

// Triangle-count units: graphs with oriented edges, most oriented edges
// first, each cut into runs of unit_len vertices.
void build_tc_units(ursa_gpu_batch* b, uint32_t unit_len, std::vector<uint2>& units) {
  std::vector<uint32_t> order;
  for (uint64_t g = 0; g < b->n_graphs; g++)
    if (b->h_mo[g]) order.push_back((uint32_t)g);
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t x, uint32_t y) { return b->h_mo[x] > b->h_mo[y]; });
  units.clear();
  for (uint32_t g : order)
    for (uint64_t f = 0; f < b->h_n[g]; f += unit_len) units.push_back(make_uint2(g, (uint32_t)f));
}

// Captures, into b->exec: the memsets of the work counters (and of the
// triangle counts), one persistent kernel per non-empty bucket (pagerank and
// components) and the batch-wide triangle kernel, on parallel branches.
void capture(ursa_gpu_batch* b, const ursa_gpu_pagerank_params& p, uint32_t what, cudaStream_t s) {
  const ursa_gpu_batch_config c = b->cfg;
  const bool run_buckets = (what & (kBkWhatPr | kBkWhatCc)) != 0;
  const bool run_tc = (what & kBkWhatTc) != 0;
  // the previous launch (any stream) may still read the work lists
  if (b->done) UG_CUDA(cudaEventSynchronize(b->done));
  std::vector<uint32_t> work;
  uint32_t begin[kBkMaxBuckets + 1] = {0, 0, 0, 0};
  if (run_buckets) build_work(b, c, work, begin);
  if (b->work.n < work.size() + 1) b->work.alloc(work.size() + 1, s);
  if (!work.empty())
    UG_CUDA(cudaMemcpyAsync(b->work.get(), work.data(), work.size() * 4, cudaMemcpyHostToDevice, s));
  std::vector<uint2> units;
  if (run_tc) build_tc_units(b, c.tc_tile, units);
  if (b->tc_units.n < units.size() + 1) b->tc_units.alloc(units.size() + 1, s);
  if (!units.empty())
    UG_CUDA(cudaMemcpyAsync(b->tc_units.get(), units.data(), units.size() * sizeof(uint2),
                            cudaMemcpyHostToDevice, s));
  if (!b->counters.get()) b->counters.alloc(kBkMaxBuckets + 1, s);
  // launch shapes (attributes are set outside the capture)
  int grid[kBkMaxBuckets] = {0};
  size_t smem[kBkMaxBuckets] = {0};
  for (uint32_t k = 0; run_buckets && k < c.n_buckets; k++) {
    const uint32_t nw = begin[k + 1] - begin[k];
    if (!nw) continue;
    smem[k] = (size_t)c.cap[k] * 4u;
    const int resident = resident_ctas(batch_fn_for(c.threads[k]), c.threads[k], smem[k], b->device);
    grid[k] = (int)std::min<uint64_t>((uint64_t)resident, nw);
  }
  int tc_grid = 0;
  uint64_t max_bitmap_n = 1;
  for (uint64_t g = 0; g < b->n_graphs; g++)
    if (b->h_mo[g] && b->h_n[g] <= kTcBitCap) max_bitmap_n = std::max(max_bitmap_n, b->h_n[g]);
  const uint32_t tc_words = (uint32_t)((max_bitmap_n + 31) / 32);
  const size_t tc_smem = (size_t)(c.tc_threads / 32) * tc_words * 4u;
  if (!units.empty()) {
    const int resident = resident_ctas(tc_fn_for(c.tc_threads), c.tc_threads, tc_smem, b->device);
    const uint64_t want = (units.size() + c.tc_threads / 32 - 1) / (c.tc_threads / 32);
    tc_grid = (int)std::min<uint64_t>((uint64_t)resident, want);
  }
  UG_CUDA(cudaStreamSynchronize(s));
  for (auto& st : b->side)
    if (!st) UG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  for (auto& e : b->ev)
    if (!e) UG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  b->captured = false;
  b->n_kernels = 0;
  cudaStream_t cs = b->side[0];
  cudaEvent_t fork = b->ev[kBkMaxBuckets + 1];
  UG_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = cudaSuccess;
  auto rec = [&](cudaError_t e) {
    if (err == cudaSuccess && e != cudaSuccess) err = e;
  };
  rec(cudaMemsetAsync(b->counters.get(), 0, (kBkMaxBuckets + 1) * sizeof(uint32_t), cs));
  if (run_tc && b->n_nodes)
    rec(cudaMemsetAsync(b->tri.get(), 0, b->n_nodes * sizeof(uint32_t), cs));
  rec(cudaEventRecord(fork, cs));
  // the largest-graph bucket first, on the origin stream, so its long CTAs
  // start first; the other buckets and the triangle kernel fork onto side
  // streams and join back
  for (int k = (int)c.n_buckets - 1; k >= 0; k--) {
    if (!grid[k]) continue;
    const bool origin = k == (int)c.n_buckets - 1;
    cudaStream_t ks = origin ? cs : b->side[k + 1];  // k + 1 <= 2 here
    if (!origin) rec(cudaStreamWaitEvent(ks, fork, 0));
    BucketArgs a;
    a.desc = b->desc.get();
    a.work = b->work.get() + begin[k];
    a.n_work = begin[k + 1] - begin[k];
    a.next = b->counters.get() + k;
    a.cap = c.cap[k];
    a.what = what;
    a.max_iter = p.max_iter;
    a.damping = p.damping;
    a.tol = p.tol;
    a.iters = b->iters.get();
    a.delta = b->delta.get();
    void* args[] = {&a};
    rec(cudaLaunchKernel(batch_fn_for(c.threads[k]), dim3(grid[k]), dim3(c.threads[k]), args,
                         smem[k], ks));
    b->n_kernels++;
    if (!origin) {
      rec(cudaEventRecord(b->ev[k], ks));
      rec(cudaStreamWaitEvent(cs, b->ev[k], 0));
    }
  }
  if (tc_grid) {
    cudaStream_t ts = b->side[kBkMaxBuckets];
    rec(cudaStreamWaitEvent(ts, fork, 0));
    TcArgs ta;
    ta.desc = b->desc.get();
    ta.units = b->tc_units.get();
    ta.n_units = (uint32_t)units.size();
    ta.unit_len = c.tc_tile;
    ta.words = tc_words;
    ta.next = b->counters.get() + kBkMaxBuckets;
    void* args[] = {&ta};
    rec(cudaLaunchKernel(tc_fn_for(c.tc_threads), dim3(tc_grid), dim3(c.tc_threads), args, tc_smem,
                         ts));
    b->n_kernels++;
    rec(cudaEventRecord(b->ev[kBkMaxBuckets], ts));
    rec(cudaStreamWaitEvent(cs, b->ev[kBkMaxBuckets], 0));
  }
  cudaGraph_t graph = nullptr;
  cudaError_t end = cudaStreamEndCapture(cs, &graph);
  rec(end);
  if (err != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    UG_CUDA(err);
  }
  b->graph = graph;
  UG_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  b->captured = true;
  b->cap_params = p;
  b->cap_what = what;
}

bool same_params(const ursa_gpu_pagerank_params& a, const ursa_gpu_pagerank_params& b) {
  return a.damping == b.damping && a.tol == b.tol && a.max_iter == b.max_iter;
}

// One launch of the captured graph on s (re-captured when the parameters,
// the algorithm mask or the configuration changed).
void batch_launch(ursa_gpu_batch* b, const ursa_gpu_pagerank_params& p, uint32_t what,
                  cudaStream_t s) {
  if (!b->cfg_set) {
    b->cfg = default_config();
    b->cfg_set = true;
  }
  if (!b->captured || !same_params(p, b->cap_params) || what != b->cap_what) capture(b, p, what, s);
  UG_CUDA(cudaGraphLaunch(b->exec, s));
  for (uint32_t k = 0; k < b->n_kernels; k++) count_launch();
  if (!b->done) UG_CUDA(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
  UG_CUDA(cudaEventRecord(b->done, s));
}

}  // namespace

void* batch_kernel_for(uint32_t threads) { return batch_fn_for(threads); }

int batch_kernel_resident(uint32_t threads, size_t smem, int device) {
  return resident_ctas(batch_fn_for(threads), threads, smem, device);
}

const GraphDesc* batch_host_desc(const ursa_gpu_batch* b, uint64_t g) {
  return b && g < b->h_desc.size() ? &b->h_desc[g] : nullptr;
}

}  // namespace ug

extern "C" {

int ursa_gpu_batch_build(uint64_t n_graphs, const uint64_t* node_counts,
                         const uint64_t* edge_counts, const uint32_t* src, const uint32_t* dst,
                         ursa_gpu_batch** out) {
  return guard([&] {
    UG_CHECK(out, URSA_GPU_EINVAL, "out is NULL");
    *out = nullptr;
    UG_CHECK(n_graphs == 0 || (node_counts && edge_counts), URSA_GPU_EINVAL,
             "node_counts / edge_counts is NULL");
    UG_CHECK(n_graphs < (1ull << 29), URSA_GPU_EINVAL, "more than 2^29 graphs in one batch");
    uint64_t N = 0, M = 0;
    std::vector<uint32_t> node_off(n_graphs + 1), edge_off(n_graphs + 1);
    for (uint64_t g = 0; g < n_graphs; g++) {
      node_off[g] = (uint32_t)N;
      edge_off[g] = (uint32_t)M;
      N += node_counts[g];
      M += edge_counts[g];
      UG_CHECK(N <= 0xFFFFFFFFull, URSA_GPU_EINVAL, "batch: more than u32::MAX nodes in total");
      UG_CHECK(M <= 0xFFFFFFFFull, URSA_GPU_EINVAL, "batch: more than u32::MAX edges in total");
    }
    node_off[n_graphs] = (uint32_t)N;
    edge_off[n_graphs] = (uint32_t)M;
    if (M) UG_CHECK(src && dst, URSA_GPU_EINVAL, "src / dst is NULL");
    int dev = 0;
    UG_CUDA(cudaGetDevice(&dev));
    cudaStream_t s = thread_stream(dev);
    std::unique_ptr<ursa_gpu_batch> b(new ursa_gpu_batch());
    b->device = dev;
    b->n_graphs = n_graphs;
    b->n_nodes = N;
    b->n_edges = M;
    b->h_n.assign(node_counts, node_counts + n_graphs);
    b->h_m.assign(edge_counts, edge_counts + n_graphs);

    Scratch<uint32_t> d_node_off(n_graphs + 1, s), d_edge_off(n_graphs + 1, s);
    UG_CUDA(cudaMemcpyAsync(d_node_off.get(), node_off.data(), (n_graphs + 1) * 4,
                            cudaMemcpyHostToDevice, s));
    UG_CUDA(cudaMemcpyAsync(d_edge_off.get(), edge_off.data(), (n_graphs + 1) * 4,
                            cudaMemcpyHostToDevice, s));
    {
      Scratch<uint32_t> d_src(M, s), d_dst(M, s);
      if (M) {
        UG_CUDA(cudaMemcpyAsync(d_src.get(), src, M * 4, cudaMemcpyHostToDevice, s));
        UG_CUDA(cudaMemcpyAsync(d_dst.get(), dst, M * 4, cudaMemcpyHostToDevice, s));
        Scratch<unsigned> bad(1, s);
        UG_CUDA(cudaMemsetAsync(bad.get(), 0, 4, s));
        bk_offset_ids_k<<<grid_for(M), kBlock, 0, s>>>(d_edge_off.get(), n_graphs, M,
                                                       d_node_off.get(), d_src.get(), d_dst.get(),
                                                       bad.get());
        UG_LAUNCH_CHECK();
        unsigned hb = 0;
        UG_CUDA(cudaMemcpyAsync(&hb, bad.get(), 4, cudaMemcpyDeviceToHost, s));
        UG_CUDA(cudaStreamSynchronize(s));
        UG_CHECK(hb == 0, URSA_GPU_EINVAL,
                 "batch: a local endpoint id is not below its graph's node count");
      }
      if (N) topo_from_device(N, d_src.get(), d_dst.get(), M, s, dev, &b->topo);
    }
    b->h_mo.assign(n_graphs, 0);
    std::vector<uint32_t> cls_off_h(n_graphs * 8 + 1, 0);
    TopoImpl* t = b->topo ? &b->topo->impl : nullptr;
    b->rows.alloc(N ? N : 1, s);
    if (N) {
      orient_build(t, b->orient, s);
      {  // per-graph oriented edge counts (work-list ordering)
        std::vector<uint32_t> tmp(N + 1);
        UG_CUDA(cudaMemcpyAsync(tmp.data(), b->orient.off.get(), (N + 1) * 4,
                                cudaMemcpyDeviceToHost, s));
        UG_CUDA(cudaStreamSynchronize(s));
        for (uint64_t g = 0; g < n_graphs; g++)
          b->h_mo[g] = tmp[node_off[g + 1]] - tmp[node_off[g]];
      }
      // the batch keeps the out offsets, the in-CSR and the oriented CSR only
      t->und_off.release();
      t->und_tgt.release();
      t->has_und = false;
      t->out.tgt.release();
      t->out.eid.release();
      t->in.eid.release();
      // rows grouped by (graph, degree class); class offsets per graph
      Scratch<uint32_t> key(N, s), key_sorted(N, s), cls_off(n_graphs * 8 + 1, s);
      bk_class_keys_k<<<grid_for(N), kBlock, 0, s>>>(d_node_off.get(), n_graphs, N,
                                                      t->in.off.get(), key.get());
      UG_LAUNCH_CHECK();
      radix_sort_pairs(key.get(), nullptr, N, bits_for(n_graphs * 8), key_sorted.get(),
                       b->rows.get(), nullptr, nullptr, s);
      offsets_from_sorted(key_sorted.get(), N, n_graphs * 8, cls_off.get(), s);
      bk_local_rows_k<<<grid_for(N), kBlock, 0, s>>>(key_sorted.get(), d_node_off.get(), N,
                                                      b->rows.get());
      UG_LAUNCH_CHECK();
      UG_CUDA(cudaMemcpyAsync(cls_off_h.data(), cls_off.get(), (n_graphs * 8 + 1) * 4,
                              cudaMemcpyDeviceToHost, s));
      UG_CUDA(cudaStreamSynchronize(s));
    }
    // results and shares
    const uint64_t n_pad = (N + 3) & ~3ull;
    b->rank.alloc(N ? N : 1, s);
    b->x.alloc(2 * (n_pad ? n_pad : 4), s);
    b->cc.alloc(N ? N : 1, s);
    b->tri.alloc(N ? N : 1, s);
    b->iters.alloc(n_graphs ? n_graphs : 1, s);
    b->delta.alloc(n_graphs ? n_graphs : 1, s);
    std::vector<GraphDesc> desc(n_graphs);
    for (uint64_t g = 0; g < n_graphs; g++) {
      GraphDesc& d = desc[g];
      std::memset(&d, 0, sizeof(d));
      const uint32_t base = node_off[g];
      d.n = (uint32_t)node_counts[g];
      if (d.n == 0) continue;  // never dereferenced
      d.in_off = t->in.off.get() + base;
      d.in_src = t->in.tgt.get();
      d.out_off = t->out.off.get() + base;
      d.o_off = b->orient.off.get() + base;
      d.o_tgt = b->orient.tgt.get();
      d.rows = b->rows.get() + base;
      d.rank = b->rank.get() + base;
      d.x0 = b->x.get() + base;
      d.x1 = b->x.get() + n_pad + base;
      d.cc = b->cc.get() + base;
      d.tri = b->tri.get() + base;
      for (int c = 0; c < 6; c++) d.cls[c] = cls_off_h[g * 8 + c] - base;
      d.cls[6] = d.cls[7] = d.n;
      d.id_base = base;
    }
    b->h_desc = desc;
    b->desc.alloc(n_graphs ? n_graphs : 1, s);
    if (n_graphs)
      UG_CUDA(cudaMemcpyAsync(b->desc.get(), desc.data(), n_graphs * sizeof(GraphDesc),
                              cudaMemcpyHostToDevice, s));
    UG_CUDA(cudaStreamSynchronize(s));
    *out = b.release();
  });
}

void ursa_gpu_batch_free(ursa_gpu_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->done) cudaEventSynchronize(b->done);
  delete b;
}

uint64_t ursa_gpu_batch_n_graphs(const ursa_gpu_batch* b) { return b ? b->n_graphs : 0; }
uint64_t ursa_gpu_batch_n_nodes(const ursa_gpu_batch* b) { return b ? b->n_nodes : 0; }
uint64_t ursa_gpu_batch_n_edges(const ursa_gpu_batch* b) { return b ? b->n_edges : 0; }

uint64_t ursa_gpu_batch_device_bytes(const ursa_gpu_batch* b) {
  if (!b) return 0;
  uint64_t bytes = ursa_gpu_topo_device_bytes(b->topo);
  bytes += 4ull * (b->orient.off.n + b->orient.tgt.n + b->rows.n + b->cc.n + b->tri.n + b->iters.n +
                   b->work.n + b->counters.n);
  bytes += 8ull * (b->rank.n + b->delta.n) + 4ull * b->x.n + sizeof(GraphDesc) * b->desc.n;
  return bytes;
}

int ursa_gpu_batch_set_config(ursa_gpu_batch* b, const ursa_gpu_batch_config* cfg) {
  return guard([&] {
    UG_CHECK(b && cfg, URSA_GPU_EINVAL, "batch / config is NULL");
    check_config(*cfg);
    std::lock_guard<std::mutex> g(b->mu);
    b->cfg = *cfg;
    b->cfg_set = true;
    b->captured = false;
  });
}

int ursa_gpu_batch_get_config(ursa_gpu_batch* b, ursa_gpu_batch_config* cfg) {
  return guard([&] {
    UG_CHECK(b && cfg, URSA_GPU_EINVAL, "batch / config is NULL");
    std::lock_guard<std::mutex> g(b->mu);
    *cfg = b->cfg_set ? b->cfg : default_config();
  });
}

int ursa_gpu_batch_run(ursa_gpu_batch* b, const ursa_gpu_pagerank_params* params, uint32_t what,
                       void* stream) {
  return guard([&] {
    UG_CHECK(b && params, URSA_GPU_EINVAL, "batch / params is NULL");
    UG_CHECK(what != 0 && (what & ~7u) == 0, URSA_GPU_EINVAL,
             "batch: what must combine URSA_GPU_BATCH_PAGERANK / _COMPONENTS / _TRIANGLES");
    UG_CHECK(params->damping >= 0.0 && params->damping <= 1.0, URSA_GPU_EINVAL,
             "damping must be in [0, 1]");
    std::lock_guard<std::mutex> g(b->mu);
    UG_CUDA(cudaSetDevice(b->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream(b->device);
    if (b->n_graphs == 0) return;
    batch_launch(b, *params, what, s);
    if (!stream) UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_batch_tune(ursa_gpu_batch* b, const ursa_gpu_pagerank_params* params, uint32_t what,
                        ursa_gpu_batch_config* chosen, float* best_ms) {
  return guard([&] {
    UG_CHECK(b && params, URSA_GPU_EINVAL, "batch / params is NULL");
    UG_CHECK(what != 0 && (what & ~7u) == 0, URSA_GPU_EINVAL, "batch: invalid algorithm mask");
    std::lock_guard<std::mutex> g(b->mu);
    UG_CUDA(cudaSetDevice(b->device));
    cudaStream_t s = thread_stream(b->device);
    if (!b->cfg_set) b->cfg = default_config();
    b->cfg_set = true;
    cudaEvent_t e0, e1;
    UG_CUDA(cudaEventCreate(&e0));
    UG_CUDA(cudaEventCreate(&e1));
    // time of one launch of the captured graph for a configuration: the
    // minimum of two launches after one warm-up launch
    auto time_cfg = [&](const ursa_gpu_batch_config& c) -> float {
      b->cfg = c;
      b->captured = false;
      batch_launch(b, *params, what, s);
      float best = 1e30f;
      for (int r = 0; r < 2; r++) {
        UG_CUDA(cudaEventRecord(e0, s));
        batch_launch(b, *params, what, s);
        UG_CUDA(cudaEventRecord(e1, s));
        UG_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        UG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best = std::min(best, ms);
      }
      return best;
    };
    ursa_gpu_batch_config best = b->cfg;
    float best_t = 0.f;
    try {
      if (b->n_graphs) {
        best_t = time_cfg(best);
        const uint32_t big = smem_cap_nodes();
        // 1) bucket capacities
        const uint32_t caps[][3] = {{big, 0, 0},         {4096, big, 0},     {8192, big, 0},
                                    {2048, 16384, big},  {4096, 16384, big}, {4096, 24576, big},
                                    {8192, 32768, big}};
        const uint32_t ncaps[] = {1, 2, 2, 3, 3, 3, 3};
        const uint32_t def_threads[3][3] = {{1024, 0, 0}, {256, 1024, 0}, {256, 512, 1024}};
        for (size_t i = 0; (what & (kBkWhatPr | kBkWhatCc)) && i < sizeof(ncaps) / sizeof(ncaps[0]);
             i++) {
          ursa_gpu_batch_config c = best;
          c.n_buckets = ncaps[i];
          for (uint32_t k = 0; k < 3; k++) {
            c.cap[k] = caps[i][k];
            c.threads[k] = def_threads[ncaps[i] - 1][k];
          }
          if (std::memcmp(&c, &best, sizeof(c)) == 0) continue;
          const float t = time_cfg(c);
          if (t < best_t) {
            best_t = t;
            best = c;
          }
        }
        // 2) CTA size per bucket, 3) triangle kernel CTA size and unit; two rounds
        const uint32_t ths[] = {128, 256, 512, 1024};
        const uint32_t tc_ths[] = {128, 256, 512};
        const uint32_t tiles[] = {8, 16, 32, 64, 128};
        auto try_cfg = [&](const ursa_gpu_batch_config& c) {
          const float t = time_cfg(c);
          if (t < best_t) {
            best_t = t;
            best = c;
          }
        };
        for (int round = 0; round < 2; round++) {
          if (what & (kBkWhatPr | kBkWhatCc))
            for (uint32_t k = 0; k < best.n_buckets; k++)
              for (uint32_t th : ths) {
                if (th == best.threads[k]) continue;
                ursa_gpu_batch_config c = best;
                c.threads[k] = th;
                try_cfg(c);
              }
          if (what & kBkWhatTc) {
            for (uint32_t th : tc_ths) {
              if (th == best.tc_threads) continue;
              ursa_gpu_batch_config c = best;
              c.tc_threads = th;
              try_cfg(c);
            }
            for (uint32_t tile : tiles) {
              if (tile == best.tc_tile) continue;
              ursa_gpu_batch_config c = best;
              c.tc_tile = tile;
              try_cfg(c);
            }
          }
        }
      }
    } catch (...) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->cfg = best;
    b->captured = false;
    if (chosen) *chosen = best;
    if (best_ms) *best_ms = best_t;
  });
}

int ursa_gpu_batch_results(ursa_gpu_batch* b, double* pagerank, uint32_t* components,
                           uint32_t* triangles, uint32_t* pr_iterations, double* pr_last_delta) {
  return guard([&] {
    UG_CHECK(b, URSA_GPU_EINVAL, "batch is NULL");
    std::lock_guard<std::mutex> g(b->mu);
    UG_CUDA(cudaSetDevice(b->device));
    cudaStream_t s = thread_stream(b->device);
    const uint64_t N = b->n_nodes, G = b->n_graphs;
    if (b->done) UG_CUDA(cudaStreamWaitEvent(s, b->done, 0));
    if (pagerank && N) UG_CUDA(cudaMemcpyAsync(pagerank, b->rank.get(), N * 8, cudaMemcpyDeviceToHost, s));
    if (components && N) UG_CUDA(cudaMemcpyAsync(components, b->cc.get(), N * 4, cudaMemcpyDeviceToHost, s));
    if (triangles && N) UG_CUDA(cudaMemcpyAsync(triangles, b->tri.get(), N * 4, cudaMemcpyDeviceToHost, s));
    if (pr_iterations && G)
      UG_CUDA(cudaMemcpyAsync(pr_iterations, b->iters.get(), G * 4, cudaMemcpyDeviceToHost, s));
    if (pr_last_delta && G)
      UG_CUDA(cudaMemcpyAsync(pr_last_delta, b->delta.get(), G * 8, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_batch_device_results(ursa_gpu_batch* b, const double** pagerank,
                                  const uint32_t** components, const uint32_t** triangles) {
  return guard([&] {
    UG_CHECK(b, URSA_GPU_EINVAL, "batch is NULL");
    if (pagerank) *pagerank = b->rank.get();
    if (components) *components = b->cc.get();
    if (triangles) *triangles = b->tri.get();
  });
}

}  // extern "C"
