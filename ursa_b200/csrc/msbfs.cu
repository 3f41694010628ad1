// msbfs.cu -- BFS from many sources at once: closeness
// (ursa-core/src/algo/closeness.rs:69-135) and the path statistics
// avg_path_length / diameter (ursa-plan/src/stats.rs:82-170).
//
// Sources are taken 64 at a time; bit b of a node's 64-bit masks belongs to
// source b of the batch.  One persistent cooperative kernel runs a group of
// batches; each BFS level (following out-edges) ends in a bounded grid
// barrier and goes one of two ways (direction-optimising BFS):
//   top-down while the frontier's out-edges are below m / 8: each frontier
//   node ORs its mask into acc[w] for out-edges v -> w whose target lacks some
//   of its sources; after a barrier every w settles new = acc[w] & ~visited[w];
//   bottom-up otherwise: each w with sources still to find
//   (need = active & ~visited[w]) ORs its in-neighbours' frontier masks,
//   stopping as soon as every needed bit is found; new = acc & need.
//   Nodes with at most 32 edges to scan are handled by one lane, up to
//   kMsHub by the whole warp; the in-edges of longer rows are cut into
//   kMsChunk-edge chunks that any warp takes, ORed into a per-row
//   accumulator and settled after one more barrier (a warp scanning long
//   rows one after another held every other warp at the level barrier).
//   visited[w] |= new; next[w] = new.
// A source that reached no new node on a level is finished and leaves the
// active mask.  Per source, the number of nodes first reached on the level is
// a column popcount of the new masks (one warp ballot per bit), summed per
// block in shared memory and per grid in a level-indexed counter row, which
// also carries the new frontier's out-edge count for the next direction.
// Block 0 folds the counts after the barrier: reach[b] += count[b];
// dist_sum[b] += level * count[b]; max_dist[b] = level where count[b] > 0.
// The folds are integer and exact, so the reference's results follow
// bit-for-bit: closeness = reach / sum (an i64 sum in closeness_one), and the
// stats' f64 sums of integer distances are exact while the total stays below
// 2^53 (checked).  A level with no new node ends the batch.
#include <algorithm>
#include <cstring>
#include <cmath>
#include <vector>

#include "frontier.cuh"
#include "primitives.cuh"

namespace ug {

namespace {

constexpr int kMsBlock = 256;
constexpr int kMsWarps = kMsBlock / 32;
constexpr uint64_t kMsSourcesPerLaunch = 1024;
constexpr uint64_t kMsWaitNs = 5000000000ull;  // one grid-barrier wait
constexpr uint64_t kMsPushDiv = 8;  // push while the frontier's out-edges are below m / 8
constexpr uint32_t kMsHub = 64;    // in-degree above which a node's scan is split
constexpr uint32_t kMsChunk = 128;  // in-edges per chunk of a split scan

// W 64-bit words per node: bit j of word q belongs to source 64 q + j of the
// batch.  A node's W words are contiguous (one 32-byte sector for W = 4).
template <int W>
struct Msk {
  unsigned long long v[W];
};

template <int W>
__device__ __forceinline__ Msk<W> mk_zero() {
  Msk<W> r;
#pragma unroll
  for (int q = 0; q < W; q++) r.v[q] = 0;
  return r;
}
template <int W>
__device__ __forceinline__ Msk<W> mk_load(const unsigned long long* p, uint64_t node) {
  Msk<W> r;
  p += node * W;
  if constexpr (W == 1) {
    r.v[0] = __ldcg(p);
  } else {
#pragma unroll
    for (int q = 0; q < W; q += 2) {
      const ulonglong2 x = __ldcg(reinterpret_cast<const ulonglong2*>(p + q));
      r.v[q] = x.x;
      r.v[q + 1] = x.y;
    }
  }
  return r;
}
template <int W>
__device__ __forceinline__ void mk_store(unsigned long long* p, uint64_t node, const Msk<W>& m) {
  p += node * W;
  if constexpr (W == 1) {
    p[0] = m.v[0];
  } else {
#pragma unroll
    for (int q = 0; q < W; q += 2)
      *reinterpret_cast<ulonglong2*>(p + q) = make_ulonglong2(m.v[q], m.v[q + 1]);
  }
}
template <int W>
__device__ __forceinline__ bool mk_any(const Msk<W>& m) {
  unsigned long long x = 0;
#pragma unroll
  for (int q = 0; q < W; q++) x |= m.v[q];
  return x != 0;
}
template <int W>
__device__ __forceinline__ Msk<W> mk_andnot(const Msk<W>& a, const Msk<W>& b) {  // a & ~b
  Msk<W> r;
#pragma unroll
  for (int q = 0; q < W; q++) r.v[q] = a.v[q] & ~b.v[q];
  return r;
}
template <int W>
__device__ __forceinline__ void mk_or(Msk<W>& a, const Msk<W>& b) {
#pragma unroll
  for (int q = 0; q < W; q++) a.v[q] |= b.v[q];
}
template <int W>
__device__ __forceinline__ bool mk_covers(const Msk<W>& acc, const Msk<W>& need) {  // need ⊆ acc
  unsigned long long x = 0;
#pragma unroll
  for (int q = 0; q < W; q++) x |= need.v[q] & ~acc.v[q];
  return x == 0;
}
template <int W>
__device__ __forceinline__ Msk<W> mk_shfl(const Msk<W>& m, int j) {
  Msk<W> r;
#pragma unroll
  for (int q = 0; q < W; q++) r.v[q] = __shfl_sync(0xffffffffu, m.v[q], j);
  return r;
}
__device__ __forceinline__ unsigned long long warp_or64(unsigned long long v) {
  const unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)v);
  const unsigned hi = __reduce_or_sync(0xffffffffu, (unsigned)(v >> 32));
  return ((unsigned long long)hi << 32) | lo;
}

struct MsArgs {
  // pull: the CSR whose rows list the nodes that reach each node in one step
  // (the in-CSR when following out-edges); push: the CSR of the steps taken
  const uint32_t* in_off;
  const uint32_t* in_src;
  const uint32_t* out_off;
  const uint32_t* out_tgt;
  uint64_t n, m;  // m: rows of the push CSR
  int32_t* dist;  // optional: n_sources rows of n hop distances (-1 preset)
  const uint32_t* sources;  // n_sources ids < n
  uint64_t n_sources;
  uint64_t b_begin, b_end;  // batches of 64 W sources run by this launch
  unsigned long long* visited;  // n W words each
  unsigned long long* fr0;      // frontier masks, odd levels' input
  unsigned long long* fr1;      // even levels' input
  unsigned long long* acc;      // pushed masks of a top-down level; all zero between levels
  const uint32_t* hubs;         // nodes with in-degree > kMsHub, ascending
  uint64_t n_hubs;
  const uint32_t* chunk_hub;    // per kMsChunk-edge chunk of a hub's in-edges: hub index,
  const uint32_t* chunk_lo;     //   first in-CSR slot
  uint64_t n_chunks;
  unsigned long long* hacc;     // n_hubs x W: OR of a bottom-up level's chunk results; zero between levels
  unsigned long long* count;    // 3 rows of 64 W + 8, row = level % 3; [64 W] = frontier out-edges
  unsigned long long* reach;
  unsigned long long* dsum;
  uint32_t* maxd;
  unsigned* bar;  // grid barrier count, generation
  int* err;
};

// Top-down half of a level: every frontier node v ORs its mask into acc[w]
// for each out-edge v -> w whose target still lacks some of those sources.
template <int W>
__device__ __forceinline__ void ms_push(const MsArgs& a, const unsigned long long* cur, uint64_t gwarp,
                                        uint64_t nwarps, int lane) {
  for (uint64_t c0 = gwarp * 32; c0 < a.n; c0 += nwarps * 32) {
    const uint64_t v = c0 + lane;
    Msk<W> f = mk_zero<W>();
    uint32_t e0 = 0, e1 = 0;
    if (v < a.n) {
      f = mk_load<W>(cur, v);
      if (mk_any(f)) {
        e0 = __ldg(&a.out_off[v]);
        e1 = __ldg(&a.out_off[v + 1]);
      }
    }
    const bool heavy = e1 - e0 > 32;
    if (!heavy) {
      for (uint32_t e = e0; e < e1; e++) {
        const uint32_t w = __ldg(&a.out_tgt[e]);
        const Msk<W> add = mk_andnot(f, mk_load<W>(a.visited, w));
#pragma unroll
        for (int q = 0; q < W; q++)
          if (add.v[q]) atomicOr(&a.acc[(uint64_t)w * W + q], add.v[q]);
      }
    }
    unsigned hm = __ballot_sync(0xffffffffu, heavy);
    while (hm) {
      const int j = __ffs(hm) - 1;
      hm &= hm - 1;
      const uint32_t h0 = __shfl_sync(0xffffffffu, e0, j), h1 = __shfl_sync(0xffffffffu, e1, j);
      const Msk<W> hf = mk_shfl(f, j);
      for (uint32_t e = h0 + lane; e < h1; e += 32) {
        const uint32_t w = __ldg(&a.out_tgt[e]);
        const Msk<W> add = mk_andnot(hf, mk_load<W>(a.visited, w));
#pragma unroll
        for (int q = 0; q < W; q++)
          if (add.v[q]) atomicOr(&a.acc[(uint64_t)w * W + q], add.v[q]);
      }
    }
  }
}

// Settles node w (lanes with valid) for this level: visited |= new,
// next[w] = new, and adds the per-source counts and the new nodes'
// out-edges to the block's tallies.  Every lane of the warp calls it.
template <int W>
__device__ __forceinline__ void ms_settle(const MsArgs& a, unsigned long long* nxt, uint64_t w, bool valid,
                                          const Msk<W>& vis, const Msk<W>& nw, unsigned* sc,
                                          unsigned long long* s_mf, int lane, uint32_t level, uint64_t s0) {
  unsigned long long od = 0;
  const bool got = mk_any(nw);
  if (valid) {
    if (got) {
      Msk<W> nv = vis;
      mk_or(nv, nw);
      mk_store<W>(a.visited, w, nv);
      od = __ldg(&a.out_off[w + 1]) - __ldg(&a.out_off[w]);
      if (a.dist) {
#pragma unroll
        for (int q = 0; q < W; q++)
          for (unsigned long long x = nw.v[q]; x; x &= x - 1)
            a.dist[(s0 + 64 * q + (__ffsll((long long)x) - 1)) * a.n + w] = (int32_t)level;
      }
    }
    mk_store<W>(nxt, w, nw);
  }
  if (__any_sync(0xffffffffu, got)) {
#pragma unroll
    for (int q = 0; q < W; q++) {
      if (!__any_sync(0xffffffffu, nw.v[q] != 0)) continue;
#pragma unroll 8
      for (int b = 0; b < 64; b++) {
        const unsigned c = __popc(__ballot_sync(0xffffffffu, (nw.v[q] >> b) & 1ull));
        if (lane == 0 && c) atomicAdd(&sc[64 * q + b], c);
      }
    }
    for (int o = 16; o; o >>= 1) od += __shfl_down_sync(0xffffffffu, od, o);
    if (lane == 0) atomicAdd(s_mf, od);
  }
}

// Bottom-up scan of one chunk of a hub's in-edges: ORs the frontier masks of
// up to kMsChunk in-neighbours (stopping once every needed source is found)
// into hacc of the hub.  One warp per chunk.
template <int W>
__device__ __forceinline__ void ms_hub_chunk(const MsArgs& a, const unsigned long long* cur,
                                             const Msk<W>& active, uint64_t c, int lane) {
  const uint32_t h = __ldg(&a.chunk_hub[c]);
  const uint32_t w = __ldg(&a.hubs[h]);
  const Msk<W> need = mk_andnot(active, mk_load<W>(a.visited, w));
  if (!mk_any(need)) return;  // warp-uniform: one chunk per warp
  const uint32_t e0 = __ldg(&a.chunk_lo[c]);
  const uint32_t end = __ldg(&a.in_off[w + 1]);
  const uint32_t e1 = end - e0 > kMsChunk ? e0 + kMsChunk : end;
  Msk<W> acc = mk_zero<W>();
  constexpr int U = W == 1 ? 4 : 2;  // in-edges per lane per step
  for (uint32_t e = e0; e < e1; e += 32 * U) {
    Msk<W> f = mk_zero<W>();
#pragma unroll
    for (int q = 0; q < U; q++) {
      const uint32_t x = e + q * 32 + lane;
      if (x < e1) mk_or(f, mk_load<W>(cur, __ldg(&a.in_src[x])));
    }
#pragma unroll
    for (int q = 0; q < W; q++) acc.v[q] |= warp_or64(f.v[q]);
    if (mk_covers(acc, need)) break;
  }
  unsigned long long y = 0;  // lane q ORs word q
#pragma unroll
  for (int q = 0; q < W; q++)
    if (lane == q) y = acc.v[q] & need.v[q];
  if (y) atomicOr(&a.hacc[(uint64_t)h * W + lane], y);
}

template <int W>
__global__ void __launch_bounds__(kMsBlock) ms_persist_k(MsArgs a) {
  constexpr int S = 64 * W;     // sources per batch
  constexpr int R = 64 * W + 8;  // counter row length
  static_assert(S <= kMsBlock, "one thread per source of a batch");
  __shared__ unsigned sc[S];
  __shared__ unsigned long long s_mf;
  __shared__ unsigned s_act[2 * W];
  const int lane = threadIdx.x & 31;
  const uint64_t n = a.n;
  const uint64_t nwarps = (uint64_t)gridDim.x * kMsWarps;
  const uint64_t gwarp = (uint64_t)blockIdx.x * kMsWarps + (threadIdx.x >> 5);
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (uint64_t bt = a.b_begin; bt < a.b_end; bt++) {
    const uint64_t s0 = bt * S;
    const uint64_t left = a.n_sources - s0;
    const uint32_t k = left < (uint64_t)S ? (uint32_t)left : (uint32_t)S;
    Msk<W> active;  // sources whose search still grows
#pragma unroll
    for (int q = 0; q < W; q++) {
      const int bits = (int)k - 64 * q;
      active.v[q] = bits >= 64 ? ~0ull : (bits <= 0 ? 0ull : ((1ull << bits) - 1));
    }
    for (uint64_t x = gtid; x < n * W; x += nthreads) {
      a.visited[x] = 0;
      a.fr0[x] = 0;
    }
    grid_barrier(a.bar, a.bar + 1, gridDim.x, a.err, kMsWaitNs);
    if (*(volatile int*)a.err) return;
    if (blockIdx.x == 0) {  // every block has read the previous batch's last counter row
      for (int x = threadIdx.x; x < 3 * R; x += kMsBlock) a.count[x] = 0;
      __syncthreads();
      if (threadIdx.x < k) {
        const uint32_t src = a.sources[s0 + threadIdx.x];
        const uint64_t wd = (uint64_t)src * W + (threadIdx.x >> 6);
        atomicOr(&a.visited[wd], 1ull << (threadIdx.x & 63));
        atomicOr(&a.fr0[wd], 1ull << (threadIdx.x & 63));
        atomicAdd(&a.count[S], (unsigned long long)(a.out_off[src + 1] - a.out_off[src]));
        if (a.dist) a.dist[(s0 + threadIdx.x) * n + src] = 0;
      }
    }
    grid_barrier(a.bar, a.bar + 1, gridDim.x, a.err, kMsWaitNs);
    if (*(volatile int*)a.err) return;
    unsigned long long reach = 0, dsum = 0;  // block 0, thread b < k: source s0 + b
    uint32_t maxd = 0;
    for (uint32_t level = 1;; level++) {
      const unsigned long long* cur = (level & 1) ? a.fr0 : a.fr1;
      unsigned long long* nxt = (level & 1) ? a.fr1 : a.fr0;
      unsigned long long* row = a.count + (level % 3) * R;
      const unsigned long long mf = __ldcg(&a.count[((level - 1) % 3) * R + S]);
      const bool push = mf * kMsPushDiv < a.m;
      for (int x = threadIdx.x; x < S; x += kMsBlock) sc[x] = 0;
      if (threadIdx.x == 0) s_mf = 0;
      // row (level + 1) % 3 was last read before the previous barrier
      if (blockIdx.x == 0)
        for (int x = threadIdx.x; x < R; x += kMsBlock) a.count[((level + 1) % 3) * R + x] = 0;
      __syncthreads();
      if (push) {
        ms_push<W>(a, cur, gwarp, nwarps, lane);
        grid_barrier(a.bar, a.bar + 1, gridDim.x, a.err, kMsWaitNs);
        if (*(volatile int*)a.err) return;
      }
      if (!push)
        for (uint64_t c = gwarp; c < a.n_chunks; c += nwarps) ms_hub_chunk<W>(a, cur, active, c, lane);
      for (uint64_t c0 = gwarp * 32; c0 < n; c0 += nwarps * 32) {
        const uint64_t w = c0 + lane;
        Msk<W> vis = mk_zero<W>(), nw = mk_zero<W>();
        if (push) {
          if (w < n) {
            const Msk<W> p = mk_load<W>(a.acc, w);
            if (mk_any(p)) {
              mk_store<W>(a.acc, w, mk_zero<W>());
              vis = mk_load<W>(a.visited, w);
              nw = mk_andnot(p, vis);
            }
          }
        } else {
          // bottom-up: OR the in-neighbours' frontier masks until every
          // needed source is found
          Msk<W> need = mk_zero<W>(), acc = mk_zero<W>();
          uint32_t e0 = 0, e1 = 0;
          if (w < n) {
            vis = mk_load<W>(a.visited, w);
            need = mk_andnot(active, vis);
            if (mk_any(need)) {
              e0 = __ldg(&a.in_off[w]);
              e1 = __ldg(&a.in_off[w + 1]);
              if (e1 - e0 > kMsHub) {  // a hub: settled from its chunks below
                need = mk_zero<W>();
                e1 = e0;
              }
            }
          }
          const bool heavy = e1 - e0 > 32;
          if (!heavy) {
            constexpr int UL = W == 1 ? 4 : 2;  // in-edges per step
            for (uint32_t e = e0; e < e1; e += UL) {
              uint32_t v[UL];
              v[0] = __ldg(&a.in_src[e]);
#pragma unroll
              for (int q = 1; q < UL; q++) v[q] = e + q < e1 ? __ldg(&a.in_src[e + q]) : v[0];
#pragma unroll
              for (int q = 0; q < UL; q++) mk_or(acc, mk_load<W>(cur, v[q]));
              if (mk_covers(acc, need)) break;
            }
          }
          unsigned hm = __ballot_sync(0xffffffffu, heavy);
          while (hm) {
            const int j = __ffs(hm) - 1;
            hm &= hm - 1;
            const uint32_t h0 = __shfl_sync(0xffffffffu, e0, j), h1 = __shfl_sync(0xffffffffu, e1, j);
            const Msk<W> hneed = mk_shfl(need, j);
            Msk<W> hacc = mk_zero<W>();
            constexpr int U = W == 1 ? 4 : 2;  // in-edges per lane per step
            for (uint32_t e = h0; e < h1; e += 32 * U) {
              Msk<W> f = mk_zero<W>();
#pragma unroll
              for (int q = 0; q < U; q++) {
                const uint32_t x = e + q * 32 + lane;
                if (x < h1) mk_or(f, mk_load<W>(cur, __ldg(&a.in_src[x])));
              }
#pragma unroll
              for (int q = 0; q < W; q++) hacc.v[q] |= warp_or64(f.v[q]);
              if (mk_covers(hacc, hneed)) break;
            }
            if (lane == j) acc = hacc;
          }
#pragma unroll
          for (int q = 0; q < W; q++) nw.v[q] = acc.v[q] & need.v[q];
        }
        ms_settle<W>(a, nxt, w, w < n, vis, nw, sc, &s_mf, lane, level, s0);
      }
      if (!push && a.n_hubs) {
        // hubs: their chunks' ORs are all in hacc after the barrier
        grid_barrier(a.bar, a.bar + 1, gridDim.x, a.err, kMsWaitNs);
        if (*(volatile int*)a.err) return;
        for (uint64_t i0 = gwarp * 32; i0 < a.n_hubs; i0 += nwarps * 32) {
          const uint64_t i = i0 + lane;
          uint32_t w = 0;
          Msk<W> vis = mk_zero<W>(), nw = mk_zero<W>();
          if (i < a.n_hubs) {
            w = __ldg(&a.hubs[i]);
            const Msk<W> p = mk_load<W>(a.hacc, i);
            if (mk_any(p)) {
              mk_store<W>(a.hacc, i, mk_zero<W>());
              vis = mk_load<W>(a.visited, w);
              nw = mk_andnot(p, vis);
            }
          }
          ms_settle<W>(a, nxt, w, i < a.n_hubs, vis, nw, sc, &s_mf, lane, level, s0);
        }
      }
      __syncthreads();
      for (int x = threadIdx.x; x < S; x += kMsBlock)
        if (sc[x]) atomicAdd(&row[x], (unsigned long long)sc[x]);
      if (threadIdx.x == 0 && s_mf) atomicAdd(&row[S], s_mf);
      grid_barrier(a.bar, a.bar + 1, gridDim.x, a.err, kMsWaitNs);
      if (*(volatile int*)a.err) return;
      unsigned long long c = 0;
      if (threadIdx.x < S) c = __ldcg(&row[threadIdx.x]);
      if (blockIdx.x == 0 && c) {  // only bits < k are ever counted
        reach += c;
        dsum += (unsigned long long)level * c;
        maxd = level;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, c != 0);
      if (lane == 0 && threadIdx.x < S) s_act[threadIdx.x >> 5] = bal;
      __syncthreads();
      // a source that reached nobody new on this level is finished
#pragma unroll
      for (int q = 0; q < W; q++)
        active.v[q] = ((unsigned long long)s_act[2 * q + 1] << 32) | s_act[2 * q];
      if (!mk_any(active)) break;
    }
    if (blockIdx.x == 0 && threadIdx.x < k && a.reach) {
      a.reach[s0 + threadIdx.x] = reach;
      a.dsum[s0 + threadIdx.x] = dsum;
      a.maxd[s0 + threadIdx.x] = maxd;
    }
  }
}

template <int W>
void ms_launch(MsArgs a, uint64_t n_sources, int device, cudaStream_t s) {
  int per_sm = 0;
  UG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ms_persist_k<W>, kMsBlock, 0));
  UG_CHECK(per_sm > 0, URSA_GPU_ECUDA, "msbfs: kernel cannot be resident");
  // one warp per 32 nodes is all a level pass uses; fewer blocks make
  // cheaper grid barriers
  const uint64_t want = (a.n + 32 * kMsWarps - 1) / (32 * kMsWarps);
  const uint64_t cap = (uint64_t)per_sm * sm_count(device);
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min(want, cap));
  const uint64_t batches = (n_sources + 64 * W - 1) / (64 * W);
  const uint64_t per_launch = std::max<uint64_t>(1, kMsSourcesPerLaunch / (64 * W));
  for (uint64_t b = 0; b < batches; b += per_launch) {
    a.b_begin = b;
    a.b_end = std::min(batches, b + per_launch);
    void* args[] = {&a};
    UG_CUDA(cudaLaunchCooperativeKernel((void*)ms_persist_k<W>, dim3(grid), dim3(kMsBlock), args, 0, s));
    count_launch();
  }
}


// ---- weighted closeness (closeness.rs:137-224), many sources at once ----
//
// A batch is G sub-rows of 32 sources; lane l of a warp works for source
// 32 sub + l.  dist is node-major (n x 32 G distance bit patterns) and
// flags[v G + sub] marks the sources whose distance at v fell in the last
// round.  A round (ending in a grid barrier) walks the out-CSR in 32-edge
// chunks, one (chunk, sub-row) per warp, so a hub's edges spread over many
// warps: for each edge v -> w of weight x whose source v is flagged, the
// flagged lanes relax dist[w] = min(dist[w], fl(dist[v] + x)) with an
// atomicMin on the bits (non-negative doubles order like their bit
// patterns) and flag w for the next round where they lowered it.  Three
// flag buffers rotate: a round reads one, sets the next and clears the one
// read two rounds before.  Rounds end when one lowers nothing.
// The fixpoint is Dijkstra's: dist[v] = min over in-edges of fl(dist[u] + x),
// the minimum left-to-right f64 path sum (fl(a + x) is monotone in a and
// >= a for x >= 0).  A launch relaxes up to R batches, each into its own
// slot of a distance ring, then every warp of the grid folds one (batch,
// sub-row): each lane sums its source's distances in node order exactly as
// closeness_weighted does (f64 sum over reachable v != u), 16 loads ahead of
// its adds -- the sums are sequential, so many sources fold at once.

constexpr unsigned long long kWsInf = 0x7FF0000000000000ull;
constexpr uint64_t kWsDistBudget = 64ull << 20;  // distance rows of one batch: stay in L2
constexpr uint64_t kWsRingBudget = 2ull << 30;   // distance slots of one launch

struct WsArgs {
  const uint32_t* off;   // out-CSR
  const uint32_t* tgt;
  const uint32_t* esrc;  // source node of each out-CSR slot
  const double* wt;      // weights in out-CSR slot order
  uint64_t n, m;
  const uint32_t* sources;  // n_sources ids < n
  uint64_t n_sources;
  uint64_t b_begin, b_end;  // batches of 32 G sources run by this launch
  unsigned G;
  unsigned long long* dist;  // ring: one n x 32 G slot per batch of the launch
  uint32_t* fl[3];           // n x G flags each; round r reads fl[r % 3]
  unsigned long long* count;  // 3 counters, index round % 3: blocks that lowered a distance
  double* out;               // closeness per source
  unsigned* bar;
  int* err;
};

__global__ void __launch_bounds__(kMsBlock) ws_persist_k(WsArgs a) {
  __shared__ int s_any;
  const int lane = threadIdx.x & 31;
  const uint64_t n = a.n, m = a.m, G = a.G, S = 32ull * a.G;
  const uint64_t nwarps = (uint64_t)gridDim.x * kMsWarps;
  const uint64_t gwarp = (uint64_t)blockIdx.x * kMsWarps + (threadIdx.x >> 5);
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t items = (m + 31) / 32 * G;
  uint32_t* const f0 = a.fl[0];
  uint32_t* const f1 = a.fl[1];
  uint32_t* const f2 = a.fl[2];
  for (uint64_t bt = a.b_begin; bt < a.b_end; bt++) {
    const uint64_t s0 = bt * S;
    const uint64_t left = a.n_sources - s0;
    const uint32_t k = left < S ? (uint32_t)left : (uint32_t)S;
    unsigned long long* const dist = a.dist + (bt - a.b_begin) * n * S;
    for (uint64_t x = gtid; x < n * S; x += nthreads) dist[x] = kWsInf;
    for (uint64_t x = gtid; x < n * G; x += nthreads) {
      f0[x] = 0;
      f1[x] = 0;
      f2[x] = 0;
    }
    grid_barrier(a.bar, a.bar + 1, gridDim.x, a.err, kMsWaitNs);
    if (*(volatile int*)a.err) return;
    if (blockIdx.x == 0) {
      if (threadIdx.x < 3) a.count[threadIdx.x] = 0;
      if (threadIdx.x < k) {
        const uint32_t src = a.sources[s0 + threadIdx.x];
        dist[(uint64_t)src * S + threadIdx.x] = 0;  // +0.0
        atomicOr(&f0[(uint64_t)src * G + (threadIdx.x >> 5)], 1u << (threadIdx.x & 31));
      }
    }
    grid_barrier(a.bar, a.bar + 1, gridDim.x, a.err, kMsWaitNs);
    if (*(volatile int*)a.err) return;
    for (uint32_t round = 0;; round++) {
      const uint32_t r3 = round % 3;
      const uint32_t* cur = r3 == 0 ? f0 : (r3 == 1 ? f1 : f2);
      uint32_t* nxt = r3 == 0 ? f1 : (r3 == 1 ? f2 : f0);
      uint32_t* clr = r3 == 0 ? f2 : (r3 == 1 ? f0 : f1);  // read two rounds ago, set next round
      if (threadIdx.x == 0) s_any = 0;
      // counter (round + 1) % 3 was last read before the previous barrier
      if (blockIdx.x == 0 && threadIdx.x == 0) a.count[(round + 1) % 3] = 0;
      for (uint64_t x = gtid; x < n * G; x += nthreads) clr[x] = 0;
      __syncthreads();
      bool lowered = false;
      for (uint64_t item = gwarp; item < items; item += nwarps) {
        const uint64_t sub = item % G;
        const uint64_t e = item / G * 32 + lane;
        uint32_t v = 0, w = 0, c = 0;
        double x = 0.0;
        if (e < m) {
          v = __ldg(&a.esrc[e]);
          c = __ldcg(&cur[(uint64_t)v * G + sub]);
          if (c) {
            w = __ldg(&a.tgt[e]);
            x = __ldg(&a.wt[e]);
          }
        }
        unsigned act = __ballot_sync(0xffffffffu, c != 0);
        const uint64_t col = sub * 32 + lane;
        while (act) {
          const int j = __ffs(act) - 1;
          act &= act - 1;
          const uint32_t vj = __shfl_sync(0xffffffffu, v, j), wj = __shfl_sync(0xffffffffu, w, j);
          const uint32_t cj = __shfl_sync(0xffffffffu, c, j);
          const double xj = __shfl_sync(0xffffffffu, x, j);
          bool imp = false;
          if ((cj >> lane) & 1u) {
            const double dv = __longlong_as_double((long long)__ldcg(&dist[(uint64_t)vj * S + col]));
            const unsigned long long nd = (unsigned long long)__double_as_longlong(__dadd_rn(dv, xj));
            unsigned long long* p = &dist[(uint64_t)wj * S + col];
            if (nd < __ldcg(p)) imp = atomicMin(p, nd) > nd;
          }
          const unsigned b = __ballot_sync(0xffffffffu, imp);
          if (b) {
            lowered = true;
            if (lane == 0) atomicOr(&nxt[(uint64_t)wj * G + sub], b);
          }
        }
      }
      if (lowered) s_any = 1;
      __syncthreads();
      if (threadIdx.x == 0 && s_any) atomicAdd(&a.count[r3], 1ull);
      grid_barrier(a.bar, a.bar + 1, gridDim.x, a.err, kMsWaitNs);
      if (*(volatile int*)a.err) return;
      const bool more = __ldcg(&a.count[r3]) != 0;
      __syncthreads();
      if (!more) break;
    }
  }
  // every batch's relaxations ended at a barrier: fold the launch's batches,
  // one (batch, sub-row) per warp (closeness.rs:196-223)
  const uint64_t nb = a.b_end - a.b_begin;
  for (uint64_t item = gwarp; item < nb * G; item += nwarps) {
    const uint64_t slot = item / G, sub = item % G;
    const uint64_t s0 = (a.b_begin + slot) * S;
    const uint64_t col = sub * 32 + lane;
    if (s0 + col >= a.n_sources) continue;
    const uint32_t u = a.sources[s0 + col];
    const unsigned long long* const base = a.dist + slot * n * S + col;
    double sum = 0.0;
    long long reach = 0;
    uint64_t v = 0;
    for (; v + 16 <= n; v += 16) {
      unsigned long long b[16];
#pragma unroll
      for (int i = 0; i < 16; i++) b[i] = __ldcg(base + (v + i) * S);
#pragma unroll
      for (int i = 0; i < 16; i++)
        if (v + i != u && b[i] < kWsInf) {  // finite (no NaN reaches a distance)
          sum = __dadd_rn(sum, __longlong_as_double((long long)b[i]));
          reach++;
        }
    }
    for (; v < n; v++) {
      const unsigned long long bits = __ldcg(base + v * S);
      if (v != u && bits < kWsInf) {
        sum = __dadd_rn(sum, __longlong_as_double((long long)bits));
        reach++;
      }
    }
    a.out[s0 + col] = sum > 0.0 ? (double)reach / sum : 0.0;
  }
}

__global__ void ws_slot_src_k(const uint32_t* __restrict__ off, uint64_t n, uint64_t m, uint32_t* esrc) {
  for_each_slot_owner(off, n, m, [&](uint64_t k, uint32_t u) { esrc[k] = u; });
}

__global__ void ms_iota_k(uint32_t* out, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (uint32_t)i;
}

// closeness.rs:117-127: reachable as f64 / sum as f64, 0.0 if the sum is 0
// (IEEE division, correctly rounded as on the host).
__global__ void ms_closeness_k(const unsigned long long* __restrict__ reach,
                               const unsigned long long* __restrict__ dsum, uint64_t n, double* out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = dsum[i] > 0 ? (double)(long long)reach[i] / (double)(long long)dsum[i] : 0.0;
}

}  // namespace

// The pull and push CSRs of a traversal following `dir` (0 out-edges, 1
// in-edges, 2 both; both uses the undirected CSR for either role).
struct MsCsrs {
  const uint32_t *pull_off, *pull_src, *push_off, *push_tgt;
  uint64_t push_rows;
};
static MsCsrs ms_csrs(TopoImpl* t, int dir, cudaStream_t s) {
  if (dir == 2) {
    ensure_undirected(t, s);
    return {t->und_off.get(), t->und_tgt.get(), t->und_off.get(), t->und_tgt.get(), t->m_und};
  }
  ensure_in(t, s);
  if (dir == 1) return {t->out.off.get(), t->out.tgt.get(), t->in.off.get(), t->in.tgt.get(), t->m};
  return {t->in.off.get(), t->in.tgt.get(), t->out.off.get(), t->out.tgt.get(), t->m};
}

// Builds (once per topology and direction) the hub list and the chunks of
// the hubs' pull rows: hubs have more than kMsHub pull entries, chunks are
// kMsChunk slots.
static const TopoImpl::MsHubs& ensure_ms_hubs(TopoImpl* t, int dir, const MsCsrs& c, cudaStream_t s) {
  std::lock_guard<std::mutex> g(t->mu);
  TopoImpl::MsHubs& h = t->ms_hubs[dir];
  if (h.built) return h;
  const uint64_t n = t->n;
  std::vector<uint32_t> off(n + 1), hubs, chunk_hub, chunk_lo;
  UG_CUDA(cudaMemcpyAsync(off.data(), c.pull_off, (n + 1) * 4, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  for (uint64_t w = 0; w < n; w++) {
    if (off[w + 1] - off[w] <= kMsHub) continue;
    for (uint32_t e = off[w]; e < off[w + 1]; e += kMsChunk) {
      chunk_hub.push_back((uint32_t)hubs.size());
      chunk_lo.push_back(e);
    }
    hubs.push_back((uint32_t)w);
  }
  h.n_hubs = hubs.size();
  h.n_chunks = chunk_hub.size();
  h.hubs.alloc(hubs.size() ? hubs.size() : 1, s);
  h.chunk_hub.alloc(chunk_hub.size() ? chunk_hub.size() : 1, s);
  h.chunk_lo.alloc(chunk_lo.size() ? chunk_lo.size() : 1, s);
  if (!hubs.empty()) {
    UG_CUDA(cudaMemcpyAsync(h.hubs.get(), hubs.data(), hubs.size() * 4, cudaMemcpyHostToDevice, s));
    UG_CUDA(cudaMemcpyAsync(h.chunk_hub.get(), chunk_hub.data(), chunk_hub.size() * 4,
                            cudaMemcpyHostToDevice, s));
    UG_CUDA(cudaMemcpyAsync(h.chunk_lo.get(), chunk_lo.data(), chunk_lo.size() * 4,
                            cudaMemcpyHostToDevice, s));
  }
  UG_CUDA(cudaStreamSynchronize(s));
  h.built = true;
  return h;
}

// Enqueues a BFS from each of the device ids d_src (< n) following `dir`.
// Per source (device arrays of n_sources entries, or NULL): reach = nodes at
// distance >= 1, dsum = their summed distances, maxd = eccentricity; d_dist
// (or NULL): n_sources rows of n hop distances, -1 where unreached.
// d_ctl: 4 zeroed words (grid barrier; word 2 turns nonzero if a barrier
// wait expired).  Batches are 256 sources wide when there are enough
// sources to fill them and the masks of a graph of at most 2^21 nodes (64 MB
// per mask array) stay in L2; otherwise 64 wide (fewer registers per
// thread, more warps per SM).
static void msbfs_enqueue(TopoImpl* t, int dir, const uint32_t* d_src, uint64_t n_sources,
                          unsigned long long* d_reach, unsigned long long* d_dsum, uint32_t* d_maxd,
                          int32_t* d_dist, unsigned* d_ctl, cudaStream_t s) {
  const uint64_t n = t->n;
  if (n_sources == 0) return;
  const MsCsrs c = ms_csrs(t, dir, s);
  const TopoImpl::MsHubs& hb = ensure_ms_hubs(t, dir, c, s);
  const int W = n_sources >= 256 && n <= (1ull << 21) ? 4 : 1;
  Scratch<unsigned long long> visited(n * W, s), fa(n * W, s), fb(n * W, s), acc(n * W, s);
  Scratch<unsigned long long> count(3 * (64 * W + 8), s);
  UG_CUDA(cudaMemsetAsync(acc.get(), 0, n * W * 8, s));
  const uint64_t nh = hb.n_hubs, nc = hb.n_chunks;
  Scratch<unsigned long long> hacc((nh ? nh : 1) * W, s);
  UG_CUDA(cudaMemsetAsync(hacc.get(), 0, (nh ? nh : 1) * W * 8, s));
  if (d_dist) UG_CUDA(cudaMemsetAsync(d_dist, 0xFF, n_sources * n * 4, s));
  MsArgs a;
  a.in_off = c.pull_off;
  a.in_src = c.pull_src;
  a.out_off = c.push_off;
  a.out_tgt = c.push_tgt;
  a.n = n;
  a.m = c.push_rows;
  a.dist = d_dist;
  a.sources = d_src;
  a.n_sources = n_sources;
  a.visited = visited.get();
  a.fr0 = fa.get();
  a.fr1 = fb.get();
  a.acc = acc.get();
  a.hubs = hb.hubs.get();
  a.n_hubs = nh;
  a.chunk_hub = hb.chunk_hub.get();
  a.chunk_lo = hb.chunk_lo.get();
  a.n_chunks = nc;
  a.hacc = hacc.get();
  a.count = count.get();
  a.reach = d_reach;
  a.dsum = d_dsum;
  a.maxd = d_maxd;
  a.bar = d_ctl;
  a.err = (int*)(d_ctl + 2);
  if (W == 4)
    ms_launch<4>(a, n_sources, t->device, s);
  else
    ms_launch<1>(a, n_sources, t->device, s);
}

// Hop distances from each of the device ids d_src (< n), following `dir`:
// d_dist holds n_sources rows of n (-1 where unreached); returns after the
// work completes.
void msbfs_distances(TopoImpl* t, int dir, const uint32_t* d_src, uint64_t n_sources, int32_t* d_dist,
                     cudaStream_t s) {
  if (n_sources == 0 || t->n == 0) return;
  Scratch<unsigned> ctl(4, s);
  UG_CUDA(cudaMemsetAsync(ctl.get(), 0, 16, s));
  msbfs_enqueue(t, dir, d_src, n_sources, nullptr, nullptr, nullptr, d_dist, ctl.get(), s);
  int err = 0;
  UG_CUDA(cudaMemcpyAsync(&err, ctl.get() + 2, 4, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  UG_CHECK(err == 0, URSA_GPU_ETIMEOUT, "bfs: a grid barrier wait expired");
}

// Host form of msbfs_enqueue: host sources in, host folds out.
void msbfs_run(TopoImpl* t, const uint32_t* sources, uint64_t n_sources, uint64_t* reach,
               uint64_t* dsum, uint32_t* maxd, cudaStream_t s) {
  if (n_sources == 0) return;
  Scratch<unsigned long long> d_reach(n_sources, s), d_dsum(n_sources, s);
  Scratch<uint32_t> d_maxd(n_sources, s), d_src(n_sources, s);
  Scratch<unsigned> ctl(4, s);
  UG_CUDA(cudaMemsetAsync(ctl.get(), 0, 16, s));
  UG_CUDA(cudaMemcpyAsync(d_src.get(), sources, n_sources * 4, cudaMemcpyHostToDevice, s));
  msbfs_enqueue(t, 0, d_src.get(), n_sources, d_reach.get(), d_dsum.get(), d_maxd.get(), nullptr, ctl.get(), s);
  int err = 0;
  UG_CUDA(cudaMemcpyAsync(&err, ctl.get() + 2, 4, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaMemcpyAsync(reach, d_reach.get(), n_sources * 8, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaMemcpyAsync(dsum, d_dsum.get(), n_sources * 8, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaMemcpyAsync(maxd, d_maxd.get(), n_sources * 4, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  UG_CHECK(err == 0, URSA_GPU_ETIMEOUT, "msbfs: a grid barrier wait expired");
}

// Closeness of every node into the device array d_out, enqueued on s;
// returns after completion, with the device time of the enqueued work.
void closeness_device(TopoImpl* t, double* d_out, cudaStream_t s, float* device_ms) {
  const uint64_t n = t->n;
  Scratch<unsigned long long> d_reach(n, s), d_dsum(n, s);
  Scratch<uint32_t> d_maxd(n, s), d_src(n, s);
  Scratch<unsigned> ctl(4, s);
  cudaEvent_t e0, e1;
  UG_CUDA(cudaEventCreate(&e0));
  UG_CUDA(cudaEventCreate(&e1));
  UG_CUDA(cudaEventRecord(e0, s));
  UG_CUDA(cudaMemsetAsync(ctl.get(), 0, 16, s));
  ms_iota_k<<<grid_for(n), kBlock, 0, s>>>(d_src.get(), n);
  UG_LAUNCH_CHECK();
  msbfs_enqueue(t, 0, d_src.get(), n, d_reach.get(), d_dsum.get(), d_maxd.get(), nullptr, ctl.get(), s);
  ms_closeness_k<<<grid_for(n), kBlock, 0, s>>>(d_reach.get(), d_dsum.get(), n, d_out);
  UG_LAUNCH_CHECK();
  UG_CUDA(cudaEventRecord(e1, s));
  int err = 0;
  UG_CUDA(cudaMemcpyAsync(&err, ctl.get() + 2, 4, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (device_ms) *device_ms = ms;
  UG_CHECK(err == 0, URSA_GPU_ETIMEOUT, "closeness: a grid barrier wait expired");
}

// stats.rs:82-101: `None` -> every node; `Some(frac)` -> k = round(n * frac)
// (at least 1, at most n) sources evenly strided by max(n / k, 1).
static std::vector<uint32_t> stats_sources(uint64_t n, int has_frac, double frac) {
  std::vector<uint32_t> out;
  if (!has_frac) {
    out.resize(n);
    for (uint64_t i = 0; i < n; i++) out[i] = (uint32_t)i;
    return out;
  }
  double f = frac < 0.0 ? 0.0 : (frac > 1.0 ? 1.0 : frac);
  double kd = std::round((double)n * f);
  if (kd < 1.0) kd = 1.0;
  uint64_t k = (uint64_t)kd;
  if (k > n) k = n;
  if (k == 0) return out;
  double step = (double)n / (double)k;
  if (step < 1.0) step = 1.0;
  out.resize(k);
  for (uint64_t i = 0; i < k; i++) {
    uint64_t v = (uint64_t)std::floor((double)i * step);
    out[i] = (uint32_t)(v < n - 1 ? v : n - 1);
  }
  return out;
}

// Weighted closeness of every node into d_out (enqueued on s, returns after
// completion).  d_w: edge weights by original edge row (device).
void closeness_weighted_device(TopoImpl* t, const double* d_w, double* d_out, cudaStream_t s) {
  const uint64_t n = t->n;
  DirView dv = dir_view(t, 0, s);
  DirWeights dw;
  gather_dir_weights(t, dv, d_w, dw, s);
  uint64_t G = kWsDistBudget / (n * 256);
  G = G < 1 ? 1 : (G > 8 ? 8 : G);
  const uint64_t S = 32 * G;
  const uint64_t m = t->m;
  const uint64_t batches = (n + S - 1) / S;
  uint64_t R = kWsRingBudget / (n * S * 8);
  R = std::max<uint64_t>(1, std::min<uint64_t>(R, std::min<uint64_t>(64, batches)));
  Scratch<unsigned long long> dist(R * n * S, s), count(3, s);
  Scratch<uint32_t> fa(n * G, s), fb(n * G, s), fc(n * G, s), src(n, s), esrc(m ? m : 1, s);
  if (m) {
    ws_slot_src_k<<<grid_for(m, kBlock, 148u * 64u), kBlock, 0, s>>>(dv.off0, n, m, esrc.get());
    UG_LAUNCH_CHECK();
  }
  Scratch<unsigned> ctl(4, s);
  UG_CUDA(cudaMemsetAsync(ctl.get(), 0, 16, s));
  ms_iota_k<<<grid_for(n), kBlock, 0, s>>>(src.get(), n);
  UG_LAUNCH_CHECK();
  int per_sm = 0;
  UG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ws_persist_k, kMsBlock, 0));
  UG_CHECK(per_sm > 0, URSA_GPU_ECUDA, "closeness_weighted: kernel cannot be resident");
  const uint64_t want = ((m + 31) / 32 * G + kMsWarps - 1) / kMsWarps;  // a warp per (chunk, sub-row)
  const uint64_t cap = (uint64_t)per_sm * sm_count(t->device);
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min(want, cap));
  WsArgs a;
  a.off = dv.off0;
  a.tgt = dv.tgt0;
  a.esrc = esrc.get();
  a.wt = dw.w0.get();
  a.n = n;
  a.m = m;
  a.sources = src.get();
  a.n_sources = n;
  a.G = (unsigned)G;
  a.dist = dist.get();
  a.fl[0] = fa.get();
  a.fl[1] = fb.get();
  a.fl[2] = fc.get();
  a.count = count.get();
  a.out = d_out;
  a.bar = ctl.get();
  a.err = (int*)(ctl.get() + 2);
  for (uint64_t b = 0; b < batches; b += R) {
    a.b_begin = b;
    a.b_end = std::min(batches, b + R);
    void* args[] = {&a};
    UG_CUDA(cudaLaunchCooperativeKernel((void*)ws_persist_k, dim3(grid), dim3(kMsBlock), args, 0, s));
    count_launch();
  }
  int err = 0;
  UG_CUDA(cudaMemcpyAsync(&err, ctl.get() + 2, 4, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  UG_CHECK(err == 0, URSA_GPU_ETIMEOUT, "closeness_weighted: a grid barrier wait expired");
}

}  // namespace ug

using namespace ug;

extern "C" {

int ursa_gpu_closeness(ursa_gpu_topo* t, double* out) {
  return guard([&] {
    UG_CHECK(t, URSA_GPU_EINVAL, "topology is NULL");
    TopoImpl* ti = &t->impl;
    const uint64_t n = ti->n;
    if (n == 0) return;
    UG_CHECK(out, URSA_GPU_EINVAL, "out is NULL");
    cudaStream_t s = thread_stream(ti->device);
    Scratch<double> d_out(n, s);
    closeness_device(ti, d_out.get(), s, nullptr);
    UG_CUDA(cudaMemcpyAsync(out, d_out.get(), n * 8, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_closeness_device(ursa_gpu_topo* t, double* d_out, void* stream, float* device_ms) {
  return guard([&] {
    UG_CHECK(t, URSA_GPU_EINVAL, "topology is NULL");
    TopoImpl* ti = &t->impl;
    if (device_ms) *device_ms = 0.f;
    if (ti->n == 0) return;
    UG_CHECK(d_out, URSA_GPU_EINVAL, "d_out is NULL");
    cudaStream_t ts = thread_stream(ti->device);  // also selects the device
    cudaStream_t s = stream ? (cudaStream_t)stream : ts;
    closeness_device(ti, d_out, s, device_ms);
  });
}

int ursa_gpu_bfs_distances_multi(ursa_gpu_topo* t, const uint32_t* sources, uint64_t n_sources, int dir,
                                 int32_t* out) {
  return guard([&] {
    UG_CHECK(t, URSA_GPU_EINVAL, "topology is NULL");
    UG_CHECK(dir >= 0 && dir <= 2, URSA_GPU_EINVAL, "direction must be 0, 1 or 2");
    TopoImpl* ti = &t->impl;
    const uint64_t n = ti->n;
    if (n == 0 || n_sources == 0) return;
    UG_CHECK(sources && out, URSA_GPU_EINVAL, "sources / out is NULL");
    // bfs.rs:21-23: an unknown source's row is all -1
    std::vector<uint32_t> valid;
    std::vector<uint64_t> row;
    for (uint64_t i = 0; i < n_sources; i++) {
      if ((uint64_t)sources[i] < n) {
        valid.push_back(sources[i]);
        row.push_back(i);
      } else {
        std::memset(out + i * n, 0xFF, n * 4);
      }
    }
    if (valid.empty()) return;
    cudaStream_t s = thread_stream(ti->device);
    Scratch<uint32_t> d_src(valid.size(), s);
    Scratch<int32_t> d_dist(valid.size() * n, s);
    UG_CUDA(cudaMemcpyAsync(d_src.get(), valid.data(), valid.size() * 4, cudaMemcpyHostToDevice, s));
    msbfs_distances(ti, dir, d_src.get(), valid.size(), d_dist.get(), s);
    if (valid.size() == n_sources) {
      UG_CUDA(cudaMemcpyAsync(out, d_dist.get(), n_sources * n * 4, cudaMemcpyDeviceToHost, s));
    } else {
      for (size_t j = 0; j < valid.size(); j++)
        UG_CUDA(cudaMemcpyAsync(out + row[j] * n, d_dist.get() + j * n, n * 4, cudaMemcpyDeviceToHost, s));
    }
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_closeness_weighted(ursa_gpu_topo* t, const double* weights, uint64_t n_weights,
                                double* out) {
  return guard([&] {
    UG_CHECK(t, URSA_GPU_EINVAL, "topology is NULL");
    TopoImpl* ti = &t->impl;
    UG_CHECK(n_weights == ti->m, URSA_GPU_EINVAL, "weights length must equal the edge count");
    UG_CHECK(ti->m == 0 || weights, URSA_GPU_EINVAL, "weights is NULL");
    const uint64_t n = ti->n;
    if (n == 0) return;
    UG_CHECK(out, URSA_GPU_EINVAL, "out is NULL");
    cudaStream_t s = thread_stream(ti->device);
    Scratch<double> dw(ti->m ? ti->m : 1, s), d_out(n, s);
    if (ti->m) UG_CUDA(cudaMemcpyAsync(dw.get(), weights, ti->m * 8, cudaMemcpyHostToDevice, s));
    check_sssp_weights_device(dw.get(), ti->m, s);
    closeness_weighted_device(ti, dw.get(), d_out.get(), s);
    UG_CUDA(cudaMemcpyAsync(out, d_out.get(), n * 8, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_avg_path_length(ursa_gpu_topo* t, int has_sample, double sample, double* out) {
  return guard([&] {
    UG_CHECK(t && out, URSA_GPU_EINVAL, "topology / out is NULL");
    TopoImpl* ti = &t->impl;
    *out = 0.0;
    std::vector<uint32_t> src = stats_sources(ti->n, has_sample, sample);
    if (src.empty()) return;
    cudaStream_t s = thread_stream(ti->device);
    std::vector<uint64_t> reach(src.size()), dsum(src.size());
    std::vector<uint32_t> maxd(src.size());
    msbfs_run(ti, src.data(), src.size(), reach.data(), dsum.data(), maxd.data(), s);
    // stats.rs:107-140: f64 sums of integer distances, folded in source order;
    // exact (and so equal to the integer totals) below 2^53
    unsigned long long sum = 0, count = 0;
    for (size_t i = 0; i < src.size(); i++) {
      sum += dsum[i];
      count += reach[i];
    }
    UG_CHECK(sum < (1ull << 53), URSA_GPU_EINVAL,
             "avg_path_length: distance total at or above 2^53 (f64 sums would round)");
    *out = count == 0 ? 0.0 : (double)sum / (double)count;
  });
}

int ursa_gpu_diameter(ursa_gpu_topo* t, int approximate, int64_t* out) {
  return guard([&] {
    UG_CHECK(t && out, URSA_GPU_EINVAL, "topology / out is NULL");
    TopoImpl* ti = &t->impl;
    *out = 0;
    const uint64_t n = ti->n;
    // stats.rs:154-166: approximate -> frac = min(128 / n, 1)
    std::vector<uint32_t> src =
        approximate && n > 0 ? stats_sources(n, 1, std::min(128.0 / (double)n, 1.0))
                             : stats_sources(n, 0, 0.0);
    if (src.empty()) return;
    cudaStream_t s = thread_stream(ti->device);
    std::vector<uint64_t> reach(src.size()), dsum(src.size());
    std::vector<uint32_t> maxd(src.size());
    msbfs_run(ti, src.data(), src.size(), reach.data(), dsum.data(), maxd.data(), s);
    uint32_t mx = 0;
    for (uint32_t d : maxd) mx = d > mx ? d : mx;
    *out = (int64_t)mx;
  });
}

}  // extern "C"
