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
//   Nodes with at most 32 edges to scan are handled by one lane, heavier ones
//   by the whole warp.  visited[w] |= new; next[w] = new.
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
#include <cmath>
#include <vector>

#include "frontier.cuh"
#include "primitives.cuh"

namespace ug {

void dijkstra_run(TopoImpl* t, const double* d_weights, uint32_t source, int dir, double* d_out,
                  cudaStream_t s);

namespace {

constexpr int kMsBlock = 256;
constexpr int kMsWarps = kMsBlock / 32;
constexpr uint64_t kMsBatchesPerLaunch = 16;
constexpr uint64_t kMsWaitNs = 5000000000ull;  // one grid-barrier wait
constexpr int kMsRow = 72;  // per-level counter row: 64 per-source counts, [64] = frontier out-edges
constexpr uint64_t kMsPushDiv = 8;  // push while the frontier's out-edges are below m / 8

struct MsArgs {
  const uint32_t* in_off;
  const uint32_t* in_src;
  const uint32_t* out_off;
  const uint32_t* out_tgt;
  uint64_t n, m;
  const uint32_t* sources;  // n_sources ids < n
  uint64_t n_sources;
  uint64_t b_begin, b_end;  // batches of 64 sources run by this launch
  unsigned long long* visited;
  unsigned long long* fr0;    // frontier masks, odd levels' input
  unsigned long long* fr1;    // even levels' input
  unsigned long long* acc;    // pushed masks of a top-down level; all zero between levels
  unsigned long long* count;  // 3 rows of kMsRow, row = level % 3
  unsigned long long* reach;
  unsigned long long* dsum;
  uint32_t* maxd;
  unsigned* bar;  // grid barrier count, generation
  int* err;
};

__device__ __forceinline__ unsigned long long warp_or64(unsigned long long v) {
  const unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)v);
  const unsigned hi = __reduce_or_sync(0xffffffffu, (unsigned)(v >> 32));
  return ((unsigned long long)hi << 32) | lo;
}

// Top-down half of a level: every frontier node v ORs its mask into acc[w]
// for each out-edge v -> w whose target still lacks some of those sources.
__device__ __forceinline__ void ms_push(const MsArgs& a, const unsigned long long* cur, uint64_t gwarp,
                                        uint64_t nwarps, int lane) {
  for (uint64_t c0 = gwarp * 32; c0 < a.n; c0 += nwarps * 32) {
    const uint64_t v = c0 + lane;
    unsigned long long f = 0;
    uint32_t e0 = 0, e1 = 0;
    if (v < a.n) {
      f = __ldcg(&cur[v]);
      if (f) {
        e0 = __ldg(&a.out_off[v]);
        e1 = __ldg(&a.out_off[v + 1]);
      }
    }
    const bool heavy = f && e1 - e0 > 32;
    if (f && !heavy) {
      for (uint32_t e = e0; e < e1; e++) {
        const uint32_t w = __ldg(&a.out_tgt[e]);
        const unsigned long long add = f & ~__ldcg(&a.visited[w]);
        if (add) atomicOr(&a.acc[w], add);
      }
    }
    unsigned hm = __ballot_sync(0xffffffffu, heavy);
    while (hm) {
      const int j = __ffs(hm) - 1;
      hm &= hm - 1;
      const uint32_t h0 = __shfl_sync(0xffffffffu, e0, j), h1 = __shfl_sync(0xffffffffu, e1, j);
      const unsigned long long hf = __shfl_sync(0xffffffffu, f, j);
      for (uint32_t e = h0 + lane; e < h1; e += 32) {
        const uint32_t w = __ldg(&a.out_tgt[e]);
        const unsigned long long add = hf & ~__ldcg(&a.visited[w]);
        if (add) atomicOr(&a.acc[w], add);
      }
    }
  }
}

__global__ void __launch_bounds__(kMsBlock) ms_persist_k(MsArgs a) {
  __shared__ unsigned sc[64];
  __shared__ unsigned long long s_mf;
  __shared__ unsigned s_act[2];
  const int lane = threadIdx.x & 31;
  const uint64_t n = a.n;
  const uint64_t nwarps = (uint64_t)gridDim.x * kMsWarps;
  const uint64_t gwarp = (uint64_t)blockIdx.x * kMsWarps + (threadIdx.x >> 5);
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (uint64_t bt = a.b_begin; bt < a.b_end; bt++) {
    const uint64_t s0 = bt * 64;
    const uint64_t left = a.n_sources - s0;
    const uint32_t k = left < 64 ? (uint32_t)left : 64u;
    const unsigned long long full = k == 64 ? ~0ull : ((1ull << k) - 1);
    for (uint64_t w = gtid; w < n; w += nthreads) {
      a.visited[w] = 0;
      a.fr0[w] = 0;
    }
    grid_barrier(a.bar, a.bar + 1, gridDim.x, a.err, kMsWaitNs);
    if (*(volatile int*)a.err) return;
    if (blockIdx.x == 0) {  // every block has read the previous batch's last counter row
      if (threadIdx.x < 3 * kMsRow) a.count[threadIdx.x] = 0;
      __syncthreads();
      if (threadIdx.x < k) {
        const uint32_t src = a.sources[s0 + threadIdx.x];
        atomicOr(&a.visited[src], 1ull << threadIdx.x);
        atomicOr(&a.fr0[src], 1ull << threadIdx.x);
        atomicAdd(&a.count[64], (unsigned long long)(a.out_off[src + 1] - a.out_off[src]));
      }
    }
    grid_barrier(a.bar, a.bar + 1, gridDim.x, a.err, kMsWaitNs);
    if (*(volatile int*)a.err) return;
    unsigned long long reach = 0, dsum = 0;  // block 0, thread b < k: source s0 + b
    uint32_t maxd = 0;
    unsigned long long active = full;  // sources whose search still grows
    for (uint32_t level = 1;; level++) {
      const unsigned long long* cur = (level & 1) ? a.fr0 : a.fr1;
      unsigned long long* nxt = (level & 1) ? a.fr1 : a.fr0;
      unsigned long long* row = a.count + (level % 3) * kMsRow;
      const unsigned long long mf = __ldcg(&a.count[((level - 1) % 3) * kMsRow + 64]);
      const bool push = mf * kMsPushDiv < a.m;
      if (threadIdx.x < 64) sc[threadIdx.x] = 0;
      if (threadIdx.x == 0) s_mf = 0;
      // row (level + 1) % 3 was last read before the previous barrier
      if (blockIdx.x == 0 && threadIdx.x < kMsRow) a.count[((level + 1) % 3) * kMsRow + threadIdx.x] = 0;
      __syncthreads();
      if (push) {
        ms_push(a, cur, gwarp, nwarps, lane);
        grid_barrier(a.bar, a.bar + 1, gridDim.x, a.err, kMsWaitNs);
        if (*(volatile int*)a.err) return;
      }
      for (uint64_t c0 = gwarp * 32; c0 < n; c0 += nwarps * 32) {
        const uint64_t w = c0 + lane;
        unsigned long long vis = 0, nw = 0;
        if (push) {
          if (w < n) {
            const unsigned long long p = __ldcg(&a.acc[w]);
            if (p) {
              a.acc[w] = 0;
              vis = __ldcg(&a.visited[w]);
              nw = p & ~vis;
            }
          }
        } else {
          // bottom-up: OR the in-neighbours' frontier masks until every
          // needed source is found
          unsigned long long need = 0, acc = 0;
          uint32_t e0 = 0, e1 = 0;
          if (w < n) {
            vis = __ldcg(&a.visited[w]);
            need = active & ~vis;
            if (need) {
              e0 = __ldg(&a.in_off[w]);
              e1 = __ldg(&a.in_off[w + 1]);
            }
          }
          const bool heavy = need && e1 - e0 > 32;
          if (need && !heavy) {
            for (uint32_t e = e0; e < e1; e += 4) {
              const uint32_t r = e1 - e;
              const uint32_t v0 = __ldg(&a.in_src[e]);
              const uint32_t v1 = r > 1 ? __ldg(&a.in_src[e + 1]) : v0;
              const uint32_t v2 = r > 2 ? __ldg(&a.in_src[e + 2]) : v0;
              const uint32_t v3 = r > 3 ? __ldg(&a.in_src[e + 3]) : v0;
              acc |= __ldcg(&cur[v0]) | __ldcg(&cur[v1]) | __ldcg(&cur[v2]) | __ldcg(&cur[v3]);
              if ((acc & need) == need) break;
            }
          }
          unsigned hm = __ballot_sync(0xffffffffu, heavy);
          while (hm) {
            const int j = __ffs(hm) - 1;
            hm &= hm - 1;
            const uint32_t h0 = __shfl_sync(0xffffffffu, e0, j), h1 = __shfl_sync(0xffffffffu, e1, j);
            const unsigned long long hneed = __shfl_sync(0xffffffffu, need, j);
            unsigned long long hacc = 0;
            for (uint32_t e = h0; e < h1; e += 128) {
              unsigned long long f = 0;
#pragma unroll
              for (int q = 0; q < 4; q++) {
                const uint32_t x = e + q * 32 + lane;
                if (x < h1) f |= __ldcg(&cur[__ldg(&a.in_src[x])]);
              }
              hacc |= warp_or64(f);
              if ((hacc & hneed) == hneed) break;
            }
            if (lane == j) acc = hacc;
          }
          nw = acc & need;
        }
        unsigned long long od = 0;
        if (w < n) {
          if (nw) {
            a.visited[w] = vis | nw;
            od = __ldg(&a.out_off[w + 1]) - __ldg(&a.out_off[w]);
          }
          nxt[w] = nw;
        }
        if (__any_sync(0xffffffffu, nw != 0)) {
#pragma unroll 8
          for (int b = 0; b < 64; b++) {
            const unsigned c = __popc(__ballot_sync(0xffffffffu, (nw >> b) & 1ull));
            if (lane == 0 && c) atomicAdd(&sc[b], c);
          }
          for (int o = 16; o; o >>= 1) od += __shfl_down_sync(0xffffffffu, od, o);
          if (lane == 0) atomicAdd(&s_mf, od);
        }
      }
      __syncthreads();
      if (threadIdx.x < 64 && sc[threadIdx.x])
        atomicAdd(&row[threadIdx.x], (unsigned long long)sc[threadIdx.x]);
      if (threadIdx.x == 0 && s_mf) atomicAdd(&row[64], s_mf);
      grid_barrier(a.bar, a.bar + 1, gridDim.x, a.err, kMsWaitNs);
      if (*(volatile int*)a.err) return;
      unsigned long long c = 0;
      if (threadIdx.x < 64) c = __ldcg(&row[threadIdx.x]);
      if (blockIdx.x == 0 && c) {  // only bits < k are ever counted
        reach += c;
        dsum += (unsigned long long)level * c;
        maxd = level;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, c != 0);
      if (threadIdx.x == 0) s_act[0] = bal;
      if (threadIdx.x == 32) s_act[1] = bal;
      __syncthreads();
      // a source that reached nobody new on this level is finished
      active = ((unsigned long long)s_act[1] << 32) | s_act[0];
      if (!active) break;
    }
    if (blockIdx.x == 0 && threadIdx.x < k) {
      a.reach[s0 + threadIdx.x] = reach;
      a.dsum[s0 + threadIdx.x] = dsum;
      a.maxd[s0 + threadIdx.x] = maxd;
    }
  }
}

}  // namespace

// Per-source BFS folds (reach = nodes at distance >= 1, dsum = their summed
// distances, maxd = eccentricity) for `sources` (host ids < n), following
// out-edges.  Outputs are host arrays of n_sources entries.
void msbfs_run(TopoImpl* t, const uint32_t* sources, uint64_t n_sources, uint64_t* reach,
               uint64_t* dsum, uint32_t* maxd, cudaStream_t s) {
  const uint64_t n = t->n;
  if (n_sources == 0) return;
  ensure_in(t, s);
  Scratch<unsigned long long> visited(n, s), fa(n, s), fb(n, s), acc(n, s), count(3 * kMsRow, s);
  Scratch<unsigned long long> d_reach(n_sources, s), d_dsum(n_sources, s);
  Scratch<uint32_t> d_maxd(n_sources, s), d_src(n_sources, s);
  Scratch<unsigned> ctl(4, s);
  UG_CUDA(cudaMemsetAsync(ctl.get(), 0, 16, s));
  UG_CUDA(cudaMemsetAsync(acc.get(), 0, n * 8, s));
  UG_CUDA(cudaMemcpyAsync(d_src.get(), sources, n_sources * 4, cudaMemcpyHostToDevice, s));
  int per_sm = 0;
  UG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ms_persist_k, kMsBlock, 0));
  UG_CHECK(per_sm > 0, URSA_GPU_ECUDA, "msbfs: kernel cannot be resident");
  const unsigned grid = (unsigned)(per_sm * sm_count(t->device));
  MsArgs a;
  a.in_off = t->in.off.get();
  a.in_src = t->in.tgt.get();
  a.out_off = t->out.off.get();
  a.out_tgt = t->out.tgt.get();
  a.n = n;
  a.m = t->m;
  a.sources = d_src.get();
  a.n_sources = n_sources;
  a.visited = visited.get();
  a.fr0 = fa.get();
  a.fr1 = fb.get();
  a.acc = acc.get();
  a.count = count.get();
  a.reach = d_reach.get();
  a.dsum = d_dsum.get();
  a.maxd = d_maxd.get();
  a.bar = ctl.get();
  a.err = (int*)(ctl.get() + 2);
  const uint64_t batches = (n_sources + 63) / 64;
  for (uint64_t b = 0; b < batches; b += kMsBatchesPerLaunch) {
    a.b_begin = b;
    a.b_end = std::min(batches, b + kMsBatchesPerLaunch);
    void* args[] = {&a};
    UG_CUDA(cudaLaunchCooperativeKernel((void*)ms_persist_k, dim3(grid), dim3(kMsBlock), args, 0, s));
    count_launch();
  }
  int err = 0;
  UG_CUDA(cudaMemcpyAsync(&err, ctl.get() + 2, 4, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaMemcpyAsync(reach, d_reach.get(), n_sources * 8, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaMemcpyAsync(dsum, d_dsum.get(), n_sources * 8, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaMemcpyAsync(maxd, d_maxd.get(), n_sources * 4, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  UG_CHECK(err == 0, URSA_GPU_ETIMEOUT, "msbfs: a grid barrier wait expired");
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
    std::vector<uint32_t> src(n);
    for (uint64_t i = 0; i < n; i++) src[i] = (uint32_t)i;
    std::vector<uint64_t> reach(n), dsum(n);
    std::vector<uint32_t> maxd(n);
    msbfs_run(ti, src.data(), n, reach.data(), dsum.data(), maxd.data(), s);
    // closeness.rs:117-127: reachable as f64 / sum as f64, 0.0 if sum == 0
    for (uint64_t u = 0; u < n; u++)
      out[u] = dsum[u] > 0 ? (double)(int64_t)reach[u] / (double)(int64_t)dsum[u] : 0.0;
  });
}

int ursa_gpu_closeness_weighted(ursa_gpu_topo* t, const double* weights, uint64_t n_weights,
                                double* out) {
  return guard([&] {
    UG_CHECK(t, URSA_GPU_EINVAL, "topology is NULL");
    TopoImpl* ti = &t->impl;
    UG_CHECK(n_weights == ti->m, URSA_GPU_EINVAL, "weights length must equal the edge count");
    const uint64_t n = ti->n;
    if (n == 0) return;
    UG_CHECK(out, URSA_GPU_EINVAL, "out is NULL");
    cudaStream_t s = thread_stream(ti->device);
    Scratch<double> dw(ti->m ? ti->m : 1, s), dd(n, s);
    if (ti->m) UG_CUDA(cudaMemcpyAsync(dw.get(), weights, ti->m * 8, cudaMemcpyHostToDevice, s));
    std::vector<double> dist(n);
    for (uint64_t u = 0; u < n; u++) {
      // exact f64 distances on the device (sssp.cu), then the reference's
      // node-order f64 fold (closeness.rs:196-223) on the host
      dijkstra_run(ti, dw.get(), (uint32_t)u, 0, dd.get(), s);
      UG_CUDA(cudaMemcpyAsync(dist.data(), dd.get(), n * 8, cudaMemcpyDeviceToHost, s));
      UG_CUDA(cudaStreamSynchronize(s));
      double sum = 0.0;
      int64_t reachable = 0;
      for (uint64_t v = 0; v < n; v++)
        if (v != u && std::isfinite(dist[v])) {
          sum += dist[v];
          reachable++;
        }
      out[u] = sum > 0.0 ? (double)reachable / sum : 0.0;
    }
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
