// msbfs.cu -- BFS from many sources at once: closeness
// (ursa-core/src/algo/closeness.rs:69-135) and the path statistics
// avg_path_length / diameter (ursa-plan/src/stats.rs:82-170).
//
// Sources are taken 64 at a time; bit b of a node's 64-bit masks belongs to
// source b of the batch.  Per BFS level (following out-edges):
//   pull:  next[w] |= frontier[v] & ~visited[w] for every in-edge v -> w
//          (edge-parallel over the in-CSR, 64-bit atomicOr);
//   settle: new = next[w] & ~visited[w]; visited |= new; frontier = new;
//          per source, the number of nodes first reached on this level is a
//          column popcount of the new masks (one warp ballot per bit);
//   fold:  reach[b] += count[b]; dist_sum[b] += level * count[b];
//          max_dist[b] = level where count[b] > 0.
// The folds are integer and exact, so the reference's results follow
// bit-for-bit: closeness = reach / sum (an i64 sum in closeness_one), and the
// stats' f64 sums of integer distances are exact while the total stays below
// 2^53 (checked).  Costs O(n / 64 * levels * (m + n)).
#include <algorithm>
#include <cmath>
#include <vector>

#include "frontier.cuh"
#include "primitives.cuh"

namespace ug {

void dijkstra_run(TopoImpl* t, const double* d_weights, uint32_t source, int dir, double* d_out,
                  cudaStream_t s);

namespace {

__global__ void ms_init_k(const uint32_t* __restrict__ src, uint32_t k, unsigned long long* visited,
                          unsigned long long* frontier) {
  const uint32_t b = threadIdx.x;
  if (b < k) {
    atomicOr(&visited[src[b]], 1ull << b);
    atomicOr(&frontier[src[b]], 1ull << b);
  }
}

// next[w] |= frontier[v] & ~visited[w] over the in-edges v -> w of w.
__global__ void ms_pull_k(const uint32_t* __restrict__ in_off, const uint32_t* __restrict__ in_src,
                          uint64_t n, uint64_t m, const unsigned long long* __restrict__ frontier,
                          const unsigned long long* __restrict__ visited, unsigned long long* next) {
  for_each_slot_owner(in_off, n, m, [&](uint64_t k, uint32_t w) {
    const unsigned long long f = frontier[in_src[k]];
    if (f) {
      const unsigned long long add = f & ~visited[w];
      if (add) atomicOr(&next[w], add);
    }
  });
}

// Settles the level and counts, per source bit, the nodes first reached.
__global__ void ms_settle_k(uint64_t n, unsigned long long* __restrict__ visited,
                            unsigned long long* __restrict__ frontier,
                            unsigned long long* __restrict__ next,
                            unsigned long long* __restrict__ count) {
  __shared__ unsigned int sc[64];
  if (threadIdx.x < 64) sc[threadIdx.x] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n;
       base += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t w = base + threadIdx.x;
    unsigned long long nw = 0;
    if (w < n) {
      const unsigned long long nx = next[w];
      if (nx) {
        nw = nx & ~visited[w];
        visited[w] |= nw;
        next[w] = 0;
      }
      frontier[w] = nw;
    }
    if (__any_sync(0xffffffffu, nw != 0)) {
      // column popcount: bit b of the 32 lanes' masks
#pragma unroll 8
      for (int b = 0; b < 64; b++) {
        const unsigned c = __popc(__ballot_sync(0xffffffffu, (nw >> b) & 1ull));
        if (lane == 0 && c) atomicAdd(&sc[b], c);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < 64 && sc[threadIdx.x]) atomicAdd(&count[threadIdx.x], (unsigned long long)sc[threadIdx.x]);
}

// Folds one level's counts into the per-source results and reports whether
// any node was reached.
__global__ void ms_fold_k(uint32_t level, uint32_t k, unsigned long long* __restrict__ count,
                          unsigned long long* __restrict__ reach,
                          unsigned long long* __restrict__ dsum, uint32_t* __restrict__ maxd,
                          unsigned* __restrict__ any) {
  const uint32_t b = threadIdx.x;
  if (b < 64) {
    const unsigned long long c = count[b];
    count[b] = 0;
    if (b < k && c) {
      reach[b] += c;
      dsum[b] += (unsigned long long)level * c;
      maxd[b] = level;
      atomicOr(any, 1u);
    }
  }
}

}  // namespace

// Per-source BFS folds (reach = nodes at distance >= 1, dsum = their summed
// distances, maxd = eccentricity) for `sources` (host ids < n), following
// out-edges.  Outputs are host arrays of n_sources entries.
void msbfs_run(TopoImpl* t, const uint32_t* sources, uint64_t n_sources, uint64_t* reach,
               uint64_t* dsum, uint32_t* maxd, cudaStream_t s) {
  const uint64_t n = t->n, m = t->m;
  if (n_sources == 0) return;
  ensure_in(t, s);
  Scratch<unsigned long long> visited(n, s), frontier(n, s), next(n, s);
  Scratch<unsigned long long> count(64, s), d_reach(64, s), d_dsum(64, s);
  Scratch<uint32_t> d_maxd(64, s), d_src(64, s);
  Scratch<unsigned> any(1, s);
  UG_CUDA(cudaMemsetAsync(next.get(), 0, n * 8, s));
  UG_CUDA(cudaMemsetAsync(count.get(), 0, 64 * 8, s));
  for (uint64_t b0 = 0; b0 < n_sources; b0 += 64) {
    const uint32_t k = (uint32_t)std::min<uint64_t>(64, n_sources - b0);
    UG_CUDA(cudaMemsetAsync(visited.get(), 0, n * 8, s));
    UG_CUDA(cudaMemsetAsync(frontier.get(), 0, n * 8, s));
    UG_CUDA(cudaMemsetAsync(d_reach.get(), 0, 64 * 8, s));
    UG_CUDA(cudaMemsetAsync(d_dsum.get(), 0, 64 * 8, s));
    UG_CUDA(cudaMemsetAsync(d_maxd.get(), 0, 64 * 4, s));
    UG_CUDA(cudaMemcpyAsync(d_src.get(), sources + b0, k * 4, cudaMemcpyHostToDevice, s));
    ms_init_k<<<1, 64, 0, s>>>(d_src.get(), k, visited.get(), frontier.get());
    UG_LAUNCH_CHECK();
    for (uint32_t level = 1;; level++) {
      if (m) {
        ms_pull_k<<<grid_for(m, kBlock, 148u * 64u), kBlock, 0, s>>>(
            t->in.off.get(), t->in.tgt.get(), n, m, frontier.get(), visited.get(), next.get());
        UG_LAUNCH_CHECK();
      }
      ms_settle_k<<<grid_for(n), kBlock, 0, s>>>(n, visited.get(), frontier.get(), next.get(),
                                                 count.get());
      UG_LAUNCH_CHECK();
      UG_CUDA(cudaMemsetAsync(any.get(), 0, 4, s));
      ms_fold_k<<<1, 64, 0, s>>>(level, k, count.get(), d_reach.get(), d_dsum.get(), d_maxd.get(),
                                 any.get());
      UG_LAUNCH_CHECK();
      if (read_u32(any.get(), s) == 0) break;  // no node reached on this level
    }
    UG_CUDA(cudaMemcpyAsync(reach + b0, d_reach.get(), k * 8, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaMemcpyAsync(dsum + b0, d_dsum.get(), k * 8, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaMemcpyAsync(maxd + b0, d_maxd.get(), k * 4, cudaMemcpyDeviceToHost, s));
  }
  UG_CUDA(cudaStreamSynchronize(s));
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
