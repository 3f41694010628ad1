// tc.cu -- triangle_count and clustering_coefficient
// (ursa-core/src/algo/triangle.rs:23-62, clustering.rs:21-40).
//
// The reference counts, for every node u and neighbour a = N(u)[i], the
// common elements of N(u)[i+1..] and N(a): every triangle is counted once at
// each of its three vertices.  Here each undirected edge is oriented from
// the lower to the higher (degree, id) rank, which bounds every oriented
// list by O(sqrt(m)); each triangle {u, v, w} with rank u < v < w is then
// found exactly once, as w in N+(u) ∩ N+(v), and credited to all three
// vertices with integer atomics.  Integer results are order-independent, so
// the counts are bit-identical to the reference.
#include "frontier.cuh"

namespace ug {

namespace {

__device__ __forceinline__ bool rank_less(uint32_t du, uint32_t u, uint32_t dv, uint32_t v) {
  return du < dv || (du == dv && u < v);
}

__global__ void orient_flags_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                               uint64_t n, uint64_t ms, uint32_t* __restrict__ flag) {
  if (blockIdx.x == 0 && threadIdx.x == 0) flag[ms] = 0u;
  for_each_slot_owner(off, n, ms, [&](uint64_t k, uint32_t u) {
    uint32_t v = tgt[k];
    uint32_t du = off[u + 1] - off[u], dv = off[v + 1] - off[v];
    flag[k] = rank_less(du, u, dv, v) ? 1u : 0u;
  });
}

__global__ void orient_fill_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                              uint64_t n, uint64_t ms, const uint32_t* __restrict__ pos,
                              uint32_t* __restrict__ o_off, uint32_t* __restrict__ o_tgt) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < ms;
       k += (uint64_t)gridDim.x * blockDim.x) {
    if (pos[k + 1] != pos[k]) o_tgt[pos[k]] = tgt[k];
  }
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u <= n;
       u += (uint64_t)gridDim.x * blockDim.x)
    o_off[u] = pos[off[u]];
}

// Counting, one warp per vertex u at a time (vertices taken kTcGrab at a
// time from a global counter).  N+(u) goes into a hash set in the warp's
// shared memory (open addressing, load <= 1/2; lists longer than kTcHashMax
// are searched by binary search in global memory instead).  Then the
// concatenation of N+(v), v in N+(u), 32 lists at a time, is streamed with
// lane p taking element p (its list found by a warp scan of the lengths and
// a shuffle binary search), so every load is coalesced whatever the list
// lengths; a hit w in N+(u) is the triangle (u, v, w), credited to w at once
// and to v and u through per-list counters in shared memory.
constexpr int kTcThreads = 256;
constexpr int kTcWarps = kTcThreads / 32;
constexpr uint32_t kTcSlots = 2048;  // hash slots per warp
constexpr uint32_t kTcHashMax = kTcSlots / 2;
constexpr uint32_t kTcGrab = 16;
constexpr uint32_t kTcEmpty = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t tc_hash(uint32_t w, uint32_t bits) {
  return (w * 0x9E3779B1u) >> (32 - bits);
}

__global__ void __launch_bounds__(kTcThreads) count_warp_k(const uint32_t* __restrict__ o_off,
                                                          const uint32_t* __restrict__ o_tgt,
                                                          uint64_t n, uint32_t* __restrict__ tri,
                                                          unsigned long long* __restrict__ next) {
  extern __shared__ uint32_t tc_sm[];
  const uint32_t FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t* T = tc_sm + (size_t)w * kTcSlots;
  uint32_t* cnt = tc_sm + (size_t)kTcWarps * kTcSlots + w * 32;
  for (uint32_t i = lane; i < kTcSlots; i += 32) T[i] = kTcEmpty;
  cnt[lane] = 0;
  __syncwarp();
  while (true) {
    unsigned long long g = 0;
    if (lane == 0) g = atomicAdd(next, (unsigned long long)kTcGrab);
    g = __shfl_sync(FULL, g, 0);
    if (g >= n) break;
    const uint64_t g_end = g + kTcGrab < n ? g + kTcGrab : n;
    for (uint64_t u = g; u < g_end; u++) {
      const uint32_t ob = o_off[u], oe = o_off[u + 1], du = oe - ob;
      if (du < 2) continue;  // u is the lowest vertex of no triangle
      const bool hashed = du <= kTcHashMax;
      uint32_t bits = 6;
      while ((1u << bits) < 2 * du) bits++;
      const uint32_t mask = (1u << bits) - 1;
      if (hashed) {
        for (uint32_t i = ob + lane; i < oe; i += 32) {
          const uint32_t x = o_tgt[i];
          uint32_t h = tc_hash(x, bits);
          while (atomicCAS(&T[h], kTcEmpty, x) != kTcEmpty) h = (h + 1) & mask;
        }
        __syncwarp();
      }
      uint32_t cu = 0;
      for (uint32_t vb = ob; vb < oe; vb += 32) {
        const uint32_t i = vb + lane;
        uint32_t v = 0, st = 0, len = 0;
        if (i < oe) {
          v = o_tgt[i];
          st = o_off[v];
          len = o_off[v + 1] - st;
        }
        uint32_t incl = len;  // inclusive scan of the list lengths
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(FULL, incl, o);
          if (lane >= o) incl += t;
        }
        const uint32_t total = __shfl_sync(FULL, incl, 31);
        for (uint32_t pb = 0; pb < total; pb += 32) {
          const uint32_t p = pb + lane;
          uint32_t j = 0;  // first list whose inclusive end exceeds p
#pragma unroll
          for (int step = 16; step >= 1; step >>= 1) {
            const uint32_t t = __shfl_sync(FULL, incl, j + step - 1);
            if (t <= p) j += step;
          }
          const uint32_t sj = __shfl_sync(FULL, st, j & 31);
          const uint32_t ij = __shfl_sync(FULL, incl, j & 31);
          const uint32_t lj = __shfl_sync(FULL, len, j & 31);
          if (p < total) {
            const uint32_t x = o_tgt[sj + (p - (ij - lj))];
            bool hit = false;
            if (hashed) {
              uint32_t h = tc_hash(x, bits);
              while (true) {
                const uint32_t t = T[h];
                if (t == x) {
                  hit = true;
                  break;
                }
                if (t == kTcEmpty) break;
                h = (h + 1) & mask;
              }
            } else {
              uint32_t lo = ob, hi = oe;
              while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (o_tgt[mid] < x) lo = mid + 1; else hi = mid;
              }
              hit = lo < oe && o_tgt[lo] == x;
            }
            if (hit) {
              atomicAdd(&tri[x], 1u);
              atomicAdd(&cnt[j], 1u);
            }
          }
        }
        __syncwarp();
        const uint32_t c = cnt[lane];
        if (c) {
          atomicAdd(&tri[v], c);
          cu += c;
          cnt[lane] = 0;
        }
        __syncwarp();
      }
      cu = __reduce_add_sync(FULL, cu);
      if (lane == 0 && cu) atomicAdd(&tri[u], cu);
      if (hashed) {
        __syncwarp();
        for (uint32_t k = lane; k <= mask; k += 32) T[k] = kTcEmpty;
        __syncwarp();
      }
    }
  }
}

size_t tc_smem_bytes() { return ((size_t)kTcWarps * kTcSlots + kTcWarps * 32) * sizeof(uint32_t); }

// clustering.rs:21-40: 2 T / (k (k - 1)), 0.0 for k < 2, in f64.
__global__ void clustering_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tri,
                             uint64_t n, double* __restrict__ out) {
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    double k = (double)(off[u + 1] - off[u]);
    out[u] = k < 2.0 ? 0.0 : __ddiv_rn(__dmul_rn(2.0, (double)tri[u]), __dmul_rn(k, __dsub_rn(k, 1.0)));
  }
}

}  // namespace

// Orientation of the undirected CSR (host-synchronising; done once).
void orient_build(TopoImpl* t, OrientedCsr& o, cudaStream_t s) {
  const uint64_t n = t->n;
  ensure_undirected(t, s);
  const uint64_t ms = t->m_und;
  o.off.alloc(n + 1, s);
  o.mo = 0;
  if (ms == 0) {
    UG_CUDA(cudaMemsetAsync(o.off.get(), 0, (n + 1) * sizeof(uint32_t), s));
    o.tgt.alloc(1, s);
    return;
  }
  Scratch<uint32_t> pos(ms + 1, s);
  orient_flags_k<<<grid_for(ms), kBlock, 0, s>>>(t->und_off.get(), t->und_tgt.get(), n, ms,
                                                 pos.get());
  UG_LAUNCH_CHECK();
  Scratch<uint32_t> total(1, s);
  exclusive_scan_u32(pos.get(), pos.get(), ms + 1, total.get(), s);
  o.mo = read_u32(total.get(), s);
  o.tgt.alloc(o.mo ? o.mo : 1, s);
  orient_fill_k<<<grid_for(ms), kBlock, 0, s>>>(t->und_off.get(), t->und_tgt.get(), n, ms,
                                                pos.get(), o.off.get(), o.tgt.get());
  UG_LAUNCH_CHECK();
}

// Triangle counts from an oriented CSR: kernels only, so it can be captured
// into a CUDA graph.
void triangle_count_oriented(const OrientedCsr& o, uint64_t n, uint32_t* d_tri, cudaStream_t s) {
  UG_CUDA(cudaMemsetAsync(d_tri, 0, n * sizeof(uint32_t), s));
  if (o.mo) {
    int dev = 0;
    UG_CUDA(cudaGetDevice(&dev));
    UG_CHECK(dev >= 0 && dev < 64, URSA_GPU_EINVAL, "device index out of range");
    static std::mutex mu;
    static int per_sm_of[64] = {0};  // blocks per SM, once the smem limit is raised on that device
    int per_sm = 0;
    {
      std::lock_guard<std::mutex> g(mu);
      if (!per_sm_of[dev]) {
        UG_CUDA(cudaFuncSetAttribute(count_warp_k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)tc_smem_bytes()));
        UG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_of[dev], count_warp_k,
                                                              kTcThreads, tc_smem_bytes()));
        UG_CHECK(per_sm_of[dev] > 0, URSA_GPU_ECUDA, "triangle kernel cannot be resident");
      }
      per_sm = per_sm_of[dev];
    }
    Scratch<unsigned long long> next(1, s);
    UG_CUDA(cudaMemsetAsync(next.get(), 0, sizeof(unsigned long long), s));
    count_warp_k<<<per_sm * sm_count(dev), kTcThreads, tc_smem_bytes(), s>>>(o.off.get(), o.tgt.get(),
                                                                             n, d_tri, next.get());
    UG_LAUNCH_CHECK();
  }
}

void triangle_count_run(TopoImpl* t, uint32_t* d_tri, cudaStream_t s) {
  const uint64_t n = t->n;
  if (n == 0) return;
  OrientedCsr o;
  orient_build(t, o, s);
  triangle_count_oriented(o, n, d_tri, s);
  UG_CUDA(cudaStreamSynchronize(s));  // o's buffers are released on return
}

void clustering_run(TopoImpl* t, double* d_out, cudaStream_t s) {
  const uint64_t n = t->n;
  if (n == 0) return;
  Scratch<uint32_t> tri(n, s);
  triangle_count_run(t, tri.get(), s);
  clustering_k<<<grid_for(n), kBlock, 0, s>>>(t->und_off.get(), tri.get(), n, d_out);
  UG_LAUNCH_CHECK();
}

}  // namespace ug

using namespace ug;

extern "C" {

int ursa_gpu_triangle_count(ursa_gpu_topo* t, uint32_t* out) {
  return guard([&] {
    UG_CHECK(t, URSA_GPU_EINVAL, "topology is NULL");
    TopoImpl* ti = &t->impl;
    if (ti->n == 0) return;  // triangle.rs:56-58
    UG_CHECK(out, URSA_GPU_EINVAL, "out is NULL");
    cudaStream_t s = thread_stream(ti->device);
    Scratch<uint32_t> d(ti->n, s);
    triangle_count_run(ti, d.get(), s);
    UG_CUDA(cudaMemcpyAsync(out, d.get(), ti->n * 4, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_clustering_coefficient(ursa_gpu_topo* t, double* out) {
  return guard([&] {
    UG_CHECK(t, URSA_GPU_EINVAL, "topology is NULL");
    TopoImpl* ti = &t->impl;
    if (ti->n == 0) return;  // clustering.rs:23-25
    UG_CHECK(out, URSA_GPU_EINVAL, "out is NULL");
    cudaStream_t s = thread_stream(ti->device);
    Scratch<double> d(ti->n, s);
    clustering_run(ti, d.get(), s);
    UG_CUDA(cudaMemcpyAsync(out, d.get(), ti->n * 8, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

}  // extern "C"
