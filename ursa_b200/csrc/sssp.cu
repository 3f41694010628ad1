// sssp.cu -- weighted shortest paths (ursa-core/src/algo/bfs.rs:126-259).
//
// dijkstra_distances: frontier Bellman-Ford.  Distances are non-negative
// doubles, whose IEEE bit patterns order like u64, so a relaxation is one
// atomicMin on the bits.  Every improvement re-queues the node (once per
// round, flag-deduplicated) until nothing changes.  The fixpoint is the same
// set of f64 values Dijkstra settles: dist[v] = min over edges of
// fl(dist[u] + w), and fl(a + w) is monotone in a with fl(a + w) >= a for
// w >= 0, so both compute the minimum left-to-right f64 path sum.
//
// shortest_path_weighted_with_cost: distances as above, then the path is
// walked back from the target.  The reference's parent of v is the first
// node, in Dijkstra's settle order, whose relaxation produced dist[v]
// (strict '<' at bfs.rs:237); with positive weights the settle order is the
// heap order (dist, node id), so the parent is the tight predecessor u
// (fl(dist[u] + w) == dist[v]) with the smallest (dist[u], u).  With
// zero-weight edges Dijkstra's settle order among equal distances depends on
// discovery order; there the path is a valid minimum-cost path but may pick
// a different tie.
#include <vector>

#include "frontier.cuh"

namespace ug {

namespace {

constexpr unsigned long long kInfBits = 0x7FF0000000000000ull;

__device__ __forceinline__ void append_w(uint32_t* Q, uint32_t* cnt, bool take, uint32_t v) {
  uint32_t mask = __ballot_sync(0xffffffffu, take);
  if (!take) return;
  int lane = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(cnt, (uint32_t)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  Q[base + __popc(mask & ((1u << lane) - 1u))] = v;
}

__device__ __forceinline__ unsigned long long ld_bits(const unsigned long long* p) {
  return *(const volatile unsigned long long*)p;
}

__global__ void relax_k(DirView d, const double* __restrict__ w0, const double* __restrict__ w1,
                        const uint32_t* __restrict__ F, uint64_t f, const uint64_t* __restrict__ pos,
                        uint64_t T, unsigned long long* dist, uint32_t* inq, uint32_t* __restrict__ N,
                        uint32_t* __restrict__ cnt) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t span = ((T + stride - 1) / stride) * stride;  // warp-uniform trip count
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < span; e += stride) {
    bool take = false;
    uint32_t v = 0;
    if (e < T) {
      uint64_t i = owner_in_pos(pos, f, e);
      uint32_t u = F[i];
      uint32_t slot;
      bool second;
      v = dv_nbr(d, u, (uint32_t)(e - pos[i]), &slot, &second);
      double w = second ? w1[slot] : w0[slot];
      double nd = __dadd_rn(__longlong_as_double((long long)ld_bits(&dist[u])), w);
      unsigned long long nb = (unsigned long long)__double_as_longlong(nd);
      if (nb < ld_bits(&dist[v])) {
        unsigned long long old = atomicMin(&dist[v], nb);
        if (nb < old) take = atomicExch(&inq[v], 1u) == 0u;
      }
    }
    append_w(N, cnt, take, v);
  }
}

__global__ void unqueue_k(const uint32_t* __restrict__ N, uint32_t cnt, uint32_t* __restrict__ inq) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += (uint64_t)gridDim.x * blockDim.x)
    inq[N[i]] = 0u;
}

// Hop levels over tight edges (fl(dist[u] + w) == dist[v]) from the source;
// used to walk paths when zero-weight edges create equal-distance ties.
__global__ void tight_level_k(DirView d, const double* __restrict__ w0, const double* __restrict__ w1,
                              const uint32_t* __restrict__ F, uint64_t f,
                              const uint64_t* __restrict__ pos, uint64_t T,
                              const unsigned long long* __restrict__ dist, int32_t* level,
                              int32_t lvl, uint32_t* __restrict__ N, uint32_t* __restrict__ cnt) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t span = ((T + stride - 1) / stride) * stride;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < span; e += stride) {
    bool take = false;
    uint32_t v = 0;
    if (e < T) {
      uint64_t i = owner_in_pos(pos, f, e);
      uint32_t u = F[i];
      uint32_t slot;
      bool second;
      v = dv_nbr(d, u, (uint32_t)(e - pos[i]), &slot, &second);
      double w = second ? w1[slot] : w0[slot];
      double nd = __dadd_rn(__longlong_as_double((long long)dist[u]), w);
      if ((unsigned long long)__double_as_longlong(nd) == dist[v] && dist[v] != kInfBits &&
          level[v] < 0)
        take = atomicCAS(&level[v], -1, lvl + 1) == -1;
    }
    append_w(N, cnt, take, v);
  }
}

__global__ void fill_u64_k(unsigned long long* p, uint64_t n, unsigned long long v) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

__global__ void seed_k(unsigned long long* dist, uint32_t* F, uint32_t source) {
  dist[source] = 0ull;  // +0.0
  F[0] = source;
}

// One block walks the path back from the target: at node v it scans the
// reverse adjacency for tight predecessors and keeps the smallest
// (dist, id), restricted to (dist[u], u) < (dist[v], v) so a zero-weight
// cycle cannot loop -- or, when level is given, to predecessors one tight
// hop closer to the source.
__global__ void weighted_backtrack_k(DirView rev, const double* __restrict__ rw0,
                                     const double* __restrict__ rw1,
                                     const unsigned long long* __restrict__ dist,
                                     const int32_t* __restrict__ level, uint32_t source,
                                     uint32_t target, uint64_t cap, uint32_t* __restrict__ path,
                                     unsigned long long* __restrict__ out_len) {
  __shared__ unsigned long long best_d[kBlock / 32];
  __shared__ uint32_t best_u[kBlock / 32];
  __shared__ uint32_t s_cur;
  __shared__ uint64_t s_len;
  __shared__ int s_fail;
  if (threadIdx.x == 0) {
    s_cur = target;
    s_len = 0;
    s_fail = 0;
    path[0] = target;
    s_len = 1;
  }
  __syncthreads();
  while (true) {
    uint32_t v = s_cur;
    if (v == source || s_fail || s_len >= cap) break;
    unsigned long long dv = dist[v];
    double dvd = __longlong_as_double((long long)dv);
    unsigned long long bd = ~0ull;
    uint32_t bu = 0xFFFFFFFFu;
    uint32_t deg = dv_deg(rev, v);
    for (uint32_t j = threadIdx.x; j < deg; j += blockDim.x) {
      uint32_t slot;
      bool second;
      uint32_t u = dv_nbr(rev, v, j, &slot, &second);
      if (u == v) continue;
      unsigned long long du = dist[u];
      if (du == kInfBits) continue;
      double w = second ? rw1[slot] : rw0[slot];
      double nd = __dadd_rn(__longlong_as_double((long long)du), w);
      if ((unsigned long long)__double_as_longlong(nd) != dv || !(nd == dvd)) continue;
      bool before = level ? (level[u] >= 0 && level[u] + 1 == level[v])
                          : (du < dv || (du == dv && u < v));
      if (!before) continue;
      if (du < bd || (du == bd && u < bu)) {
        bd = du;
        bu = u;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      unsigned long long od = __shfl_down_sync(0xffffffffu, bd, o);
      uint32_t ou = __shfl_down_sync(0xffffffffu, bu, o);
      if (od < bd || (od == bd && ou < bu)) {
        bd = od;
        bu = ou;
      }
    }
    if ((threadIdx.x & 31) == 0) {
      best_d[threadIdx.x >> 5] = bd;
      best_u[threadIdx.x >> 5] = bu;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long fd = ~0ull;
      uint32_t fu = 0xFFFFFFFFu;
      for (int k = 0; k < (int)(blockDim.x / 32); k++)
        if (best_d[k] < fd || (best_d[k] == fd && best_u[k] < fu)) {
          fd = best_d[k];
          fu = best_u[k];
        }
      if (fu == 0xFFFFFFFFu) {
        s_fail = 1;
      } else {
        path[s_len] = fu;
        s_len = s_len + 1;
        s_cur = fu;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *out_len = s_fail ? 0ull : s_len;
}

__global__ void bits_to_costs_k(const uint32_t* __restrict__ path, uint64_t len,
                                const unsigned long long* __restrict__ dist,
                                double* __restrict__ cost) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (uint64_t)gridDim.x * blockDim.x)
    cost[i] = __longlong_as_double((long long)dist[path[i]]);
}

}  // namespace

// Distances from source over view d with per-slot weights w0/w1 into
// dist (n u64 bit patterns of f64, +inf = unreachable).
void sssp_run(const DirView& d, const double* w0, const double* w1, uint64_t n, uint32_t source,
              unsigned long long* dist, cudaStream_t s) {
  fill_u64_k<<<grid_for(n), kBlock, 0, s>>>(dist, n, kInfBits);
  UG_LAUNCH_CHECK();
  if ((uint64_t)source >= n) return;
  FrontierBufs b;
  b.alloc(n, s);
  Scratch<uint32_t> inq(n, s);
  UG_CUDA(cudaMemsetAsync(inq.get(), 0, n * sizeof(uint32_t), s));
  seed_k<<<1, 1, 0, s>>>(dist, b.F.get(), source);
  UG_LAUNCH_CHECK();
  uint32_t f = 1;
  while (f > 0) {
    uint64_t T = frontier_scan(d, b.F.get(), f, b.pos.get(), s);
    if (T == 0) break;
    UG_CUDA(cudaMemsetAsync(b.count.get(), 0, sizeof(uint32_t), s));
    relax_k<<<grid_for(T, kBlock, 148u * 64u), kBlock, 0, s>>>(d, w0, w1, b.F.get(), f, b.pos.get(),
                                                                T, dist, inq.get(), b.N.get(),
                                                                b.count.get());
    UG_LAUNCH_CHECK();
    uint32_t next = read_u32(b.count.get(), s);
    if (next) {
      unqueue_k<<<grid_for(next), kBlock, 0, s>>>(b.N.get(), next, inq.get());
      UG_LAUNCH_CHECK();
    }
    swap(b.F, b.N);
    f = next;
  }
}

void dijkstra_run(TopoImpl* t, const double* d_weights, uint32_t source, int dir, double* d_out,
                  cudaStream_t s) {
  DirView d = dir_view(t, dir, s);
  DirWeights w;
  gather_dir_weights(t, d, d_weights, w, s);
  sssp_run(d, w.w0.get(), w.w1.get(), t->n, source, (unsigned long long*)d_out, s);
}

int64_t weighted_path_run(TopoImpl* t, const double* d_weights, uint32_t source, uint32_t target,
                          int dir, uint32_t* path, double* costs, uint64_t cap, cudaStream_t s) {
  const uint64_t n = t->n;
  if ((uint64_t)source >= n || (uint64_t)target >= n) return -1;  // bfs.rs:208-210
  if (source == target) {                                          // bfs.rs:211-213
    UG_CHECK(cap >= 1, URSA_GPU_ETRUNC, "path buffer too small");
    path[0] = source;
    if (costs) costs[0] = 0.0;
    return 1;
  }
  DirView d = dir_view(t, dir, s);
  DirWeights w;
  gather_dir_weights(t, d, d_weights, w, s);
  Scratch<unsigned long long> dist(n, s);
  sssp_run(d, w.w0.get(), w.w1.get(), n, source, dist.get(), s);
  unsigned long long dt = 0;
  UG_CUDA(cudaMemcpyAsync(&dt, dist.get() + target, 8, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  if (dt == kInfBits) return -1;  // unreachable (bfs.rs:245-247)
  DirView rv = reverse_view(t, dir, s);
  DirWeights rw;
  gather_dir_weights(t, rv, d_weights, rw, s);
  Scratch<uint32_t> dpath(n, s);
  Scratch<unsigned long long> dlen(1, s);
  weighted_backtrack_k<<<1, kBlock, 0, s>>>(rv, rw.w0.get(), rw.w1.get(), dist.get(), nullptr,
                                            source, target, n, dpath.get(), dlen.get());
  UG_LAUNCH_CHECK();
  unsigned long long len = 0;
  UG_CUDA(cudaMemcpyAsync(&len, dlen.get(), 8, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  if (len == 0) {
    // Zero-weight ties: walk back along hop levels of the tight-edge graph.
    Scratch<int32_t> level(n, s);
    UG_CUDA(cudaMemsetAsync(level.get(), 0xFF, n * sizeof(int32_t), s));
    FrontierBufs b;
    b.alloc(n, s);
    UG_CUDA(cudaMemsetAsync(level.get() + source, 0, sizeof(int32_t), s));
    UG_CUDA(cudaMemcpyAsync(b.F.get(), &source, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    uint32_t f = 1;
    int32_t lvl = 0;
    while (f > 0) {
      uint64_t T = frontier_scan(d, b.F.get(), f, b.pos.get(), s);
      if (T == 0) break;
      UG_CUDA(cudaMemsetAsync(b.count.get(), 0, sizeof(uint32_t), s));
      tight_level_k<<<grid_for(T, kBlock, 148u * 64u), kBlock, 0, s>>>(
          d, w.w0.get(), w.w1.get(), b.F.get(), f, b.pos.get(), T, dist.get(), level.get(), lvl,
          b.N.get(), b.count.get());
      UG_LAUNCH_CHECK();
      uint32_t next = read_u32(b.count.get(), s);
      swap(b.F, b.N);
      f = next;
      lvl++;
    }
    weighted_backtrack_k<<<1, kBlock, 0, s>>>(rv, rw.w0.get(), rw.w1.get(), dist.get(), level.get(),
                                              source, target, n, dpath.get(), dlen.get());
    UG_LAUNCH_CHECK();
    UG_CUDA(cudaMemcpyAsync(&len, dlen.get(), 8, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  }
  UG_CHECK(len > 0, URSA_GPU_EINVAL, "weighted path walk found no predecessor");
  if (len > cap) return -(int64_t)len - 2;
  // reverse into forward order on the host copy
  std::vector<uint32_t> h(len);
  UG_CUDA(cudaMemcpyAsync(h.data(), dpath.get(), len * 4, cudaMemcpyDeviceToHost, s));
  Scratch<double> dcost(len, s);
  std::vector<double> hc(len);
  if (costs) {
    bits_to_costs_k<<<grid_for(len), kBlock, 0, s>>>(dpath.get(), len, dist.get(), dcost.get());
    UG_LAUNCH_CHECK();
    UG_CUDA(cudaMemcpyAsync(hc.data(), dcost.get(), len * 8, cudaMemcpyDeviceToHost, s));
  }
  UG_CUDA(cudaStreamSynchronize(s));
  for (uint64_t i = 0; i < len; i++) {
    path[i] = h[len - 1 - i];
    if (costs) costs[i] = hc[len - 1 - i];
  }
  return (int64_t)len;
}

}  // namespace ug

using namespace ug;

extern "C" {

int ursa_gpu_dijkstra_distances(ursa_gpu_topo* t, const double* weights, uint64_t n_weights,
                                uint32_t source, int dir, double* out) {
  return guard([&] {
    UG_CHECK(t, URSA_GPU_EINVAL, "topology is NULL");
    UG_CHECK(dir >= 0 && dir <= 2, URSA_GPU_EINVAL, "direction must be 0, 1 or 2");
    TopoImpl* ti = &t->impl;
    UG_CHECK(n_weights == ti->m, URSA_GPU_EINVAL, "weights length must equal the edge count");
    UG_CHECK(ti->m == 0 || weights, URSA_GPU_EINVAL, "weights is NULL");
    if (ti->n == 0) return;
    UG_CHECK(out, URSA_GPU_EINVAL, "out is NULL");
    cudaStream_t s = thread_stream(ti->device);
    Scratch<double> dw(ti->m ? ti->m : 1, s), dout(ti->n, s);
    if (ti->m) UG_CUDA(cudaMemcpyAsync(dw.get(), weights, ti->m * 8, cudaMemcpyHostToDevice, s));
    check_sssp_weights_device(dw.get(), ti->m, s);
    dijkstra_run(ti, dw.get(), source, dir, dout.get(), s);
    UG_CUDA(cudaMemcpyAsync(out, dout.get(), ti->n * 8, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_shortest_path_weighted_with_cost(ursa_gpu_topo* t, const double* weights,
                                              uint64_t n_weights, uint32_t source,
                                              uint32_t target, int dir, uint32_t* path,
                                              double* costs, uint64_t cap, int64_t* len) {
  return guard([&] {
    UG_CHECK(t && len, URSA_GPU_EINVAL, "topology or len is NULL");
    UG_CHECK(dir >= 0 && dir <= 2, URSA_GPU_EINVAL, "direction must be 0, 1 or 2");
    *len = -1;
    TopoImpl* ti = &t->impl;
    UG_CHECK(n_weights == ti->m, URSA_GPU_EINVAL, "weights length must equal the edge count");
    UG_CHECK(ti->m == 0 || weights, URSA_GPU_EINVAL, "weights is NULL");
    cudaStream_t s = thread_stream(ti->device);
    Scratch<double> dw(ti->m ? ti->m : 1, s);
    if (ti->m) UG_CUDA(cudaMemcpyAsync(dw.get(), weights, ti->m * 8, cudaMemcpyHostToDevice, s));
    check_sssp_weights_device(dw.get(), ti->m, s);
    int64_t r = weighted_path_run(ti, dw.get(), source, target, dir, path, costs, cap, s);
    if (r < -1) {
      *len = -r - 2;
      throw Error(URSA_GPU_ETRUNC, "path buffer too small");
    }
    *len = r;
  });
}

}  // extern "C"
