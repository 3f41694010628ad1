// frontier.cu -- BFS family on the device (ursa-core/src/algo/bfs.rs, hop.rs).
//
//  * bfs_distances: level-synchronous, direction-optimising (top-down frontier
//    queue while the frontier's edges are few, bottom-up over unvisited nodes
//    when they are many, Beamer et al.); levels are exact, so the output is
//    bit-identical to the reference's serial BFS.
//  * k_hop / shortest_path: exact-order expansion.  The reference walks the
//    frontier in order and each node's neighbours in CSR order, and the first
//    walk that reaches v discovers it (hop.rs:106-123, bfs.rs:69-87).  Here
//    every frontier edge gets its rank e in that walk (a prefix sum of the
//    frontier degrees), unvisited targets take atomicMin(claim[v], e), and a
//    stable compaction of the winning edges emits the next frontier in the
//    reference's order, with parent[v] = the winning edge's source.  Pairs,
//    parents and paths are therefore identical to the reference's.
#include <algorithm>
#include <vector>

#include "frontier.cuh"

namespace ug {

DirView dir_view(TopoImpl* t, int dir, cudaStream_t s) {
  if (dir != 0) ensure_in(t, s);
  DirView d{};
  if (dir == 0 || dir == 2) {
    d.off0 = t->out.off.get();
    d.tgt0 = t->out.tgt.get();
    d.eid0 = t->out.eid.get();
    if (dir == 2) {
      d.off1 = t->in.off.get();
      d.tgt1 = t->in.tgt.get();
      d.eid1 = t->in.eid.get();
    }
  } else {
    d.off0 = t->in.off.get();
    d.tgt0 = t->in.tgt.get();
    d.eid0 = t->in.eid.get();
  }
  return d;
}

DirView reverse_view(TopoImpl* t, int dir, cudaStream_t s) {
  if (dir == 0) return dir_view(t, 1, s);
  if (dir == 1) return dir_view(t, 0, s);
  return dir_view(t, 2, s);
}

namespace {

__global__ void fdeg_k(DirView d, const uint32_t* __restrict__ F, uint64_t f,
                       uint64_t* __restrict__ pos) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= f;
       i += (uint64_t)gridDim.x * blockDim.x)
    pos[i] = i < f ? dv_deg(d, F[i]) : 0ull;
}

__global__ void gather_w_k(const uint32_t* __restrict__ eid, const double* __restrict__ w,
                           uint64_t m, double* __restrict__ out) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m;
       k += (uint64_t)gridDim.x * blockDim.x)
    out[k] = w[eid[k]];
}

__global__ void claim_k(DirView d, const uint32_t* __restrict__ F, uint64_t f,
                        const uint64_t* __restrict__ pos, uint64_t T,
                        const uint8_t* __restrict__ visited, unsigned long long* claim) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < T;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t i = owner_in_pos(pos, f, e);
    uint32_t v = dv_nbr(d, F[i], (uint32_t)(e - pos[i]));
    if (!visited[v] && claim[v] > e) atomicMin(&claim[v], (unsigned long long)e);
  }
}

__global__ void win_flag_k(DirView d, const uint32_t* __restrict__ F, uint64_t f,
                           const uint64_t* __restrict__ pos, uint64_t T,
                           const uint8_t* __restrict__ visited,
                           const unsigned long long* __restrict__ claim,
                           uint32_t* __restrict__ flag) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < T;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t i = owner_in_pos(pos, f, e);
    uint32_t v = dv_nbr(d, F[i], (uint32_t)(e - pos[i]));
    flag[e] = (!visited[v] && claim[v] == e) ? 1u : 0u;
  }
}

__global__ void win_emit_k(DirView d, const uint32_t* __restrict__ F, uint64_t f,
                           const uint64_t* __restrict__ pos, uint64_t T,
                           const uint8_t* __restrict__ visited,
                           const unsigned long long* __restrict__ claim,
                           const uint32_t* __restrict__ at, uint32_t* __restrict__ N,
                           uint32_t* __restrict__ parent) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < T;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t i = owner_in_pos(pos, f, e);
    uint32_t u = F[i];
    uint32_t v = dv_nbr(d, u, (uint32_t)(e - pos[i]));
    if (!visited[v] && claim[v] == e) {
      N[at[e]] = v;
      if (parent) parent[v] = u;
    }
  }
}

__global__ void mark_k(const uint32_t* __restrict__ N, uint32_t cnt, uint8_t* __restrict__ visited,
                       unsigned long long* __restrict__ claim) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t v = N[i];
    visited[v] = 1;
    claim[v] = ~0ull;
  }
}

__global__ void unmark_k(const uint32_t* __restrict__ N, uint64_t cnt, uint8_t* __restrict__ visited) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += (uint64_t)gridDim.x * blockDim.x)
    visited[N[i]] = 0;
}

__global__ void set_one_u8_k(uint8_t* p, uint64_t i, uint8_t v) { p[i] = v; }
__global__ void set_one_u32_k(uint32_t* p, uint64_t i, uint32_t v) { p[i] = v; }
__global__ void set_one_i32_k(int32_t* p, uint64_t i, int32_t v) { p[i] = v; }
__global__ void fill_u32_k(uint32_t* p, uint64_t n, uint32_t v) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

// Warp-aggregated append of v to Q (count at *cnt).
__device__ __forceinline__ void append(uint32_t* Q, uint32_t* cnt, bool take, uint32_t v) {
  uint32_t mask = __ballot_sync(__activemask(), take);
  if (!take) return;
  int lane = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(cnt, (uint32_t)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  Q[base + __popc(mask & ((1u << lane) - 1u))] = v;
}

// Adds, per warp, the forward degrees of the nodes this round appended to the
// next frontier (the next level's scout count, read with the frontier size).
__device__ __forceinline__ void add_scout(DirView fwd, bool take, uint32_t v,
                                          unsigned long long* __restrict__ scout) {
  unsigned long long x = take ? (unsigned long long)dv_deg(fwd, v) : 0ull;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  if ((threadIdx.x & 31) == 0 && x) atomicAdd(scout, x);
}

__global__ void td_k(DirView d, const uint32_t* __restrict__ F, uint64_t f,
                     const uint64_t* __restrict__ pos, uint64_t T, int32_t* dist, int32_t level,
                     uint32_t* __restrict__ N, uint32_t* __restrict__ cnt,
                     unsigned long long* __restrict__ scout) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t span = ((T + stride - 1) / stride) * stride;  // whole warps iterate together
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < span; e += stride) {
    bool take = false;
    uint32_t v = 0;
    if (e < T) {
      uint64_t i = owner_in_pos(pos, f, e);
      v = dv_nbr(d, F[i], (uint32_t)(e - pos[i]));
      if (dist[v] < 0) take = atomicCAS(&dist[v], -1, level + 1) == -1;
    }
    append(N, cnt, take, v);
    add_scout(d, take, v, scout);
  }
}

__global__ void bu_k(DirView rev, DirView fwd, uint64_t n, int32_t* dist, int32_t level,
                     uint32_t* __restrict__ N, uint32_t* __restrict__ cnt,
                     unsigned long long* __restrict__ scout) {
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t span = ((n + stride - 1) / stride) * stride;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < span; v += stride) {
    bool take = false;
    if (v < n && dist[v] < 0) {
      uint32_t deg = dv_deg(rev, (uint32_t)v);
      for (uint32_t j = 0; j < deg; j++) {
        uint32_t u = dv_nbr(rev, (uint32_t)v, j);
        if (dist[u] == level) {
          dist[v] = level + 1;
          take = true;
          break;
        }
      }
    }
    append(N, cnt, take, (uint32_t)v);
    add_scout(fwd, take, (uint32_t)v, scout);
  }
}

// Walk parents from target back to source into path (reversed at the end).
__global__ void backtrack_k(const uint32_t* __restrict__ parent, uint32_t source, uint32_t target,
                            uint64_t cap, uint32_t* __restrict__ path, uint64_t* __restrict__ len) {
  uint64_t l = 0;
  uint32_t cur = target;
  path[l++] = cur;
  while (cur != source && l < cap) {
    cur = parent[cur];
    path[l++] = cur;
  }
  for (uint64_t i = 0; i < l / 2; i++) {
    uint32_t x = path[i];
    path[i] = path[l - 1 - i];
    path[l - 1 - i] = x;
  }
  *len = l;
}

__global__ void fill_seed_k(uint32_t* p, uint64_t n, uint32_t v) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

}  // namespace

uint64_t frontier_scan(const DirView& d, const uint32_t* F, uint64_t f, uint64_t* pos,
                       cudaStream_t s) {
  fdeg_k<<<grid_for(f + 1), kBlock, 0, s>>>(d, F, f, pos);
  UG_LAUNCH_CHECK();
  exclusive_scan_u64(pos, pos, f + 1, nullptr, s);
  uint64_t total = 0;
  UG_CUDA(cudaMemcpyAsync(&total, pos + f, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  return total;
}

void gather_dir_weights(TopoImpl* t, const DirView& d, const double* d_weights, DirWeights& out,
                        cudaStream_t s) {
  uint64_t m = t->m;
  out.w0.alloc(m ? m : 1, s);
  if (m) {
    gather_w_k<<<grid_for(m), kBlock, 0, s>>>(d.eid0, d_weights, m, out.w0.get());
    UG_LAUNCH_CHECK();
  }
  if (d.off1) {
    out.w1.alloc(m ? m : 1, s);
    if (m) {
      gather_w_k<<<grid_for(m), kBlock, 0, s>>>(d.eid1, d_weights, m, out.w1.get());
      UG_LAUNCH_CHECK();
    }
  }
}

uint32_t read_u32(const uint32_t* d, cudaStream_t s) {
  uint32_t h = 0;
  UG_CUDA(cudaMemcpyAsync(&h, d, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  return h;
}

uint32_t expand_exact(const DirView& d, uint64_t n, const uint32_t* F, uint32_t f, uint32_t* N,
                      uint8_t* visited, unsigned long long* claim, uint32_t* parent,
                      uint64_t* pos, Scratch<uint32_t>& flag_buf, cudaStream_t s) {
  (void)n;
  uint64_t T = frontier_scan(d, F, f, pos, s);
  if (T == 0) return 0;
  UG_CHECK(T < (1ull << 32), URSA_GPU_EINVAL, "frontier expansion above 2^32 edges");
  if (flag_buf.n < T) flag_buf.alloc(T, s);
  unsigned g = grid_for(T, kBlock, 148u * 64u);
  claim_k<<<g, kBlock, 0, s>>>(d, F, f, pos, T, visited, claim);
  UG_LAUNCH_CHECK();
  win_flag_k<<<g, kBlock, 0, s>>>(d, F, f, pos, T, visited, claim, flag_buf.get());
  UG_LAUNCH_CHECK();
  Scratch<uint32_t> total(1, s);
  exclusive_scan_u32(flag_buf.get(), flag_buf.get(), T, total.get(), s);
  win_emit_k<<<g, kBlock, 0, s>>>(d, F, f, pos, T, visited, claim, flag_buf.get(), N, parent);
  UG_LAUNCH_CHECK();
  uint32_t cnt = read_u32(total.get(), s);
  if (cnt) {
    mark_k<<<grid_for(cnt), kBlock, 0, s>>>(N, cnt, visited, claim);
    UG_LAUNCH_CHECK();
  }
  return cnt;
}

// ------------------------------------------------------------- bfs_distances
void bfs_distances_run(TopoImpl* t, uint32_t source, int dir, int32_t* d_dist, cudaStream_t s) {
  const uint64_t n = t->n;
  if (n == 0) return;
  UG_CUDA(cudaMemsetAsync(d_dist, 0xFF, n * sizeof(int32_t), s));
  if ((uint64_t)source >= n) return;  // bfs.rs:21-23
  DirView fw = dir_view(t, dir, s);
  DirView rv = reverse_view(t, dir, s);
  FrontierBufs b;
  b.alloc(n, s);
  set_one_i32_k<<<1, 1, 0, s>>>(d_dist, source, 0);
  UG_LAUNCH_CHECK();
  set_one_u32_k<<<1, 1, 0, s>>>(b.F.get(), 0, source);
  UG_LAUNCH_CHECK();
  uint32_t f = 1;
  int32_t level = 0;
  bool bottom_up = false;
  const double total_edges = (double)t->m * (dir == 2 ? 2.0 : 1.0);
  double edges_left = total_edges;
  const double alpha = 14.0, beta = 24.0;
  // the frontier's out-edge total ("scout count"): the source's degree, then
  // summed on the device by each level's kernel as it appends the next
  // frontier, so a level costs one host read (frontier size and scout count)
  Scratch<unsigned long long> scout(1, s);
  uint64_t T = frontier_scan(fw, b.F.get(), f, b.pos.get(), s);
  while (f > 0) {
    UG_CUDA(cudaMemsetAsync(b.count.get(), 0, sizeof(uint32_t), s));
    UG_CUDA(cudaMemsetAsync(scout.get(), 0, sizeof(unsigned long long), s));
    if (!bottom_up) {
      if ((double)T > edges_left / alpha) {
        bottom_up = true;
      } else {
        if (T) {
          // edge-balanced expansion: the frontier's degree prefix (its total is T)
          fdeg_k<<<grid_for((uint64_t)f + 1), kBlock, 0, s>>>(fw, b.F.get(), f, b.pos.get());
          UG_LAUNCH_CHECK();
          exclusive_scan_u64(b.pos.get(), b.pos.get(), (uint64_t)f + 1, nullptr, s);
          td_k<<<grid_for(T, kBlock, 148u * 64u), kBlock, 0, s>>>(fw, b.F.get(), f, b.pos.get(), T,
                                                                   d_dist, level, b.N.get(),
                                                                   b.count.get(), scout.get());
          UG_LAUNCH_CHECK();
        }
        edges_left -= (double)T;
      }
    }
    if (bottom_up) {
      bu_k<<<grid_for(n, kBlock, 148u * 64u), kBlock, 0, s>>>(rv, fw, n, d_dist, level, b.N.get(),
                                                               b.count.get(), scout.get());
      UG_LAUNCH_CHECK();
    }
    uint32_t next = 0;
    unsigned long long t_next = 0;
    UG_CUDA(cudaMemcpyAsync(&next, b.count.get(), sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaMemcpyAsync(&t_next, scout.get(), sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
    if (bottom_up && (double)next < (double)n / beta && next < f) bottom_up = false;
    swap(b.F, b.N);
    f = next;
    T = t_next;
    level++;
  }
}

// ------------------------------------------------------------------- k_hop
void k_hop_run(TopoImpl* t, const uint32_t* seeds, uint64_t n_seeds, uint32_t k, int dir,
               PairsHost& out, cudaStream_t s) {
  const uint64_t n = t->n;
  if (k == 0 || n == 0) return;  // hop.rs:55-57
  DirView d = dir_view(t, dir, s);
  Scratch<uint8_t> visited(n, s);
  Scratch<unsigned long long> claim(n, s);
  UG_CUDA(cudaMemsetAsync(visited.get(), 0, n, s));
  UG_CUDA(cudaMemsetAsync(claim.get(), 0xFF, n * sizeof(unsigned long long), s));
  FrontierBufs b;
  b.alloc(n, s);
  Scratch<uint32_t> flag_buf;
  // reached nodes of the current seed, in emission order
  Scratch<uint32_t> reached(n ? n : 1, s);
  for (uint64_t si = 0; si < n_seeds; si++) {
    uint32_t seed = seeds[si];
    if ((uint64_t)seed >= n) continue;  // unknown seed (hop.rs:86-88)
    set_one_u8_k<<<1, 1, 0, s>>>(visited.get(), seed, 1);
    UG_LAUNCH_CHECK();
    set_one_u32_k<<<1, 1, 0, s>>>(b.F.get(), 0, seed);
    UG_LAUNCH_CHECK();
    uint32_t f = 1;
    uint64_t got = 0;
    for (uint32_t level = 0; level < k; level++) {
      uint32_t cnt = expand_exact(d, n, b.F.get(), f, b.N.get(), visited.get(), claim.get(),
                                  nullptr, b.pos.get(), flag_buf, s);
      if (cnt == 0) break;
      UG_CUDA(cudaMemcpyAsync(reached.get() + got, b.N.get(), (size_t)cnt * 4,
                              cudaMemcpyDeviceToDevice, s));
      got += cnt;
      swap(b.F, b.N);
      f = cnt;
    }
    size_t base = out.reached.size();
    out.reached.resize(base + got);
    out.seeds.resize(base + got, seed);
    if (got)
      UG_CUDA(cudaMemcpyAsync(out.reached.data() + base, reached.get(), got * 4,
                              cudaMemcpyDeviceToHost, s));
    // restore visited for the next seed (hop.rs:126-128)
    set_one_u8_k<<<1, 1, 0, s>>>(visited.get(), seed, 0);
    UG_LAUNCH_CHECK();
    if (got) {
      unmark_k<<<grid_for(got), kBlock, 0, s>>>(reached.get(), got, visited.get());
      UG_LAUNCH_CHECK();
    }
    UG_CUDA(cudaStreamSynchronize(s));
  }
}

// ----------------------------------------------------------- shortest_path
int64_t shortest_path_run(TopoImpl* t, uint32_t source, uint32_t target, int dir, uint32_t* path,
                          uint64_t cap, cudaStream_t s) {
  const uint64_t n = t->n;
  if ((uint64_t)source >= n || (uint64_t)target >= n) return -1;  // bfs.rs:55-57
  if (source == target) {                                          // bfs.rs:58-60
    UG_CHECK(cap >= 1, URSA_GPU_ETRUNC, "path buffer too small");
    path[0] = source;
    return 1;
  }
  DirView d = dir_view(t, dir, s);
  Scratch<uint8_t> visited(n, s);
  Scratch<unsigned long long> claim(n, s);
  Scratch<uint32_t> parent(n, s);
  UG_CUDA(cudaMemsetAsync(visited.get(), 0, n, s));
  UG_CUDA(cudaMemsetAsync(claim.get(), 0xFF, n * sizeof(unsigned long long), s));
  UG_CUDA(cudaMemsetAsync(parent.get(), 0xFF, n * sizeof(uint32_t), s));
  FrontierBufs b;
  b.alloc(n, s);
  Scratch<uint32_t> flag_buf;
  set_one_u8_k<<<1, 1, 0, s>>>(visited.get(), source, 1);
  UG_LAUNCH_CHECK();
  set_one_u32_k<<<1, 1, 0, s>>>(parent.get(), source, source);
  UG_LAUNCH_CHECK();
  set_one_u32_k<<<1, 1, 0, s>>>(b.F.get(), 0, source);
  UG_LAUNCH_CHECK();
  uint32_t f = 1;
  bool found = false;
  uint64_t levels = 0;
  while (f > 0) {
    uint32_t cnt = expand_exact(d, n, b.F.get(), f, b.N.get(), visited.get(), claim.get(),
                                parent.get(), b.pos.get(), flag_buf, s);
    levels++;
    if (read_u32(parent.get() + target, s) != 0xFFFFFFFFu) {
      found = true;
      break;
    }
    swap(b.F, b.N);
    f = cnt;
  }
  if (!found) return -1;
  uint64_t len_needed = levels + 1;
  Scratch<uint32_t> dpath(len_needed, s);
  Scratch<uint64_t> dlen(1, s);
  backtrack_k<<<1, 1, 0, s>>>(parent.get(), source, target, len_needed, dpath.get(), dlen.get());
  UG_LAUNCH_CHECK();
  uint64_t len = 0;
  UG_CUDA(cudaMemcpyAsync(&len, dlen.get(), sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  if (len > cap) return -(int64_t)len - 2;  // caller maps to ETRUNC
  UG_CUDA(cudaMemcpyAsync(path, dpath.get(), len * 4, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  return (int64_t)len;
}

}  // namespace ug

struct ursa_gpu_pairs {
  ug::PairsHost p;
};

using namespace ug;

extern "C" {

int ursa_gpu_bfs_distances(ursa_gpu_topo* t, uint32_t source, int dir, int32_t* out) {
  return guard([&] {
    UG_CHECK(t, URSA_GPU_EINVAL, "topology is NULL");
    UG_CHECK(dir >= 0 && dir <= 2, URSA_GPU_EINVAL, "direction must be 0, 1 or 2");
    TopoImpl* ti = &t->impl;
    if (ti->n == 0) return;
    UG_CHECK(out, URSA_GPU_EINVAL, "out is NULL");
    cudaStream_t s = thread_stream(ti->device);
    Scratch<int32_t> d(ti->n, s);
    bfs_distances_run(ti, source, dir, d.get(), s);
    UG_CUDA(cudaMemcpyAsync(out, d.get(), ti->n * 4, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_shortest_path(ursa_gpu_topo* t, uint32_t source, uint32_t target, int dir,
                           uint32_t* path, uint64_t cap, int64_t* len) {
  return guard([&] {
    UG_CHECK(t && len, URSA_GPU_EINVAL, "topology or len is NULL");
    UG_CHECK(dir >= 0 && dir <= 2, URSA_GPU_EINVAL, "direction must be 0, 1 or 2");
    *len = -1;
    TopoImpl* ti = &t->impl;
    cudaStream_t s = thread_stream(ti->device);
    int64_t r = shortest_path_run(ti, source, target, dir, path, cap, s);
    if (r < -1) {
      *len = -r - 2;
      throw Error(URSA_GPU_ETRUNC, "path buffer too small");
    }
    *len = r;
  });
}

int ursa_gpu_k_hop(ursa_gpu_topo* t, const uint32_t* seeds, uint64_t n_seeds, uint32_t k, int dir,
                   ursa_gpu_pairs** out) {
  return guard([&] {
    UG_CHECK(t && out, URSA_GPU_EINVAL, "topology or out is NULL");
    UG_CHECK(dir >= 0 && dir <= 2, URSA_GPU_EINVAL, "direction must be 0, 1 or 2");
    UG_CHECK(n_seeds == 0 || seeds, URSA_GPU_EINVAL, "seeds is NULL");
    *out = nullptr;
    auto* r = new ursa_gpu_pairs();
    try {
      TopoImpl* ti = &t->impl;
      cudaStream_t s = thread_stream(ti->device);
      k_hop_run(ti, seeds, n_seeds, k, dir, r->p, s);
    } catch (...) {
      delete r;
      throw;
    }
    *out = r;
  });
}

uint64_t ursa_gpu_pairs_len(const ursa_gpu_pairs* p) { return p ? p->p.seeds.size() : 0; }

int ursa_gpu_pairs_copy(const ursa_gpu_pairs* p, uint32_t* seeds_out, uint32_t* reached_out) {
  return guard([&] {
    UG_CHECK(p, URSA_GPU_EINVAL, "pairs is NULL");
    size_t n = p->p.seeds.size();
    if (seeds_out && n) std::copy(p->p.seeds.begin(), p->p.seeds.end(), seeds_out);
    if (reached_out && n) std::copy(p->p.reached.begin(), p->p.reached.end(), reached_out);
  });
}

void ursa_gpu_pairs_free(ursa_gpu_pairs* p) { delete p; }

}  // extern "C"
