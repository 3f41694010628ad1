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

// Threads run independently (intersections vary widely in length), so the
// owner search here is a plain per-slot binary search.
__global__ void count_k(const uint32_t* __restrict__ o_off, const uint32_t* __restrict__ o_tgt,
                        uint64_t n, uint64_t mo, uint32_t* __restrict__ tri) {
  for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < mo;
       q += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t u = owner_of(o_off, n, q);
    uint32_t v = o_tgt[q];
    uint32_t i = o_off[u], ie = o_off[u + 1];
    uint32_t j = o_off[v], je = o_off[v + 1];
    uint32_t c = 0;
    if (i < ie && j < je) {
      uint32_t a = o_tgt[i], b = o_tgt[j];
      while (true) {
        if (a < b) {
          if (++i == ie) break;
          a = o_tgt[i];
        } else if (a > b) {
          if (++j == je) break;
          b = o_tgt[j];
        } else {
          c++;
          atomicAdd(&tri[a], 1u);
          if (++i == ie || ++j == je) break;
          a = o_tgt[i];
          b = o_tgt[j];
        }
      }
    }
    if (c) {
      atomicAdd(&tri[u], c);
      atomicAdd(&tri[v], c);
    }
  }
}

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
    count_k<<<grid_for(o.mo, kBlock, 148u * 64u), kBlock, 0, s>>>(o.off.get(), o.tgt.get(), n, o.mo,
                                                                   d_tri);
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
