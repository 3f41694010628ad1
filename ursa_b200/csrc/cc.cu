// cc.cu -- weak connected components (ursa-core/src/algo/components.rs:14-68).
//
// The reference runs a serial union-find (path halving, union by rank) over
// the out-edges and labels each node with its representative.  Here every
// out-edge slot is processed in parallel by a lock-free union-find: a union
// always hooks the larger root under the smaller one with a compare-and-swap
// (a failed CAS means the root moved; the walk continues from the new
// parent), and finds compress paths by pointer jumping.  Parents only ever
// decrease, so each tree's root is the minimum id of its component, and the
// final labels are the minimum member ids: the reference's partition with a
// canonical representative.
#include "frontier.cuh"

namespace ug {

namespace {

__device__ __forceinline__ uint32_t ld_parent(const uint32_t* p, uint32_t x) {
  return *(const volatile uint32_t*)&p[x];
}

// Root of x with intermediate pointer jumping (parent[x] < x off the root).
__device__ __forceinline__ uint32_t find_root(uint32_t* p, uint32_t x) {
  uint32_t par = ld_parent(p, x);
  if (par != x) {
    uint32_t prev = x, next;
    while (par > (next = ld_parent(p, par))) {
      p[prev] = next;
      prev = par;
      par = next;
    }
  }
  return par;
}

__device__ __forceinline__ void unite(uint32_t* p, uint32_t a, uint32_t b) {
  uint32_t ra = find_root(p, a), rb = find_root(p, b);
  // bounded by the depth of the forest; each failed CAS moves one link up
  while (ra != rb) {
    if (ra < rb) {
      uint32_t old = atomicCAS(&p[rb], rb, ra);
      if (old == rb) return;
      rb = old;
    } else {
      uint32_t old = atomicCAS(&p[ra], ra, rb);
      if (old == ra) return;
      ra = old;
    }
  }
}

__global__ void iota_k(uint32_t* p, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = (uint32_t)i;
}

// One thread per out-edge slot; the owning node comes from a binary search
// over the offsets, restricted to the rows overlapping the block's slots.
__global__ void union_edges_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                              uint64_t n, uint64_t m, uint32_t* parent) {
  for_each_slot_owner(off, n, m, [&](uint64_t k, uint32_t u) {
    uint32_t v = tgt[k];
    if (u != v) unite(parent, u, v);
  });
}

__global__ void flatten_k(uint32_t* parent, uint64_t n, uint32_t* __restrict__ out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t x = (uint32_t)i, par = ld_parent(parent, x);
    while (par != x) {
      x = par;
      par = ld_parent(parent, x);
    }
    out[i] = par;
  }
}

}  // namespace

void cc_weak_run(TopoImpl* t, uint32_t* d_out, cudaStream_t s) {
  const uint64_t n = t->n, m = t->m;
  if (n == 0) return;
  Scratch<uint32_t> parent(n, s);
  iota_k<<<grid_for(n), kBlock, 0, s>>>(parent.get(), n);
  UG_LAUNCH_CHECK();
  if (m) {
    union_edges_k<<<grid_for(m, kBlock, 148u * 64u), kBlock, 0, s>>>(t->out.off.get(),
                                                                      t->out.tgt.get(), n, m,
                                                                      parent.get());
    UG_LAUNCH_CHECK();
  }
  flatten_k<<<grid_for(n), kBlock, 0, s>>>(parent.get(), n, d_out);
  UG_LAUNCH_CHECK();
}

// The same kernels with a caller-supplied parent array (n u32, overwritten):
// used by the allocation-free entry point.
void cc_weak_with_parent(TopoImpl* t, uint32_t* parent, uint32_t* d_out, cudaStream_t s) {
  const uint64_t n = t->n, m = t->m;
  if (n == 0) return;
  iota_k<<<grid_for(n), kBlock, 0, s>>>(parent, n);
  UG_LAUNCH_CHECK();
  if (m) {
    union_edges_k<<<grid_for(m, kBlock, 148u * 64u), kBlock, 0, s>>>(t->out.off.get(),
                                                                      t->out.tgt.get(), n, m,
                                                                      parent);
    UG_LAUNCH_CHECK();
  }
  flatten_k<<<grid_for(n), kBlock, 0, s>>>(parent, n, d_out);
  UG_LAUNCH_CHECK();
}

}  // namespace ug

using namespace ug;

extern "C" int ursa_gpu_connected_components_weak(ursa_gpu_topo* t, uint32_t* out) {
  return guard([&] {
    UG_CHECK(t, URSA_GPU_EINVAL, "topology is NULL");
    TopoImpl* ti = &t->impl;
    if (ti->n == 0) return;
    UG_CHECK(out, URSA_GPU_EINVAL, "out is NULL");
    cudaStream_t s = thread_stream(ti->device);
    Scratch<uint32_t> d(ti->n, s);
    cc_weak_run(ti, d.get(), s);
    UG_CUDA(cudaMemcpyAsync(out, d.get(), ti->n * 4, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}
