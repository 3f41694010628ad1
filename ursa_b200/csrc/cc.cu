// cc.cu -- weak connected components (ursa-core/src/algo/components.rs:14-68).
//
// The reference runs a serial union-find (path halving, union by rank) over
// the out-edges and labels each node with its representative.  Here every
// out-edge slot is processed in parallel by the lock-free union-find of
// unionfind.cuh; each tree's root is the minimum id of its component, so the
// final labels are the minimum member ids: the reference's partition with a
// canonical representative.
#include "frontier.cuh"
#include "unionfind.cuh"

namespace ug {

namespace {

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
    if (u != v) uf_unite(parent, u, v);
  });
}

__global__ void flatten_k(uint32_t* parent, uint64_t n, uint32_t* __restrict__ out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    out[i] = uf_root(parent, (uint32_t)i);
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
