// csr.cu -- CSR build, lazy transpose and undirected CSR on the device.
//
// Semantics follow ursa-core/src/topology.rs:
//  * build (Adjacency::build, :54-187): stable counting sort by key; within a
//    node's segment the slots keep original row order, so targets/edge_ids
//    are byte-identical to the reference.  Here: a stable LSD radix sort of
//    the row ids by key, gathering `other` in the last pass, then offsets by
//    lower_bound over the sorted keys.
//  * transpose (reconstruct_endpoints + incoming, :307-348): the out-CSR is
//    un-permuted back to row order and re-sorted by destination, which gives
//    the same in-segment row order as the reference.
//  * undirected (build_undirected, :360-389): every non-self-loop edge
//    contributes (u,v) and (v,u); pairs are sorted by (first, second) with
//    two stable radix sorts and adjacent duplicates are dropped.
#include "primitives.cuh"
#include "topo.cuh"

namespace ug {

namespace {

__global__ void owners_k(const uint32_t* __restrict__ off, uint64_t n, uint64_t m,
                         uint32_t* __restrict__ owner) {
  for_each_slot_owner(off, n, m, [&](uint64_t k, uint32_t u) { owner[k] = u; });
}

// reconstruct_endpoints (topology.rs:307-321) in one pass: slot k of node u
// goes back to its original row edge_ids[k].
__global__ void unpermute_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                            const uint32_t* __restrict__ eid, uint64_t n, uint64_t m,
                            uint32_t* __restrict__ src_by_row, uint32_t* __restrict__ dst_by_row) {
  for_each_slot_owner(off, n, m, [&](uint64_t k, uint32_t u) {
    uint32_t r = eid[k];
    src_by_row[r] = u;
    dst_by_row[r] = tgt[k];
  });
}

__global__ void und_pairs_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                            uint64_t n, uint64_t m, uint32_t* __restrict__ first,
                            uint32_t* __restrict__ second) {
  for_each_slot_owner(off, n, m, [&](uint64_t k, uint32_t u) {
    uint32_t v = tgt[k];
    bool self = u == v;
    first[2 * k] = self ? (uint32_t)n : u;
    second[2 * k] = v;
    first[2 * k + 1] = self ? (uint32_t)n : v;
    second[2 * k + 1] = u;
  });
}

__global__ void und_flags_k(const uint32_t* __restrict__ first, const uint32_t* __restrict__ second,
                            uint64_t len, uint64_t n, uint32_t* __restrict__ flag) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (uint64_t)gridDim.x * blockDim.x) {
    bool keep = first[i] < n && (i == 0 || first[i] != first[i - 1] || second[i] != second[i - 1]);
    flag[i] = keep ? 1u : 0u;
  }
}

__global__ void und_compact_k(const uint32_t* __restrict__ first, const uint32_t* __restrict__ second,
                              const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos,
                              uint64_t len, uint32_t* __restrict__ ufirst,
                              uint32_t* __restrict__ utgt) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (flag[i]) {
      ufirst[pos[i]] = first[i];
      utgt[pos[i]] = second[i];
    }
  }
}

__global__ void degree_k(const uint32_t* __restrict__ off, uint64_t n, uint32_t* __restrict__ deg) {
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x)
    deg[u] = off[u + 1] - off[u];
}

}  // namespace

void csr_owners(const uint32_t* off, uint64_t n, uint64_t m, uint32_t* owner, cudaStream_t s) {
  if (!m) return;
  owners_k<<<grid_for(m), kBlock, 0, s>>>(off, n, m, owner);
  UG_LAUNCH_CHECK();
}

void build_csr(uint64_t n, const uint32_t* d_keys, const uint32_t* d_other, uint64_t m,
               DevCsr& out, cudaStream_t s, cudaEvent_t other_ready, unsigned* bad) {
  out.off.alloc(n + 1, s);
  out.tgt.alloc(m, s);
  out.eid.alloc(m, s);
  if (m == 0) {
    UG_CUDA(cudaMemsetAsync(out.off.get(), 0, (n + 1) * sizeof(uint32_t), s));
    return;
  }
  Scratch<uint32_t> sorted_keys(m, s);
  radix_sort_pairs(d_keys, nullptr, m, bits_for(n ? n - 1 : 0), sorted_keys.get(), out.eid.get(),
                   d_other, out.tgt.get(), s, other_ready, bad, n);
  offsets_from_sorted(sorted_keys.get(), m, n, out.off.get(), s);
}

void ensure_in(TopoImpl* t, cudaStream_t s) {
  std::lock_guard<std::mutex> g(t->mu);
  if (t->has_in) return;
  uint64_t n = t->n, m = t->m;
  Scratch<uint32_t> src_by_row(m, s), dst_by_row(m, s);
  if (m) {
    unpermute_k<<<grid_for(m), kBlock, 0, s>>>(t->out.off.get(), t->out.tgt.get(),
                                                t->out.eid.get(), n, m, src_by_row.get(),
                                                dst_by_row.get());
    UG_LAUNCH_CHECK();
  }
  build_csr(n, dst_by_row.get(), src_by_row.get(), m, t->in, s);
  src_by_row.release();
  dst_by_row.release();
  UG_CUDA(cudaStreamSynchronize(s));
  t->has_in = true;
}

void ensure_undirected(TopoImpl* t, cudaStream_t s) {
  std::lock_guard<std::mutex> g(t->mu);
  if (t->has_und) return;
  uint64_t n = t->n, m = t->m;
  uint64_t len = 2 * m;
  UG_CHECK(len < (1ull << 32), URSA_GPU_EINVAL,
           "undirected CSR build: 2 * n_edges must be below 2^32");
  t->und_off.alloc(n + 1, s);
  if (m == 0) {
    UG_CUDA(cudaMemsetAsync(t->und_off.get(), 0, (n + 1) * sizeof(uint32_t), s));
    t->und_tgt.alloc(0, s);
    t->m_und = 0;
    UG_CUDA(cudaStreamSynchronize(s));
    t->has_und = true;
    return;
  }
  Scratch<uint32_t> first(len, s), second(len, s);
  und_pairs_k<<<grid_for(m), kBlock, 0, s>>>(t->out.off.get(), t->out.tgt.get(), n, m,
                                              first.get(), second.get());
  UG_LAUNCH_CHECK();
  Scratch<uint32_t> k1(len, s), v1(len, s);
  // by second (stable), then by first (stable) => lexicographic (first, second)
  radix_sort_pairs(second.get(), first.get(), len, bits_for(n ? n - 1 : 0), k1.get(), v1.get(),
                   nullptr, nullptr, s);
  radix_sort_pairs(v1.get(), k1.get(), len, bits_for(n), first.get(), second.get(), nullptr,
                   nullptr, s);
  k1.release();
  v1.release();
  Scratch<uint32_t> flag(len, s), pos(len, s), total(1, s);
  und_flags_k<<<grid_for(len), kBlock, 0, s>>>(first.get(), second.get(), len, n, flag.get());
  UG_LAUNCH_CHECK();
  exclusive_scan_u32(flag.get(), pos.get(), len, total.get(), s);
  uint32_t m_und = 0;
  UG_CUDA(cudaMemcpyAsync(&m_und, total.get(), sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  t->und_tgt.alloc(m_und, s);
  Scratch<uint32_t> ufirst(m_und, s);
  if (m_und) {
    und_compact_k<<<grid_for(len), kBlock, 0, s>>>(first.get(), second.get(), flag.get(),
                                                    pos.get(), len, ufirst.get(),
                                                    t->und_tgt.get());
    UG_LAUNCH_CHECK();
  }
  offsets_from_sorted(ufirst.get(), m_und, n, t->und_off.get(), s);
  UG_CUDA(cudaStreamSynchronize(s));
  t->m_und = m_und;
  t->has_und = true;
}

void ensure_outdeg(TopoImpl* t, cudaStream_t s) {
  std::lock_guard<std::mutex> g(t->mu);
  if (t->has_outdeg) return;
  t->outdeg.alloc(t->n, s);
  if (t->n) {
    degree_k<<<grid_for(t->n), kBlock, 0, s>>>(t->out.off.get(), t->n, t->outdeg.get());
    UG_LAUNCH_CHECK();
  }
  UG_CUDA(cudaStreamSynchronize(s));
  t->has_outdeg = true;
}

}  // namespace ug
