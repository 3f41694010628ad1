// frontier.cuh -- directional neighbour views and load-balanced frontier
// expansion shared by the BFS, k-hop, shortest-path, SSSP and Brandes kernels.
#pragma once

#include "primitives.cuh"
#include "topo.cuh"

namespace ug {

// Topology::for_each_neighbor (topology.rs:395-404): Out, In, or the
// out-CSR followed by the in-CSR for Both.  Slot j of node u indexes that
// concatenation.
struct DirView {
  const uint32_t* off0;
  const uint32_t* tgt0;
  const uint32_t* eid0;
  const uint32_t* off1;  // nullptr unless Both
  const uint32_t* tgt1;
  const uint32_t* eid1;
};

DirView dir_view(TopoImpl* t, int dir, cudaStream_t s);
// The reverse view: the neighbours that reach u in direction `dir`
// (Out -> in-CSR, In -> out-CSR, Both -> both).
DirView reverse_view(TopoImpl* t, int dir, cudaStream_t s);

__device__ __forceinline__ uint32_t dv_deg(const DirView& d, uint32_t u) {
  uint32_t k = d.off0[u + 1] - d.off0[u];
  if (d.off1) k += d.off1[u + 1] - d.off1[u];
  return k;
}

// Neighbour of u at concatenated slot j; *slot_out = CSR slot, *second = in
// the second CSR.
__device__ __forceinline__ uint32_t dv_nbr(const DirView& d, uint32_t u, uint32_t j,
                                           uint32_t* slot_out = nullptr, bool* second = nullptr) {
  uint32_t b0 = d.off0[u], d0 = d.off0[u + 1] - b0;
  if (j < d0) {
    if (slot_out) *slot_out = b0 + j;
    if (second) *second = false;
    return d.tgt0[b0 + j];
  }
  uint32_t k = d.off1[u] + (j - d0);
  if (slot_out) *slot_out = k;
  if (second) *second = true;
  return d.tgt1[k];
}

// pos[i] = sum of dv_deg(F[k]) for k < i, pos[f] = total (u64). Returns total.
uint64_t frontier_scan(const DirView& d, const uint32_t* F, uint64_t f, uint64_t* pos,
                       cudaStream_t s);

// Frontier index owning expansion slot e: largest i with pos[i] <= e.
__device__ __forceinline__ uint64_t owner_in_pos(const uint64_t* __restrict__ pos, uint64_t f,
                                                 uint64_t e) {
  uint64_t lo = 0, hi = f;
  while (hi - lo > 1) {
    uint64_t mid = (lo + hi) >> 1;
    if (pos[mid] <= e)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// Device buffers reused across the levels of one traversal.
struct FrontierBufs {
  Scratch<uint32_t> F, N;   // current / next frontier (capacity n)
  Scratch<uint64_t> pos;    // n + 1
  Scratch<uint32_t> count;  // next-frontier size
  void alloc(uint64_t n, cudaStream_t s) {
    F.alloc(n ? n : 1, s);
    N.alloc(n ? n : 1, s);
    pos.alloc(n + 1, s);
    count.alloc(2, s);
  }
};

// Per-slot weights of a view, gathered once per call from row-indexed f64
// weights: w0[k] = weights[eid0[k]], w1 likewise.
struct DirWeights {
  Scratch<double> w0, w1;
};
void gather_dir_weights(TopoImpl* t, const DirView& d, const double* d_weights, DirWeights& out,
                        cudaStream_t s);

// Host-side copy of a device u32 counter.
uint32_t read_u32(const uint32_t* d, cudaStream_t s);

// Exact-order expansion (used by k_hop and shortest_path): the next frontier
// in the order the reference's serial loop discovers it -- frontier order,
// then neighbour order -- with parent[v] = its first discoverer when parent
// is given.  visited[] (u8) is updated; claim[] (u64, all ~0 on entry) is
// restored before return.  Returns the next frontier size (written to N).
uint32_t expand_exact(const DirView& d, uint64_t n, const uint32_t* F, uint32_t f, uint32_t* N,
                      uint8_t* visited, unsigned long long* claim, uint32_t* parent,
                      uint64_t* pos, Scratch<uint32_t>& flag_buf, cudaStream_t s);

}  // namespace ug
