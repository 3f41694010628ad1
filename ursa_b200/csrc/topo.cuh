// topo.cuh -- the device-resident topology behind the opaque ursa_gpu_topo.
//
// Mirrors ursa-core's Topology (ursa-core/src/topology.rs:251-261): the
// out-CSR is built eagerly, the transpose and the undirected CSR lazily on
// first use and then cached.  Device offsets are u32: ursa-core caps the edge
// count at u32::MAX (topology.rs:61-65), so every offset fits; the host mirror
// widens them to the reference's u64 on download.
#pragma once

#include <vector>

#include <memory>
#include <mutex>

#include "common.cuh"

namespace ug {

struct DevCsr {
  DevArray<uint32_t> off;  // n + 1
  DevArray<uint32_t> tgt;  // m
  DevArray<uint32_t> eid;  // m (original edge row per slot)
};

struct PrPlan;  // PageRank work partition over the in-CSR (pagerank.cu)
void pr_plan_free(PrPlan* p);
uint64_t pr_plan_bytes(const PrPlan* p);

struct TopoImpl {
  int device = 0;
  uint64_t n = 0, m = 0;
  DevCsr out, in;
  bool has_in = false;
  DevArray<uint32_t> und_off, und_tgt;
  uint64_t m_und = 0;
  bool has_und = false;
  DevArray<uint32_t> outdeg;  // out-degree per node (PageRank shares)
  bool has_outdeg = false;
  // Multi-source BFS, per direction (out, in, both): nodes whose pull scan
  // is split into chunks (hubs, ascending) and each chunk's hub index and
  // first slot of the pull CSR.
  struct MsHubs {
    DevArray<uint32_t> hubs, chunk_hub, chunk_lo;
    uint64_t n_hubs = 0, n_chunks = 0;
    bool built = false;
  } ms_hubs[3];
  PrPlan* pr_plan = nullptr;
  // a plan without edge ids, replaced by one with them for a weighted call;
  // kept until the topology goes (a call on another thread may still use it)
  PrPlan* pr_plan_retired = nullptr;
  std::mutex mu;
  ~TopoImpl() {
    if (pr_plan) pr_plan_free(pr_plan);
    if (pr_plan_retired) pr_plan_free(pr_plan_retired);
  }
};

// Stable counting-sort CSR build from device endpoint arrays (keys group,
// other is the paired endpoint); row order is kept inside each segment.
// bad (optional): set nonzero if a key is >= n (the sort reads every key once
// anyway; the result is then meant to be discarded).
void build_csr(uint64_t n, const uint32_t* d_keys, const uint32_t* d_other, uint64_t m,
               DevCsr& out, cudaStream_t s,
               cudaEvent_t other_ready = nullptr, unsigned* bad = nullptr);
// Lazily built parts; each call is a no-op once built.
void ensure_in(TopoImpl* t, cudaStream_t s);
void ensure_undirected(TopoImpl* t, cudaStream_t s);
void ensure_outdeg(TopoImpl* t, cudaStream_t s);

// Undirected CSR with every edge kept once, oriented from the lower to the
// higher (degree, id) rank (triangle counting).
struct OrientedCsr {
  DevArray<uint32_t> off, tgt;
  uint64_t mo = 0;
};
void orient_build(TopoImpl* t, OrientedCsr& o, cudaStream_t s);
void cc_weak_with_parent(TopoImpl* t, uint32_t* parent, uint32_t* d_out, cudaStream_t s);
TopoImpl* topo_from_device(uint64_t n, const uint32_t* d_src, const uint32_t* d_dst, uint64_t m,
                           cudaStream_t s, int device, ursa_gpu_topo** holder,
                           cudaEvent_t dst_ready = nullptr);

// Slot -> owning node for a CSR (binary search over offsets), n_slots = m.
void csr_owners(const uint32_t* off, uint64_t n, uint64_t m, uint32_t* owner, cudaStream_t s);

// Device-output forms of the kernels (each enqueued on s; results in device
// arrays of n entries unless stated).  d_weights: n_edges f64 by edge row.
void degree_run(TopoImpl* t, int dir, uint32_t* d_out, cudaStream_t s);
void pagerank_run(TopoImpl* t, const ursa_gpu_pagerank_params& p, const double* d_weights,
                  double* d_out, cudaStream_t s, ursa_gpu_pagerank_stats* stats);
void cc_weak_run(TopoImpl* t, uint32_t* d_out, cudaStream_t s);
void triangle_count_run(TopoImpl* t, uint32_t* d_tri, cudaStream_t s);
void clustering_run(TopoImpl* t, double* d_out, cudaStream_t s);
void betweenness_run(TopoImpl* t, const double* d_weights, bool has_sample, double sample,
                     bool has_seed, uint64_t seed, double* d_out, cudaStream_t s);
void closeness_device(TopoImpl* t, double* d_out, cudaStream_t s, float* device_ms);
void msbfs_distances(TopoImpl* t, int dir, const uint32_t* d_src, uint64_t n_sources, int32_t* d_dist,
                     cudaStream_t s);
void closeness_weighted_device(TopoImpl* t, const double* d_w, double* d_out, cudaStream_t s);

// k_hop pairs (seed, reached) in the reference's emission order, on the host.
struct PairsHost {
  std::vector<uint32_t> seeds, reached;
};
void k_hop_run(TopoImpl* t, const uint32_t* seeds, uint64_t n_seeds, uint32_t k, int dir,
               PairsHost& out, cudaStream_t s);
// Paths into host buffers of cap entries: length, -1 if unreachable, or
// -(length) - 2 if cap is too small.
int64_t shortest_path_run(TopoImpl* t, uint32_t source, uint32_t target, int dir, uint32_t* path,
                          uint64_t cap, cudaStream_t s);
int64_t weighted_path_run(TopoImpl* t, const double* d_weights, uint32_t source, uint32_t target,
                          int dir, uint32_t* path, double* costs, uint64_t cap, cudaStream_t s);

// The IdMap's device user ids (dense order) and their count; gathers
// d_out[i] = user id of d_dense[i] on the device (URSA_GPU_EINVAL if an index
// is out of range).
const int64_t* idmap_users(ursa_gpu_idmap* m, uint64_t* n_ids, int* device);
void idmap_gather_device(ursa_gpu_idmap* m, const uint32_t* d_dense, uint64_t n, int64_t* d_out,
                         cudaStream_t s);

}  // namespace ug

struct ursa_gpu_topo {
  ug::TopoImpl impl;
};
