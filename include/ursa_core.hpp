// ursa_core.hpp -- C++ host-side mirror of ursa-core's public API
// (cldixon/ursa, ursa-core/src/topology.rs and ursa-core/src/algo/mod.rs:35-50),
// implemented over the C ABI in ursa_gpu.h.  Header-only; link against
// libursa_gpu.so.
//
// Names, argument meaning and edge cases follow the Rust items: Topology
// (topology.rs:251-431) with build / out / incoming / undirected, and the
// kernel functions degree, pagerank, pagerank_weighted, bfs_distances,
// shortest_path, dijkstra_distances, shortest_path_weighted[_with_cost],
// k_hop, connected_components_weak, triangle_count, clustering_coefficient,
// betweenness, betweenness_weighted, closeness and closeness_weighted
// (algo/closeness.rs:69-224), plus ursa-plan's avg_path_length and diameter
// (ursa-plan/src/stats.rs:142-167) and, as an extension with no ursa-core
// counterpart, bfs_distances_multi.  Vec<T> becomes std::vector<T>,
// Option<T> becomes std::optional<T>.  Where the Rust code would panic (a
// contract violation, e.g. a weights length that is not the edge count), the
// mirror throws ursa_core::Error carrying the C ABI status and message.
#pragma once

#include <cstdint>
#include <memory>
#include <optional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "ursa_gpu.h"

namespace ursa_core {

struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(int status) {
  if (status != URSA_GPU_OK) throw Error(status, ursa_gpu_last_error());
}

// Direction (topology.rs:28-32).
enum class Direction : int { Out = 0, In = 1, Both = 2 };

// One direction's CSR (topology.rs:36-47).
struct Adjacency {
  std::vector<uint64_t> offsets;
  std::vector<uint32_t> targets;
  std::vector<uint32_t> edge_ids;
};

// The sorted, deduplicated undirected CSR (topology.rs:222-244).
struct UndirectedCsr {
  std::vector<uint64_t> offsets;
  std::vector<uint32_t> targets;
};

// PageRankParams (algo/pagerank.rs:22-36).
struct PageRankParams {
  double damping = 0.85;
  uint32_t max_iter = 30;
  double tol = 1e-6;
};

// The device-resident topology (Topology::build, topology.rs:276-298).
class Topology {
 public:
  static Topology build(uint64_t n_nodes, const std::vector<uint32_t>& src_dense,
                        const std::vector<uint32_t>& dst_dense) {
    if (src_dense.size() != dst_dense.size()) throw Error(URSA_GPU_EINVAL, "src/dst length mismatch");
    ursa_gpu_topo* t = nullptr;
    check(ursa_gpu_topo_build(n_nodes, src_dense.data(), dst_dense.data(), src_dense.size(), &t));
    return Topology(t);
  }
  uint64_t n_nodes() const { return ursa_gpu_topo_n_nodes(h_.get()); }
  uint64_t n_edges() const { return ursa_gpu_topo_n_edges(h_.get()); }
  Adjacency out() const { return adjacency(0); }
  Adjacency incoming() const { return adjacency(1); }
  UndirectedCsr undirected() const {
    uint64_t len = 0;
    check(ursa_gpu_topo_undirected_len(h_.get(), &len));
    UndirectedCsr u;
    u.offsets.resize(n_nodes() + 1);
    u.targets.resize(len);
    check(ursa_gpu_topo_undirected(h_.get(), u.offsets.data(), u.targets.data()));
    return u;
  }
  ursa_gpu_topo* handle() const { return h_.get(); }

 private:
  explicit Topology(ursa_gpu_topo* t) : h_(t, &ursa_gpu_topo_free) {}
  Adjacency adjacency(int dir) const {
    Adjacency a;
    a.offsets.resize(n_nodes() + 1);
    a.targets.resize(n_edges());
    a.edge_ids.resize(n_edges());
    check(ursa_gpu_topo_adjacency(h_.get(), dir, a.offsets.data(), a.targets.data(),
                                  a.edge_ids.data()));
    return a;
  }
  std::shared_ptr<ursa_gpu_topo> h_;
};

namespace algo {

inline std::vector<uint32_t> degree(const Topology& t, Direction dir) {
  std::vector<uint32_t> out(t.n_nodes());
  check(ursa_gpu_degree(t.handle(), (int)dir, out.data()));
  return out;
}

inline std::vector<double> pagerank(const Topology& t, PageRankParams p = {}) {
  std::vector<double> out(t.n_nodes());
  ursa_gpu_pagerank_params q{p.damping, p.max_iter, p.tol};
  check(ursa_gpu_pagerank(t.handle(), &q, out.data(), nullptr));
  return out;
}

inline std::vector<double> pagerank_weighted(const Topology& t, const std::vector<double>& weights,
                                             PageRankParams p = {}) {
  std::vector<double> out(t.n_nodes());
  ursa_gpu_pagerank_params q{p.damping, p.max_iter, p.tol};
  check(ursa_gpu_pagerank_weighted(t.handle(), weights.data(), weights.size(), &q, out.data(),
                                   nullptr));
  return out;
}

inline std::vector<int32_t> bfs_distances(const Topology& t, uint32_t source, Direction dir) {
  std::vector<int32_t> out(t.n_nodes());
  check(ursa_gpu_bfs_distances(t.handle(), source, (int)dir, out.data()));
  return out;
}

// Extension (no ursa-core counterpart): bfs_distances from many sources in
// one bit-parallel traversal; row i of the result is bfs_distances(sources[i]).
inline std::vector<std::vector<int32_t>> bfs_distances_multi(const Topology& t,
                                                             const std::vector<uint32_t>& sources,
                                                             Direction dir) {
  const uint64_t n = t.n_nodes();
  std::vector<int32_t> flat(sources.size() * n);
  if (!sources.empty() && n)
    check(ursa_gpu_bfs_distances_multi(t.handle(), sources.data(), sources.size(), (int)dir,
                                       flat.data()));
  std::vector<std::vector<int32_t>> out(sources.size());
  for (size_t i = 0; i < sources.size(); i++)
    out[i].assign(flat.begin() + i * n, flat.begin() + (i + 1) * n);
  return out;
}

inline std::optional<std::vector<uint32_t>> shortest_path(const Topology& t, uint32_t source,
                                                          uint32_t target, Direction dir) {
  std::vector<uint32_t> path(t.n_nodes() ? t.n_nodes() : 1);
  int64_t len = -1;
  check(ursa_gpu_shortest_path(t.handle(), source, target, (int)dir, path.data(), path.size(), &len));
  if (len < 0) return std::nullopt;
  path.resize((size_t)len);
  return path;
}

inline std::vector<double> dijkstra_distances(const Topology& t, const std::vector<double>& weights,
                                              uint32_t source, Direction dir) {
  std::vector<double> out(t.n_nodes());
  check(ursa_gpu_dijkstra_distances(t.handle(), weights.data(), weights.size(), source, (int)dir,
                                    out.data()));
  return out;
}

inline std::optional<std::pair<std::vector<uint32_t>, std::vector<double>>>
shortest_path_weighted_with_cost(const Topology& t, const std::vector<double>& weights,
                                 uint32_t source, uint32_t target, Direction dir) {
  size_t cap = t.n_nodes() ? t.n_nodes() : 1;
  std::vector<uint32_t> path(cap);
  std::vector<double> cost(cap);
  int64_t len = -1;
  check(ursa_gpu_shortest_path_weighted_with_cost(t.handle(), weights.data(), weights.size(),
                                                  source, target, (int)dir, path.data(),
                                                  cost.data(), cap, &len));
  if (len < 0) return std::nullopt;
  path.resize((size_t)len);
  cost.resize((size_t)len);
  return std::make_pair(std::move(path), std::move(cost));
}

inline std::optional<std::vector<uint32_t>> shortest_path_weighted(
    const Topology& t, const std::vector<double>& weights, uint32_t source, uint32_t target,
    Direction dir) {
  auto r = shortest_path_weighted_with_cost(t, weights, source, target, dir);
  if (!r) return std::nullopt;
  return std::move(r->first);
}

inline std::pair<std::vector<uint32_t>, std::vector<uint32_t>> k_hop(
    const Topology& t, const std::vector<uint32_t>& seeds, uint32_t k, Direction dir) {
  ursa_gpu_pairs* p = nullptr;
  check(ursa_gpu_k_hop(t.handle(), seeds.data(), seeds.size(), k, (int)dir, &p));
  std::unique_ptr<ursa_gpu_pairs, void (*)(ursa_gpu_pairs*)> guard(p, &ursa_gpu_pairs_free);
  uint64_t n = ursa_gpu_pairs_len(p);
  std::vector<uint32_t> a(n), b(n);
  if (n) check(ursa_gpu_pairs_copy(p, a.data(), b.data()));
  return {std::move(a), std::move(b)};
}

inline std::vector<uint32_t> connected_components_weak(const Topology& t) {
  std::vector<uint32_t> out(t.n_nodes());
  check(ursa_gpu_connected_components_weak(t.handle(), out.data()));
  return out;
}

inline std::vector<uint32_t> triangle_count(const Topology& t) {
  std::vector<uint32_t> out(t.n_nodes());
  check(ursa_gpu_triangle_count(t.handle(), out.data()));
  return out;
}

inline std::vector<double> clustering_coefficient(const Topology& t) {
  std::vector<double> out(t.n_nodes());
  check(ursa_gpu_clustering_coefficient(t.handle(), out.data()));
  return out;
}

inline std::vector<double> betweenness(const Topology& t, std::optional<double> sample,
                                       std::optional<uint64_t> seed) {
  std::vector<double> out(t.n_nodes());
  check(ursa_gpu_betweenness(t.handle(), sample.has_value(), sample.value_or(0.0),
                             seed.has_value(), seed.value_or(0), out.data()));
  return out;
}

inline std::vector<double> betweenness_weighted(const Topology& t, const std::vector<double>& weights,
                                                std::optional<double> sample,
                                                std::optional<uint64_t> seed) {
  std::vector<double> out(t.n_nodes());
  check(ursa_gpu_betweenness_weighted(t.handle(), weights.data(), weights.size(),
                                      sample.has_value(), sample.value_or(0.0), seed.has_value(),
                                      seed.value_or(0), out.data()));
  return out;
}

inline std::vector<double> closeness(const Topology& t) {
  std::vector<double> out(t.n_nodes());
  check(ursa_gpu_closeness(t.handle(), out.data()));
  return out;
}

inline std::vector<double> closeness_weighted(const Topology& t, const std::vector<double>& weights) {
  std::vector<double> out(t.n_nodes());
  check(ursa_gpu_closeness_weighted(t.handle(), weights.data(), weights.size(), out.data()));
  return out;
}

inline double avg_path_length(const Topology& t, std::optional<double> sample) {
  double v = 0.0;
  check(ursa_gpu_avg_path_length(t.handle(), sample.has_value(), sample.value_or(0.0), &v));
  return v;
}

inline int64_t diameter(const Topology& t, bool approximate) {
  int64_t d = 0;
  check(ursa_gpu_diameter(t.handle(), approximate ? 1 : 0, &d));
  return d;
}

}  // namespace algo
}  // namespace ursa_core
