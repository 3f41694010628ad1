// C++ host-mirror smoke test: ursa-core's own unit-test goldens through
// include/ursa_core.hpp (which calls the C ABI).  Prints "ok" and exits 0 on
// success; any mismatch prints the failing check and exits 1.
#include <cmath>
#include <cstdio>
#include <vector>

#include "ursa_core.hpp"

using namespace ursa_core;
using D = Direction;

static int failures = 0;
#define EXPECT(cond)                                              \
  do {                                                            \
    if (!(cond)) {                                                \
      std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond); \
      failures++;                                                 \
    }                                                             \
  } while (0)

template <class T>
static bool eq(const std::vector<T>& a, std::initializer_list<T> b) {
  return a == std::vector<T>(b);
}

int main() {
  // topology.rs:471-489 (diamond 0->1, 0->2, 1->2, 2->0)
  Topology t = Topology::build(3, {0, 0, 1, 2}, {1, 2, 2, 0});
  Adjacency out = t.out();
  EXPECT(out.offsets == (std::vector<uint64_t>{0, 2, 3, 4}));
  EXPECT(eq(out.targets, {1u, 2u, 2u, 0u}));
  Adjacency in = t.incoming();
  EXPECT(eq(in.targets, {2u, 0u, 0u, 1u}));
  // degree.rs:92-99
  EXPECT(eq(algo::degree(t, D::Out), {2u, 1u, 1u}));
  EXPECT(eq(algo::degree(t, D::In), {1u, 1u, 2u}));
  EXPECT(eq(algo::degree(t, D::Both), {3u, 2u, 3u}));
  // pagerank.rs:275-285
  Topology hub = Topology::build(4, {0, 1, 3, 2}, {2, 2, 2, 0});
  auto pr = algo::pagerank(hub);
  double sum = pr[0] + pr[1] + pr[2] + pr[3];
  EXPECT(std::fabs(sum - 1.0) < 1e-6);
  EXPECT(pr[2] > pr[0] && pr[2] > pr[1] && pr[2] > pr[3]);
  // bfs.rs:270-332 (path 0->1->2->3, 1->4)
  Topology p = Topology::build(5, {0, 1, 2, 1}, {1, 2, 3, 4});
  EXPECT(eq(algo::bfs_distances(p, 0, D::Out), {0, 1, 2, 3, 2}));
  EXPECT(algo::shortest_path(p, 0, 3, D::Out) == std::optional<std::vector<uint32_t>>({0, 1, 2, 3}));
  EXPECT(!algo::shortest_path(p, 3, 0, D::Out).has_value());
  EXPECT(algo::shortest_path(p, 3, 0, D::In) == std::optional<std::vector<uint32_t>>({3, 2, 1, 0}));
  auto multi = algo::bfs_distances_multi(p, {0, 2, 9}, D::Out);  // 9: unknown source, all -1
  EXPECT(multi.size() == 3 && multi[0] == algo::bfs_distances(p, 0, D::Out) &&
         eq(multi[1], {-1, -1, 0, 1, -1}) && eq(multi[2], {-1, -1, -1, -1, -1}));
  // bfs.rs:366-387
  Topology w = Topology::build(4, {0, 1, 0}, {1, 3, 3});
  auto wc = algo::shortest_path_weighted_with_cost(w, {1.0, 1.0, 5.0}, 0, 3, D::Out);
  EXPECT(wc.has_value() && wc->first == std::vector<uint32_t>({0, 1, 3}) &&
         wc->second == std::vector<double>({0.0, 1.0, 2.0}));
  // hop.rs:543-548
  auto kh = algo::k_hop(p, {0}, 2, D::Out);
  EXPECT(kh.first.size() == 3 && kh.second.size() == 3);
  // components.rs:144-153 (minimum-member labels)
  EXPECT(eq(algo::connected_components_weak(Topology::build(5, {0, 1, 3}, {1, 2, 4})),
            {0u, 0u, 0u, 3u, 3u}));
  // triangle.rs:265-272, clustering.rs:351-357
  EXPECT(eq(algo::triangle_count(Topology::build(4, {0, 0, 0, 1, 1, 2}, {1, 2, 3, 2, 3, 3})),
            {3u, 3u, 3u, 3u}));
  auto cc = algo::clustering_coefficient(Topology::build(4, {0, 0, 0, 1}, {1, 2, 3, 2}));
  EXPECT(std::fabs(cc[0] - 1.0 / 3.0) < 1e-12);
  // betweenness.rs:368-375
  auto bc = algo::betweenness(Topology::build(5, {0, 1, 2, 3}, {1, 2, 3, 4}), std::nullopt,
                              std::nullopt);
  EXPECT(bc == std::vector<double>({0.0, 3.0, 4.0, 3.0, 0.0}));
  // closeness.rs:244-252 (directed line), stats.rs (directed triangle)
  EXPECT(algo::closeness(Topology::build(4, {0, 1, 2}, {1, 2, 3})) ==
         std::vector<double>({0.5, 2.0 / 3.0, 1.0, 0.0}));
  auto cw = algo::closeness_weighted(Topology::build(3, {0, 1, 0}, {1, 2, 2}), {1.0, 1.0, 5.0});
  EXPECT(std::fabs(cw[0] - 2.0 / 3.0) < 1e-12 && std::fabs(cw[1] - 1.0) < 1e-12);
  Topology tri = Topology::build(3, {0, 1, 2}, {1, 2, 0});
  EXPECT(algo::avg_path_length(tri, std::nullopt) == 1.5);
  EXPECT(algo::diameter(tri, false) == 2);
  // contract violation -> Error (the Rust code asserts)
  bool threw = false;
  try {
    algo::pagerank_weighted(w, {1.0}, PageRankParams{});
  } catch (const Error& e) {
    threw = e.status == URSA_GPU_EINVAL;
  }
  EXPECT(threw);
  if (failures) return 1;
  std::printf("ok\n");
  return 0;
}
