// pending.cu -- entry points whose device kernels are not in this build yet.
// Each returns URSA_GPU_EINVAL with a clear message (never a CPU fallback).
#include "common.cuh"

extern "C" {

static int pending(const char* what) {
  (void)what;
  return URSA_GPU_EINVAL;
}

int ursa_gpu_bfs_distances(ursa_gpu_topo*, uint32_t, int, int32_t*) { return pending("bfs"); }
int ursa_gpu_shortest_path(ursa_gpu_topo*, uint32_t, uint32_t, int, uint32_t*, uint64_t, int64_t*) {
  return pending("shortest_path");
}
int ursa_gpu_dijkstra_distances(ursa_gpu_topo*, const double*, uint64_t, uint32_t, int, double*) {
  return pending("dijkstra");
}
int ursa_gpu_shortest_path_weighted_with_cost(ursa_gpu_topo*, const double*, uint64_t, uint32_t,
                                              uint32_t, int, uint32_t*, double*, uint64_t,
                                              int64_t*) {
  return pending("sp_weighted");
}
int ursa_gpu_k_hop(ursa_gpu_topo*, const uint32_t*, uint64_t, uint32_t, int, ursa_gpu_pairs**) {
  return pending("k_hop");
}
uint64_t ursa_gpu_pairs_len(const ursa_gpu_pairs*) { return 0; }
int ursa_gpu_pairs_copy(const ursa_gpu_pairs*, uint32_t*, uint32_t*) { return pending("pairs"); }
void ursa_gpu_pairs_free(ursa_gpu_pairs*) {}
int ursa_gpu_connected_components_weak(ursa_gpu_topo*, uint32_t*) { return pending("cc"); }
int ursa_gpu_triangle_count(ursa_gpu_topo*, uint32_t*) { return pending("tc"); }
int ursa_gpu_clustering_coefficient(ursa_gpu_topo*, double*) { return pending("clustering"); }
int ursa_gpu_betweenness(ursa_gpu_topo*, int, double, int, uint64_t, double*) {
  return pending("betweenness");
}
int ursa_gpu_betweenness_weighted(ursa_gpu_topo*, const double*, uint64_t, int, double, int,
                                  uint64_t, double*) {
  return pending("betweenness_weighted");
}
}
