/*
 * ursa_oracle.h -- CPU restatement of ursa-core's CSR topology and algorithm
 * kernels (cldixon/ursa, ursa-core/src).  TEST INFRASTRUCTURE ONLY: this is
 * the checker that the CUDA path is compared against, and the timed CPU
 * baseline.  Nothing in the product library links or calls it.
 *
 * Every function restates the reference's operation order exactly (same
 * sequential sums, same fixed-size reduction chunks, same traversal orders),
 * so results are bit-identical to ursa-core at any thread count.  Each
 * definition in ursa_oracle.c cites the reference file:line it follows.
 *
 * Conventions: node ids are uint32, CSR offsets uint64 (as in
 * ursa-core/src/topology.rs:36-47).  Direction: 0 = Out, 1 = In, 2 = Both
 * (topology.rs:28-32).  Weights are f64 indexed by original edge row.
 */
#ifndef URSA_ORACLE_H
#define URSA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_topo orc_topo;

/* Worker threads used by the parallel sweeps (results do not depend on it). */
/* IdMap::from_edge_batches, Int64 ids (id_map.rs:220-320): dense ids in
 * first-seen order over src[0], dst[0], src[1], dst[1], ...; to_user holds up
 * to 2 * n_edges ids; returns the number of distinct ids. */
uint64_t orc_idmap_build(const int64_t *src, const int64_t *dst, uint64_t n_edges,
                         uint32_t *dense_src, uint32_t *dense_dst, int64_t *to_user);
/* closeness / closeness_weighted (algo/closeness.rs:69-224) and
 * avg_path_length / diameter (ursa-plan/src/stats.rs:82-167). */
void orc_closeness(orc_topo *t, double *out);
void orc_closeness_sources(orc_topo *t, const uint32_t *sources, uint64_t k, double *out);
void orc_closeness_weighted(orc_topo *t, const double *weights, double *out);
double orc_avg_path_length(orc_topo *t, int has_sample, double sample);
int64_t orc_diameter(orc_topo *t, int approximate);
void orc_set_threads(int threads);
int orc_get_threads(void);

/* Topology::build (topology.rs:276-298). src/dst are copied. NULL on bad input. */
orc_topo *orc_topo_build(uint64_t n_nodes, const uint32_t *src,
                         const uint32_t *dst, uint64_t m);
void orc_topo_free(orc_topo *t);
uint64_t orc_topo_n_nodes(const orc_topo *t);
uint64_t orc_topo_n_edges(const orc_topo *t);

/* Copy a direction's CSR out (dir 0 = out-CSR, 1 = in-CSR, built lazily).
 * offsets: n+1, targets/edge_ids: m. Any pointer may be NULL. */
void orc_topo_csr(orc_topo *t, int dir, uint64_t *offsets, uint32_t *targets,
                  uint32_t *edge_ids);
/* Undirected sorted/deduped CSR (topology.rs:360-389). */
uint64_t orc_topo_undirected_len(orc_topo *t);
void orc_topo_undirected(orc_topo *t, uint64_t *offsets, uint32_t *targets);

/* Kernels (ursa-core/src/algo). */
void orc_degree(orc_topo *t, int dir, uint32_t *out);
/* Returns the number of iterations run. */
uint32_t orc_pagerank(orc_topo *t, double damping, uint32_t max_iter,
                      double tol, double *out);
uint32_t orc_pagerank_weighted(orc_topo *t, const double *weights,
                               double damping, uint32_t max_iter, double tol,
                               double *out);
/* The L1 residual of each iteration of this thread's last pagerank call
 * (up to cap of them); returns how many iterations ran. */
uint32_t orc_pagerank_deltas(double *out, uint32_t cap);
void orc_bfs_distances(orc_topo *t, uint32_t source, int dir, int32_t *out);
/* Path into path_out (capacity n); returns its length, or -1 for None. */
int64_t orc_shortest_path(orc_topo *t, uint32_t source, uint32_t target,
                          int dir, uint32_t *path_out);
void orc_dijkstra_distances(orc_topo *t, const double *weights,
                            uint32_t source, int dir, double *out);
int64_t orc_shortest_path_weighted_with_cost(orc_topo *t, const double *weights,
                                             uint32_t source, uint32_t target,
                                             int dir, uint32_t *path_out,
                                             double *cost_out);
/* k_hop: returns the pair count; the two output arrays are malloc(3)ed and
 * released with orc_free. */
uint64_t orc_k_hop(orc_topo *t, const uint32_t *seeds, uint64_t n_seeds,
                   uint32_t k, int dir, uint32_t **src_out, uint32_t **dst_out);
void orc_free(void *p);
void orc_connected_components_weak(orc_topo *t, uint32_t *out);
void orc_triangle_count(orc_topo *t, uint32_t *out);
/* triangle_count's per-node value for nodes[0..k) only (each node < n). */
void orc_triangle_count_nodes(orc_topo *t, const uint32_t *nodes, uint64_t k, uint32_t *out);
void orc_clustering_coefficient(orc_topo *t, double *out);
void orc_betweenness(orc_topo *t, int has_sample, double sample, int has_seed,
                     uint64_t seed, double *out);
void orc_betweenness_weighted(orc_topo *t, const double *weights,
                              int has_sample, double sample, int has_seed,
                              uint64_t seed, double *out);
/* Betweenness over an explicit source list (same chunked accumulation, no
 * n/k scaling); used to time bounded samples of the sampled workload. */
void orc_betweenness_sources(orc_topo *t, const double *weights,
                             const uint32_t *sources, uint64_t k, double *out);

/* rng.rs */
void orc_shuffled_order(uint64_t n, uint64_t seed, uint32_t *out);
uint64_t orc_sample_indices(uint64_t r, uint64_t k, int has_seed,
                            uint64_t seed, uint64_t *out);
/* betweenness.rs:349-362; returns k, writes k sources. */
uint64_t orc_sample_sources(uint64_t n, int has_sample, double frac,
                            int has_seed, uint64_t seed, uint32_t *out);

#ifdef __cplusplus
}
#endif
#endif
