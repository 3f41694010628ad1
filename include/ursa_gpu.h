/*
 * ursa_gpu.h -- C ABI of the B200 (sm_100a) implementation of ursa-core's CSR
 * topology and graph kernels (cldixon/ursa, ursa-core/src).
 *
 * Each entry point replaces one public function of ursa-core; the comment on
 * each names the Rust item (file:line, paths relative to the ursa project
 * root) whose meaning, argument order and edge-case behaviour it keeps.  A
 * Rust FFI crate binds these declarations one-to-one; the kernel functions'
 * Rust bodies call them and keep their signatures, so GraphAlgorithmExec
 * (ursa-plan/src/physical.rs:40) and the PyO3 layer see no change.
 *
 * Conventions
 *  - Node ids are uint32; host-visible CSR offsets are uint64, as in
 *    Adjacency (ursa-core/src/topology.rs:36-47).
 *  - direction: 0 = Out, 1 = In, 2 = Both (topology.rs:28-32).
 *  - Weights are f64 indexed by ORIGINAL edge row, length == n_edges
 *    (pagerank.rs:140-144); they must be non-negative (validated upstream by
 *    ursa-plan/src/weight.rs:51-106).
 *  - Every function returns URSA_GPU_OK (0) or an error status; the message
 *    of the last error on the calling thread is ursa_gpu_last_error().  The
 *    Rust shim maps a non-OK status to panic!, which the plan layer already
 *    turns into a DataFusionError (physical.rs:106-108).
 *  - Host buffers are caller-allocated.  All calls are re-entrant: each host
 *    thread gets its own CUDA stream, and a topology's lazily built parts
 *    (transpose, undirected CSR) are created once under a mutex, like the
 *    OnceLock fields of Topology (topology.rs:258-260).
 */
#ifndef URSA_GPU_H
#define URSA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  URSA_GPU_OK = 0,
  URSA_GPU_EINVAL = 1,   /* contract violation (the Rust code would assert!) */
  URSA_GPU_ENOMEM = 2,   /* device memory / admission budget exhausted */
  URSA_GPU_ECUDA = 3,    /* CUDA runtime error */
  URSA_GPU_ETIMEOUT = 4, /* a bounded device-side wait expired */
  URSA_GPU_ETRUNC = 5,   /* caller buffer too small; required size reported */
  URSA_GPU_ENODEV = 6,   /* no usable CUDA device */
  URSA_GPU_ECANCELED = 7 /* a served query was cancelled */
};

typedef struct ursa_gpu_topo ursa_gpu_topo;
typedef struct ursa_gpu_pairs ursa_gpu_pairs;

/* Message for the last non-OK status returned on this thread. */
const char *ursa_gpu_last_error(void);
/* Library ABI version (major * 10000 + minor * 100 + patch). */
int ursa_gpu_version(void);
/* Diagnostics, not part of ursa-core's surface: the number of kernels this
 * library has launched in the process so far (benchmarks difference it
 * around a timed region). */
uint64_t ursa_gpu_launch_count(void);
/* Selects the CUDA device used by topologies built afterwards on this thread. */
int ursa_gpu_set_device(int device);
/* The CUDA stream (a cudaStream_t) on which this host thread's calls on
 * `device` enqueue their work: events recorded on it around a call give the
 * call's device time. */
int ursa_gpu_thread_stream(int device, void **stream);
/* Device memory: the library takes its device buffers (topologies, per-call
 * scratch) from the device's stream-ordered memory pool and keeps every
 * freed block cached -- blocks of 4 MB and more at their own addresses, to
 * be handed out again to requests that fit, smaller ones in that pool -- so
 * repeated builds and calls neither map memory from the driver again nor pay
 * the pool's cost of placing a large block.  These report and return that
 * cache (an extension with no counterpart in the reference): *cached = bytes
 * kept that no buffer uses; release returns all of them to the driver
 * (other processes and allocators can then use the memory). */
int ursa_gpu_pool_cached_bytes(int device, uint64_t *cached);
int ursa_gpu_pool_release(int device);

/* ---- Topology (ursa-core/src/topology.rs) ------------------------------ */

/* Topology::build(n_nodes, src_dense, dst_dense) -- topology.rs:276-298.
 * Host arrays of n_edges endpoints, each < n_nodes.  Copies to the device and
 * builds the out-CSR by a stable counting sort (row order kept within each
 * node's segment: byte-identical to Adjacency::build, topology.rs:54-187).
 * n_edges > UINT32_MAX is rejected (topology.rs:61-65). */
int ursa_gpu_topo_build(uint64_t n_nodes, const uint32_t *src, const uint32_t *dst,
                        uint64_t n_edges, ursa_gpu_topo **out);
/* Same as ursa_gpu_topo_build with device-resident endpoint arrays, enqueued
 * on `stream` (a cudaStream_t, or NULL for this thread's stream).  Used by the
 * serving layer, whose uploads already live in HBM. */
int ursa_gpu_topo_build_device(uint64_t n_nodes, const uint32_t *d_src, const uint32_t *d_dst,
                               uint64_t n_edges, void *stream, ursa_gpu_topo **out);
/* Drop for Topology: frees every device buffer. NULL is a no-op. */
void ursa_gpu_topo_free(ursa_gpu_topo *t);
/* Topology::n_nodes / n_edges -- topology.rs:324-331. */
uint64_t ursa_gpu_topo_n_nodes(const ursa_gpu_topo *t);
uint64_t ursa_gpu_topo_n_edges(const ursa_gpu_topo *t);
/* Topology::out() / incoming() -- topology.rs:335-348.  dir 0 = out-CSR,
 * 1 = in-CSR (the transpose, built on first use from the out-CSR by
 * reconstructing original row order, topology.rs:307-321).  Copies the pub
 * fields offsets[n+1], targets[m], edge_ids[m] to host; NULL skips a field. */
int ursa_gpu_topo_adjacency(ursa_gpu_topo *t, int dir, uint64_t *offsets, uint32_t *targets,
                            uint32_t *edge_ids);
/* Topology::undirected() -- topology.rs:353-389: out ∪ in per node, self-loops
 * dropped, sorted, deduplicated.  *len receives targets.len(). */
int ursa_gpu_topo_undirected_len(ursa_gpu_topo *t, uint64_t *len);
int ursa_gpu_topo_undirected(ursa_gpu_topo *t, uint64_t *offsets, uint32_t *targets);
/* Builds the lazily cached parts now (1 = transpose, 2 = undirected CSR,
 * 3 = both).  Lets a caller move build cost out of a latency-critical call. */
int ursa_gpu_topo_prepare(ursa_gpu_topo *t, int what);
/* Device bytes held by the topology (CSRs plus cached plans). */
uint64_t ursa_gpu_topo_device_bytes(const ursa_gpu_topo *t);

/* ---- Kernels (ursa-core/src/algo, re-exported at algo/mod.rs:35-50) ---- */

/* degree(&Topology, Direction) -> Vec<u32> -- algo/degree.rs:12-30. */
int ursa_gpu_degree(ursa_gpu_topo *t, int dir, uint32_t *out);

/* PageRankParams -- algo/pagerank.rs:22-36 (defaults 0.85 / 30 / 1e-6). */
typedef struct {
  double damping;
  uint32_t max_iter;
  double tol;
} ursa_gpu_pagerank_params;

/* Optional run statistics (not part of the Rust signature). */
typedef struct {
  uint32_t iterations;   /* power iterations executed */
  double last_delta;     /* L1 residual of the last iteration */
  double device_ms;      /* device time of the iteration kernel */
} ursa_gpu_pagerank_stats;

/* pagerank(&Topology, PageRankParams) -> Vec<f64> -- algo/pagerank.rs:98-124.
 * Pull iteration over the in-CSR; the per-edge shares rank[v]/outdeg[v] are
 * gathered in f32 and summed per row with compensated (TwoSum) f32
 * accumulation; base term, dangling mass, L1 residual and the ranks stay
 * f64.  No final renormalisation (as in power_iterate, pagerank.rs:63-94).
 * out: n f64 (host).  stats may be NULL. */
int ursa_gpu_pagerank(ursa_gpu_topo *t, const ursa_gpu_pagerank_params *params, double *out,
                      ursa_gpu_pagerank_stats *stats);
/* Device-output form of ursa_gpu_pagerank: d_out is an n-f64 device array,
 * enqueued on `stream` (NULL = this thread's stream); returns after the
 * kernel completes. */
int ursa_gpu_pagerank_device(ursa_gpu_topo *t, const ursa_gpu_pagerank_params *params,
                             double *d_out, void *stream, ursa_gpu_pagerank_stats *stats);
/* pagerank_weighted(&Topology, &[f64], PageRankParams) -> Vec<f64> --
 * algo/pagerank.rs:135-169.  weights: n_edges f64 by original edge row. */
int ursa_gpu_pagerank_weighted(ursa_gpu_topo *t, const double *weights, uint64_t n_weights,
                               const ursa_gpu_pagerank_params *params, double *out,
                               ursa_gpu_pagerank_stats *stats);

/* bfs_distances(&Topology, u32, Direction) -> Vec<i32> -- algo/bfs.rs:18-42.
 * -1 = unreachable; out-of-range source gives all -1.  Direction-optimising
 * (top-down / bottom-up) on the device; levels are exact. */
int ursa_gpu_bfs_distances(ursa_gpu_topo *t, uint32_t source, int dir, int32_t *out);
/* Extension for analytics callers: bfs_distances from each of n_sources
 * sources at once, one bit-parallel traversal per 64 (or 256) of them;
 * out: n_sources rows of n i32, row i = bfs_distances(sources[i], dir).
 * Pays off with many sources; a single source is faster through
 * ursa_gpu_bfs_distances (its frontier queues skip the untouched nodes). */
int ursa_gpu_bfs_distances_multi(ursa_gpu_topo *t, const uint32_t *sources, uint64_t n_sources, int dir,
                                 int32_t *out);

/* shortest_path(&Topology, u32, u32, Direction) -> Option<Vec<u32>> --
 * algo/bfs.rs:48-102.  Writes the inclusive node path into path[0..cap) and
 * its length into *len (-1 = None).  The parent of each node is its first
 * discoverer in the reference's serial frontier order, so the path is the
 * reference's path.  If the path is longer than cap: URSA_GPU_ETRUNC with
 * *len set. */
int ursa_gpu_shortest_path(ursa_gpu_topo *t, uint32_t source, uint32_t target, int dir,
                           uint32_t *path, uint64_t cap, int64_t *len);

/* shortest_path over out-edges by the serving loop's algorithm, one query
 * per launch: a bidirectional BFS in one CTA (forward on the out-CSR,
 * backward on the in-CSR, the side with fewer frontier edges first; parents
 * are the smallest-id discoverer on each level; the shortest meeting wins,
 * ties to the smallest meeting id).  An extension with no counterpart in the
 * reference: the path has the reference's hop count and is the path a
 * server's shortest_path query returns, so it measures what batching adds to
 * the same algorithm.  Paths longer than 4,096 nodes or cap: URSA_GPU_ETRUNC. */
int ursa_gpu_shortest_path_bidirectional(ursa_gpu_topo *t, uint32_t source, uint32_t target,
                                         uint32_t *path, uint64_t cap, int64_t *len);

/* dijkstra_distances(&Topology, &[f64], u32, Direction) -> Vec<f64> --
 * algo/bfs.rs:126-166.  +inf = unreachable.  Distances are the same f64
 * values Dijkstra settles (min over paths of the left-to-right f64 sums). */
int ursa_gpu_dijkstra_distances(ursa_gpu_topo *t, const double *weights, uint64_t n_weights,
                                uint32_t source, int dir, double *out);

/* shortest_path_weighted_with_cost(...) -> Option<(Vec<u32>, Vec<f64>)> --
 * algo/bfs.rs:192-259; shortest_path_weighted (bfs.rs:176-184) is this with
 * costs == NULL.  path/costs have room for cap entries; *len = -1 for None. */
int ursa_gpu_shortest_path_weighted_with_cost(ursa_gpu_topo *t, const double *weights,
                                              uint64_t n_weights, uint32_t source,
                                              uint32_t target, int dir, uint32_t *path,
                                              double *costs, uint64_t cap, int64_t *len);

/* k_hop(&Topology, &[u32], u32, Direction) -> (Vec<u32>, Vec<u32>) --
 * algo/hop.rs:52-75.  Pairs are emitted per seed in seed order and, within a
 * seed, in the reference's discovery order.  The result object owns the
 * pairs: read them with ursa_gpu_pairs_len / _copy and release it with
 * ursa_gpu_pairs_free. */
int ursa_gpu_k_hop(ursa_gpu_topo *t, const uint32_t *seeds, uint64_t n_seeds, uint32_t k,
                   int dir, ursa_gpu_pairs **out);
uint64_t ursa_gpu_pairs_len(const ursa_gpu_pairs *p);
int ursa_gpu_pairs_copy(const ursa_gpu_pairs *p, uint32_t *seeds_out, uint32_t *reached_out);
void ursa_gpu_pairs_free(ursa_gpu_pairs *p);

/* connected_components_weak(&Topology) -> Vec<u32> -- algo/components.rs:58-68.
 * Labels are the minimum member id of each weak component (a valid
 * "representative id" labelling; the reference's union-find picks another
 * representative, and the partition is identical). */
int ursa_gpu_connected_components_weak(ursa_gpu_topo *t, uint32_t *out);

/* Allocation-free form of ursa_gpu_connected_components_weak.  It has no
 * counterpart in the reference; it exists for callers that must not have the
 * library allocate device memory while they run a query -- a serving loop
 * whose free HBM is already promised to resident graphs, or a host runtime
 * that owns all device memory through its own pool.  The call allocates
 * nothing: the labels go to the caller's device array d_labels (n u32, same
 * minimum-member labels as the allocating form) and the union-find scratch
 * is a fixed array inside the library, 16 MiB per GPU.
 *  - Graphs above 4,194,304 nodes are rejected with URSA_GPU_EINVAL.
 *  - The first call on a device looks up that array's device address.  With
 *    CUDA's default lazy module loading that first call is also when the
 *    16 MiB array comes into being on that GPU (the driver loads the code
 *    holding it), so make the first call on each GPU before free device
 *    memory is handed out, and before any stream capture; the array then
 *    stays until the process exits.
 *  - Like every entry point here, the call makes the topology's device
 *    current on the calling thread.
 *  - All calls on one GPU share the array: calls that overlap on the GPU
 *    (other threads, other streams) race and must be serialised by the caller.
 *  - stream: a cudaStream_t, or NULL for this thread's stream; the call
 *    returns after the kernels finish. */
int ursa_gpu_connected_components_weak_noalloc(ursa_gpu_topo *t, uint32_t *d_labels, void *stream);

/* triangle_count(&Topology) -> Vec<u32> -- algo/triangle.rs:40-62: triangles
 * through each node of the undirected simple view. */
int ursa_gpu_triangle_count(ursa_gpu_topo *t, uint32_t *out);

/* clustering_coefficient(&Topology) -> Vec<f64> -- algo/clustering.rs:21-40. */
int ursa_gpu_clustering_coefficient(ursa_gpu_topo *t, double *out);

/* betweenness(&Topology, Option<f64>, Option<u64>) -> Vec<f64> --
 * algo/betweenness.rs:153-177.  has_sample/has_seed encode the Options.  The
 * sampled source set is the reference's seeded shuffled_order prefix
 * (betweenness.rs:349-362, rng.rs:64-72), computed on the host. */
int ursa_gpu_betweenness(ursa_gpu_topo *t, int has_sample, double sample, int has_seed,
                         uint64_t seed, double *out);
/* betweenness_weighted(&Topology, &[f64], Option<f64>, Option<u64>) --
 * algo/betweenness.rs:236-270 (ties only on exact f64 equality). */
int ursa_gpu_betweenness_weighted(ursa_gpu_topo *t, const double *weights, uint64_t n_weights,
                                  int has_sample, double sample, int has_seed, uint64_t seed,
                                  double *out);

/* closeness(&Topology) -> Vec<f64> -- algo/closeness.rs:69-135: per node,
 * reachable / sum of hop distances over the nodes it reaches (out-edges),
 * 0.0 if it reaches none.  A bit-parallel BFS from 64 or 256 sources at a
 * time; exact integer folds, so bit-identical to the reference. */
int ursa_gpu_closeness(ursa_gpu_topo *t, double *out);
/* Device-output form of ursa_gpu_closeness: d_out is an n-f64 device array,
 * enqueued on `stream` (NULL = this thread's stream); returns after the
 * work completes.  device_ms (may be NULL): device time of the enqueued
 * work, from events on that stream. */
int ursa_gpu_closeness_device(ursa_gpu_topo *t, double *d_out, void *stream, float *device_ms);
/* closeness_weighted(&Topology, &[f64]) -> Vec<f64> -- algo/closeness.rs:
 * 137-224: Dijkstra distances per source (exact), summed in node order. */
int ursa_gpu_closeness_weighted(ursa_gpu_topo *t, const double *weights, uint64_t n_weights,
                                double *out);
/* avg_path_length(&Topology, Option<f64>) -- ursa-plan/src/stats.rs:142-150:
 * mean hop distance over reachable ordered pairs from all sources (or the
 * deterministic strided sample, stats.rs:82-101); 0.0 with no pair.
 * URSA_GPU_EINVAL if the distance total reaches 2^53. */
int ursa_gpu_avg_path_length(ursa_gpu_topo *t, int has_sample, double sample, double *out);
/* diameter(&Topology, bool approximate) -- stats.rs:152-167: the largest
 * finite hop distance over all sources (or a strided sample of min(128, n)
 * sources when approximate). */
int ursa_gpu_diameter(ursa_gpu_topo *t, int approximate, int64_t *out);

/* ------------------------------------------------------------------------
 * Node-id interning on the device.
 *
 * IdMap::from_edge_batches / from_edge_arrays for Int64 ids
 * (ursa-core/src/id_map.rs:197-320): the edges' user ids, chunk after chunk,
 * become dense u32 ids in first-seen order (per edge, src before dst), as
 * the ingress path does before Topology::build (ursa-plan/src/topology.rs:
 * 39-45).  The caller rejects null endpoints first, as the reference does
 * (IdError::Null).  String (Utf8) ids stay on the host.
 * ---------------------------------------------------------------------- */
typedef struct ursa_gpu_idmap ursa_gpu_idmap;

/* Interns n_chunks chunks of (src, dst) Int64 value buffers (host), each
 * chunk_lens[c] rows; at most 2^29 edges in all. */
int ursa_gpu_idmap_build(uint64_t n_chunks, const int64_t *const *src_chunks,
                         const int64_t *const *dst_chunks, const uint64_t *chunk_lens,
                         ursa_gpu_idmap **out);
void ursa_gpu_idmap_free(ursa_gpu_idmap *m);
/* IdMap::len (id_map.rs:443) and the number of interned edges. */
uint64_t ursa_gpu_idmap_len(const ursa_gpu_idmap *m);
uint64_t ursa_gpu_idmap_n_edges(const ursa_gpu_idmap *m);
/* IdMap::user_id_array (id_map.rs:359): the user ids in dense order. */
int ursa_gpu_idmap_user_ids(ursa_gpu_idmap *m, int64_t *out);
/* The edges in dense ids (the Vec<u32> pair from_edge_batches returns). */
int ursa_gpu_idmap_dense_edges(ursa_gpu_idmap *m, uint32_t *src_out, uint32_t *dst_out);
/* Topology::build(len, dense src, dense dst) straight from the device
 * columns (no host round trip). */
int ursa_gpu_idmap_topology(ursa_gpu_idmap *m, ursa_gpu_topo **out);
/* IdMap::gather_user (id_map.rs:381): user ids of dense indices
 * (URSA_GPU_EINVAL on an index >= len). */
int ursa_gpu_idmap_gather_user(ursa_gpu_idmap *m, const uint32_t *dense, uint64_t n, int64_t *out);
/* IdMap::dense_from_array (id_map.rs:402) for Int64 ids: found[i] = 0 where
 * the id is not in the map (the reference's None). */
int ursa_gpu_idmap_lookup(ursa_gpu_idmap *m, const int64_t *ids, uint64_t n, uint32_t *dense_out,
                          uint8_t *found);

/* ------------------------------------------------------------------------
 * Batched execution of many small independent graphs.
 *
 * The reference runs one graph per Topology: Topology::build
 * (topology.rs:276-298) and then pagerank (algo/pagerank.rs:98-124),
 * connected_components_weak (algo/components.rs:58-68) and triangle_count
 * (algo/triangle.rs:40-62), each call on its own.  A batch holds thousands
 * of graphs on the device at once and runs all three for every graph in ONE
 * launch of a captured CUDA graph; per graph the results equal those of the
 * single-graph calls above (pagerank within the same tolerance, components
 * and triangle counts exactly), and they do not depend on the batch's other
 * graphs or on the launch configuration.
 * ---------------------------------------------------------------------- */
typedef struct ursa_gpu_batch ursa_gpu_batch;

enum {
  URSA_GPU_BATCH_PAGERANK = 1,
  URSA_GPU_BATCH_COMPONENTS = 2,
  URSA_GPU_BATCH_TRIANGLES = 4
};

/* Launch shapes of a batch (bucket and tile shapes).  Pagerank and
 * components run per graph: a graph runs in the first bucket whose capacity
 * (nodes) holds it, and graphs above the last capacity run in the last
 * bucket with their per-node state in global memory; threads: CTA size per
 * bucket (128, 256, 512 or 1024).  Capacities rise and are at most 57,344
 * nodes (224 KB of shared memory per CTA).  Triangle counting runs over the
 * whole batch: warps take tc_tile consecutive vertices of a graph at a time
 * (1..4096), in CTAs of tc_threads (128, 256 or 512). */
typedef struct {
  uint32_t n_buckets; /* 1..3 */
  uint32_t cap[3];
  uint32_t threads[3];
  uint32_t tc_tile;
  uint32_t tc_threads;
} ursa_gpu_batch_config;

/* Uploads a batch: graph g has node_counts[g] nodes and edge_counts[g] edge
 * rows; src/dst hold every graph's rows one graph after another, with LOCAL
 * ids (0 <= id < node_counts[g]) -- per graph the (n, src, dst) of
 * Topology::build.  Totals are limited to u32::MAX nodes and edges.  Builds
 * the union's in-CSR, out-degrees and oriented undirected CSR, and groups
 * each graph's rows by in-degree.  Uses the device selected with
 * ursa_gpu_set_device. */
int ursa_gpu_batch_build(uint64_t n_graphs, const uint64_t *node_counts,
                         const uint64_t *edge_counts, const uint32_t *src, const uint32_t *dst,
                         ursa_gpu_batch **out);
void ursa_gpu_batch_free(ursa_gpu_batch *b);
uint64_t ursa_gpu_batch_n_graphs(const ursa_gpu_batch *b);
uint64_t ursa_gpu_batch_n_nodes(const ursa_gpu_batch *b);
uint64_t ursa_gpu_batch_n_edges(const ursa_gpu_batch *b);
uint64_t ursa_gpu_batch_device_bytes(const ursa_gpu_batch *b);

/* Runs the algorithms selected by `what` (URSA_GPU_BATCH_* flags) for every
 * graph as one CUDA-graph launch (captured on the first call and again
 * whenever params, `what` or the configuration change).  params: pagerank's
 * PageRankParams (pagerank.rs:22-36).  stream: a cudaStream_t to enqueue on
 * and return at once, or NULL for this thread's stream and return when
 * done. */
int ursa_gpu_batch_run(ursa_gpu_batch *b, const ursa_gpu_pagerank_params *params, uint32_t what,
                       void *stream);

/* Autotuner: times the captured launch for a set of bucket capacities, CTA
 * sizes per bucket and triangle tiles (coordinate search, min of two timed
 * launches each) and keeps the fastest.  Writes the choice and its time when
 * the pointers are non-NULL.  Results do not change with the choice. */
int ursa_gpu_batch_tune(ursa_gpu_batch *b, const ursa_gpu_pagerank_params *params, uint32_t what,
                        ursa_gpu_batch_config *chosen, float *best_ms);
int ursa_gpu_batch_set_config(ursa_gpu_batch *b, const ursa_gpu_batch_config *cfg);
int ursa_gpu_batch_get_config(ursa_gpu_batch *b, ursa_gpu_batch_config *cfg);

/* Results of the last run (the copy waits for it, on any stream),
 * concatenated graph after graph in node order (any pointer may be NULL): pagerank f64 and component labels (minimum
 * member LOCAL id) and triangle counts u32, n_nodes each; per graph the
 * pagerank iteration count and last L1 delta, n_graphs each. */
int ursa_gpu_batch_results(ursa_gpu_batch *b, double *pagerank, uint32_t *components,
                           uint32_t *triangles, uint32_t *pr_iterations, double *pr_last_delta);
/* Device addresses of the same result arrays (valid until ursa_gpu_batch_free). */
int ursa_gpu_batch_device_results(ursa_gpu_batch *b, const double **pagerank,
                                  const uint32_t **components, const uint32_t **triangles);

/* ------------------------------------------------------------------------
 * Serving loop.
 *
 * The reference answers each query with one kernel call through its plan
 * layer: shortest_path (algo/bfs.rs:48-102, via ursa-plan/src/result.rs:216),
 * k_hop (algo/hop.rs:52-130, via result.rs:180), bfs_distances
 * (algo/bfs.rs:18-42) and pagerank (algo/pagerank.rs:98-124, via
 * result.rs:82-140).  A server keeps a resident topology (shortest_path, hop
 * and bfs queries) and uploaded small graphs
 * (pagerank queries) on the device and runs submitted queries with
 * continuous batching: each lane (a stream with preallocated slots, one
 * query type) launches one kernel for up to `slots` pending queries, lanes
 * run concurrently, and a lane is refilled as soon as its launch finishes.
 * Results do not depend on the other queries of a launch:
 *  - shortest_path: a shortest path over out-edges (bidirectional BFS; hop
 *    count equal to the reference's; on ties the path may differ from the
 *    reference's serial-order choice), -1 length when there is none;
 *  - hop: the nodes k_hop(&[seed], k, Out) pairs with the seed, in the
 *    reference's emission order;
 *  - bfs: bfs_distances(source, direction) -- n i32 hop distances, -1 where
 *    unreached (all -1 for an out-of-range source); up to 64 queries of one
 *    direction share a launch (one bit each in per-node masks);
 *  - pagerank: the batch kernel's ranks of the uploaded graph.
 * Slot kernels wait for queries with bounded waits: they return when the
 * scheduler's heartbeat (bumped every heartbeat_period_us) has not moved
 * for heartbeat_limit_ns, and the server counts each such return in
 * wait_expiries (the lane is relaunched for the next query).
 * ---------------------------------------------------------------------- */
typedef struct ursa_gpu_server ursa_gpu_server;

enum {
  URSA_GPU_QUERY_SHORTEST_PATH = 1,
  URSA_GPU_QUERY_HOP = 2,
  URSA_GPU_QUERY_PAGERANK = 3,
  URSA_GPU_QUERY_BFS = 4
};

typedef struct {
  uint32_t path_lanes, path_slots; /* shortest_path: lanes and queries per launch */
  uint32_t hop_lanes, hop_slots;
  uint32_t pr_lanes, pr_slots;
  uint64_t pr_max_nodes;           /* largest uploaded graph, in nodes */
  uint64_t hbm_reserve_bytes;      /* free HBM an upload must leave */
  uint64_t upload_budget_bytes;    /* device bytes of live uploads (0 = no cap) */
  uint32_t bfs_lanes, bfs_slots;   /* bfs: lanes and queries per launch (<= 64).  Each
                                      answer (n i32) waits in one of 2 x lanes x slots
                                      pinned host buffers (allocated with the server)
                                      until its result is fetched; with none free the
                                      bfs lanes wait, the other lanes do not */
  uint64_t heartbeat_limit_ns;     /* slot kernels return after this long without a
                                      heartbeat (0 = 5 s) */
  uint64_t heartbeat_period_us;    /* the scheduler bumps the heartbeat this often
                                      (0 = every 1000 us) */
} ursa_gpu_server_config;

typedef struct {
  uint32_t type;     /* URSA_GPU_QUERY_* */
  uint32_t graph;    /* pagerank: the uploaded graph's id */
  uint32_t source;   /* shortest_path source, hop seed */
  uint32_t target;   /* shortest_path target */
  uint32_t k;        /* hop depth */
  ursa_gpu_pagerank_params pr;
  uint32_t direction; /* bfs: 0 = Out, 1 = In, 2 = Both */
} ursa_gpu_query;

typedef struct {
  int32_t status;     /* URSA_GPU_OK, URSA_GPU_ECANCELED, ... */
  uint32_t type;
  int64_t result_len; /* path nodes (-1 = no path), reached nodes, distances or ranks */
  uint32_t iterations;
  double last_delta;
  uint64_t edges;     /* edges the query scanned */
  double submit_us, launch_us, done_us; /* host steady clock */
} ursa_gpu_query_info;

typedef struct {
  uint64_t submitted, completed, launches;
  uint64_t uploads_admitted, uploads_rejected, uploads_live, upload_bytes, pending;
  uint64_t wait_expiries; /* slot kernels that returned because a bounded wait ran out */
} ursa_gpu_server_stats;

/* Creates a server over `resident` (may be NULL when no path/hop lanes are
 * configured; the caller keeps it alive until the server is destroyed).
 * Every slot's scratch is allocated here (shortest_path 32 B and hop 20 B
 * per resident node per slot). */
int ursa_gpu_server_create(ursa_gpu_topo *resident, const ursa_gpu_server_config *cfg,
                           ursa_gpu_server **out);
/* Stops the scheduler (queries in flight finish; pending ones are dropped)
 * and frees everything the server owns, uploads included. */
void ursa_gpu_server_destroy(ursa_gpu_server *s);
/* Uploads a graph (Topology::build arguments) for pagerank queries.
 * Admission by free HBM: URSA_GPU_ENOMEM when the build would leave less
 * than hbm_reserve_bytes free or exceed upload_budget_bytes. */
int ursa_gpu_server_upload(ursa_gpu_server *s, uint64_t n_nodes, const uint32_t *src,
                           const uint32_t *dst, uint64_t n_edges, uint32_t *graph_id);
/* Frees an upload once the queries that use it have finished. */
int ursa_gpu_server_release(ursa_gpu_server *s, uint32_t graph_id);
/* Queues a query; *ticket identifies it. */
int ursa_gpu_server_submit(ursa_gpu_server *s, const ursa_gpu_query *q, uint64_t *ticket);
/* Cancels a query: a queued one completes at once with URSA_GPU_ECANCELED,
 * a running shortest_path / hop stops at its next BFS level. */
int ursa_gpu_server_cancel(ursa_gpu_server *s, uint64_t ticket);
/* Waits up to timeout_us (0 = just look) for a query; URSA_GPU_ETIMEOUT if
 * it has not completed.  info may be NULL. */
int ursa_gpu_server_wait(ursa_gpu_server *s, uint64_t ticket, uint64_t timeout_us,
                         ursa_gpu_query_info *info);
/* Tickets completed since the last poll (up to cap). */
int ursa_gpu_server_poll(ursa_gpu_server *s, uint64_t *tickets, uint64_t cap, uint64_t *n_out);
/* Hands over a completed query's result and forgets the ticket: u32 nodes
 * (path, hop), i32 distances (bfs) or f64 ranks (pagerank), info.result_len
 * elements (0 for no path); URSA_GPU_ETRUNC if cap_elems is too small. */
int ursa_gpu_server_result(ursa_gpu_server *s, uint64_t ticket, ursa_gpu_query_info *info,
                           void *out, uint64_t cap_elems);
int ursa_gpu_server_get_stats(ursa_gpu_server *s, ursa_gpu_server_stats *stats);

/* ------------------------------------------------------------------------
 * Arrow results: the "Arrow arrays out" half of the operator
 * (ursa-plan/src/result.rs:144-261).
 *
 * query_batch computes every requested column on the device into one staging
 * block laid out as Arrow value buffers, translates the id column (or the
 * hop / path endpoints) dense -> user on the device, and copies the block to
 * pinned host memory once.  The result exports as an Arrow C Data Interface
 * struct array (one RecordBatch): its buffers point into that pinned block,
 * so a consumer (arrow-rs FFI_ArrowArray, pyarrow _import_from_c) takes the
 * columns without another copy; the block lives until the result and every
 * export of it are released.  Without an IdMap (ids == NULL) the id columns
 * are the dense UInt32 node indices.
 * ------------------------------------------------------------------------ */

/* The Arrow C Data Interface structures, as the Arrow specification defines
 * them (skipped if the consumer's Arrow headers already did). */
#ifndef ARROW_C_DATA_INTERFACE
#define ARROW_C_DATA_INTERFACE
#define ARROW_FLAG_DICTIONARY_ORDERED 1
#define ARROW_FLAG_NULLABLE 2
#define ARROW_FLAG_MAP_KEYS_SORTED 4
struct ArrowSchema {
  const char *format;
  const char *name;
  const char *metadata;
  int64_t flags;
  int64_t n_children;
  struct ArrowSchema **children;
  struct ArrowSchema *dictionary;
  void (*release)(struct ArrowSchema *);
  void *private_data;
};
struct ArrowArray {
  int64_t length;
  int64_t null_count;
  int64_t offset;
  int64_t n_buffers;
  int64_t n_children;
  const void **buffers;
  struct ArrowArray **children;
  struct ArrowArray *dictionary;
  void (*release)(struct ArrowArray *);
  void *private_data;
};
#endif

typedef struct ursa_gpu_result ursa_gpu_result;

/* GraphAlgo (ursa-plan/src/logical.rs:37-65). */
enum {
  URSA_GPU_ALGO_PAGERANK = 0,
  URSA_GPU_ALGO_CONNECTED_COMPONENTS = 1,
  URSA_GPU_ALGO_DEGREE = 2,
  URSA_GPU_ALGO_TRIANGLE_COUNT = 3,
  URSA_GPU_ALGO_CLUSTERING_COEFFICIENT = 4,
  URSA_GPU_ALGO_BETWEENNESS = 5,
  URSA_GPU_ALGO_CLOSENESS = 6,
  URSA_GPU_ALGO_LABEL_PROPAGATION = 7, /* host-side kernel: URSA_GPU_EINVAL here */
  URSA_GPU_ALGO_LOUVAIN = 8            /* host-side kernel: URSA_GPU_EINVAL here */
};

/* OutputColumn::Algo (result.rs:28-35; value types result.rs:52-63): a
 * named node-valued column.  Only the fields of `algo` are read.  weights:
 * n_edges f64 by edge row (host), or NULL; present for pagerank, betweenness
 * and closeness (their weighted forms).  Strong components (strong != 0)
 * run on the host: URSA_GPU_EINVAL. */
typedef struct {
  const char *name;
  int algo;
  double damping;    /* PAGERANK */
  uint32_t max_iter; /* PAGERANK */
  double tol;        /* PAGERANK */
  int strong;        /* CONNECTED_COMPONENTS */
  int direction;     /* DEGREE: 0 out, 1 in, 2 both */
  int has_sample;    /* BETWEENNESS */
  double sample;
  int has_seed;
  uint64_t seed;
  const double *weights;
  uint64_t n_weights;
} ursa_gpu_output_column;

/* query_schema + query_batch (result.rs:144-168): columns ("id", name_1,
 * ...), n_nodes rows; id is Int64 (the IdMap's user ids) or UInt32; Float64
 * for pagerank, clustering, closeness and betweenness, UInt32 otherwise; none
 * nullable.  ids, when given, must hold exactly the topology's nodes. */
int ursa_gpu_query_batch(ursa_gpu_topo *t, ursa_gpu_idmap *ids, const ursa_gpu_output_column *cols,
                         uint64_t n_cols, ursa_gpu_result **out);
/* hop_schema + hop_batch (result.rs:171-199): ("src", "dst") = (seed,
 * reached) per k_hop pair, in k_hop's order. */
int ursa_gpu_hop_batch(ursa_gpu_topo *t, ursa_gpu_idmap *ids, const uint32_t *seeds,
                       uint64_t n_seeds, uint32_t k, int dir, ursa_gpu_result **out);
/* path_schema + path_batch (result.rs:203-261): ("src", "dst", "hop" Int64,
 * "cost" Float64), one row per path edge; cost = the settled distance of the
 * edge's destination (weights given) or hop + 1.  No row for an unreachable
 * target or a one-node path. */
int ursa_gpu_path_batch(ursa_gpu_topo *t, ursa_gpu_idmap *ids, uint32_t source, uint32_t target,
                        int dir, const double *weights, uint64_t n_weights, ursa_gpu_result **out);
uint64_t ursa_gpu_result_num_rows(const ursa_gpu_result *r);
uint64_t ursa_gpu_result_num_columns(const ursa_gpu_result *r);
/* Exports the result as a struct array and its schema (format "+s", one
 * child per column).  The consumer calls each structure's release. */
int ursa_gpu_result_export(ursa_gpu_result *r, struct ArrowSchema *schema, struct ArrowArray *array);
/* Drops the caller's reference; exported arrays keep the block alive. */
void ursa_gpu_result_free(ursa_gpu_result *r);

#ifdef __cplusplus
}
#endif
#endif
