"""Host mirror of ursa-core's kernel functions (ursa-core/src/algo/mod.rs:35-50).

Same names, argument meaning and edge-case behaviour as the Rust functions;
Vecs become numpy arrays and Option becomes None.  Every call runs on the GPU
through the C ABI; a non-OK status raises UrsaGpuError.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import PageRankParams, PageRankStats
from .topology import Direction, Topology


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def default_pagerank_params() -> PageRankParams:
    """PageRankParams::default (pagerank.rs:28-36)."""
    return PageRankParams(0.85, 30, 1e-6)


def degree(topo: Topology, direction=Direction.Out) -> np.ndarray:
    """degree (algo/degree.rs:12-30)."""
    out = np.empty(topo.n_nodes(), np.uint32)
    _lib.check(_lib.load().ursa_gpu_degree(topo.handle, int(Direction.of(direction)), out.ctypes.data))
    return out


def _params(params, damping, max_iter, tol) -> PageRankParams:
    if params is None:
        params = default_pagerank_params()
        if damping is not None:
            params.damping = damping
        if max_iter is not None:
            params.max_iter = max_iter
        if tol is not None:
            params.tol = tol
    return params


def pagerank(topo: Topology, params: PageRankParams | None = None, *, damping=None, max_iter=None,
             tol=None, stats: PageRankStats | None = None) -> np.ndarray:
    """pagerank (algo/pagerank.rs:98-124)."""
    p = _params(params, damping, max_iter, tol)
    out = np.empty(topo.n_nodes(), np.float64)
    _lib.check(
        _lib.load().ursa_gpu_pagerank(topo.handle, C.byref(p), out.ctypes.data, C.byref(stats) if stats else None)
    )
    return out


def pagerank_weighted(topo: Topology, weights, params: PageRankParams | None = None, *, damping=None,
                      max_iter=None, tol=None, stats: PageRankStats | None = None) -> np.ndarray:
    """pagerank_weighted (algo/pagerank.rs:135-169)."""
    p = _params(params, damping, max_iter, tol)
    w = _f64(weights)
    out = np.empty(topo.n_nodes(), np.float64)
    _lib.check(
        _lib.load().ursa_gpu_pagerank_weighted(
            topo.handle, w.ctypes.data, w.size, C.byref(p), out.ctypes.data, C.byref(stats) if stats else None
        )
    )
    return out


def bfs_distances(topo: Topology, source: int, direction=Direction.Out) -> np.ndarray:
    """bfs_distances (algo/bfs.rs:18-42)."""
    out = np.empty(topo.n_nodes(), np.int32)
    _lib.check(_lib.load().ursa_gpu_bfs_distances(topo.handle, int(source), int(Direction.of(direction)), out.ctypes.data))
    return out


def bfs_distances_multi(topo: Topology, sources, direction=Direction.Out) -> np.ndarray:
    """bfs_distances from many sources in one bit-parallel traversal (an
    extension of algo/bfs.rs:18-42): row i is bfs_distances(sources[i])."""
    src = _u32(sources)
    out = np.empty((src.size, topo.n_nodes()), np.int32)
    if src.size and topo.n_nodes():
        _lib.check(_lib.load().ursa_gpu_bfs_distances_multi(topo.handle, src.ctypes.data, src.size,
                                                            int(Direction.of(direction)), out.ctypes.data))
    return out


def shortest_path(topo: Topology, source: int, target: int, direction=Direction.Out):
    """shortest_path (algo/bfs.rs:48-102): list of node ids, or None."""
    L = _lib.load()
    cap = max(topo.n_nodes(), 1)
    buf = np.empty(cap, np.uint32)
    ln = C.c_int64()
    _lib.check(L.ursa_gpu_shortest_path(topo.handle, int(source), int(target), int(Direction.of(direction)),
                                        buf.ctypes.data, cap, C.byref(ln)))
    return None if ln.value < 0 else [int(x) for x in buf[: ln.value]]


def shortest_path_bidirectional(topo: Topology, source: int, target: int):
    """shortest_path over out-edges by the serving loop's bidirectional BFS,
    one query per launch (an extension of algo/bfs.rs:48-102: same hop count,
    ties resolved as a server's shortest_path query): node list or None."""
    cap = 4096
    buf = np.empty(cap, np.uint32)
    ln = C.c_int64()
    _lib.check(_lib.load().ursa_gpu_shortest_path_bidirectional(topo.handle, int(source), int(target),
                                                                buf.ctypes.data, cap, C.byref(ln)))
    return None if ln.value < 0 else [int(x) for x in buf[: ln.value]]


def dijkstra_distances(topo: Topology, weights, source: int, direction=Direction.Out) -> np.ndarray:
    """dijkstra_distances (algo/bfs.rs:126-166)."""
    w = _f64(weights)
    out = np.empty(topo.n_nodes(), np.float64)
    _lib.check(_lib.load().ursa_gpu_dijkstra_distances(topo.handle, w.ctypes.data, w.size, int(source),
                                                        int(Direction.of(direction)), out.ctypes.data))
    return out


def shortest_path_weighted_with_cost(topo: Topology, weights, source: int, target: int, direction=Direction.Out):
    """shortest_path_weighted_with_cost (algo/bfs.rs:192-259): (path, costs) or None."""
    w = _f64(weights)
    cap = max(topo.n_nodes(), 1)
    buf = np.empty(cap, np.uint32)
    cost = np.empty(cap, np.float64)
    ln = C.c_int64()
    _lib.check(_lib.load().ursa_gpu_shortest_path_weighted_with_cost(
        topo.handle, w.ctypes.data, w.size, int(source), int(target), int(Direction.of(direction)),
        buf.ctypes.data, cost.ctypes.data, cap, C.byref(ln)))
    if ln.value < 0:
        return None
    return [int(x) for x in buf[: ln.value]], [float(x) for x in cost[: ln.value]]


def shortest_path_weighted(topo: Topology, weights, source: int, target: int, direction=Direction.Out):
    """shortest_path_weighted (algo/bfs.rs:176-184)."""
    r = shortest_path_weighted_with_cost(topo, weights, source, target, direction)
    return None if r is None else r[0]


def k_hop(topo: Topology, seeds, k: int, direction=Direction.Out):
    """k_hop (algo/hop.rs:52-75): (seeds_out, reached) u32 arrays."""
    L = _lib.load()
    s = _u32(seeds)
    h = C.c_void_p()
    _lib.check(L.ursa_gpu_k_hop(topo.handle, s.ctypes.data if s.size else None, s.size, int(k),
                                int(Direction.of(direction)), C.byref(h)))
    try:
        n = int(L.ursa_gpu_pairs_len(h))
        a = np.empty(n, np.uint32)
        b = np.empty(n, np.uint32)
        if n:
            _lib.check(L.ursa_gpu_pairs_copy(h, a.ctypes.data, b.ctypes.data))
    finally:
        L.ursa_gpu_pairs_free(h)
    return a, b


def connected_components_weak(topo: Topology) -> np.ndarray:
    """connected_components_weak (algo/components.rs:58-68); min-member labels."""
    out = np.empty(topo.n_nodes(), np.uint32)
    _lib.check(_lib.load().ursa_gpu_connected_components_weak(topo.handle, out.ctypes.data))
    return out


def triangle_count(topo: Topology) -> np.ndarray:
    """triangle_count (algo/triangle.rs:40-62)."""
    out = np.empty(topo.n_nodes(), np.uint32)
    _lib.check(_lib.load().ursa_gpu_triangle_count(topo.handle, out.ctypes.data))
    return out


def clustering_coefficient(topo: Topology) -> np.ndarray:
    """clustering_coefficient (algo/clustering.rs:21-40)."""
    out = np.empty(topo.n_nodes(), np.float64)
    _lib.check(_lib.load().ursa_gpu_clustering_coefficient(topo.handle, out.ctypes.data))
    return out


def betweenness(topo: Topology, sample: float | None = None, seed: int | None = None) -> np.ndarray:
    """betweenness (algo/betweenness.rs:153-177)."""
    out = np.empty(topo.n_nodes(), np.float64)
    _lib.check(_lib.load().ursa_gpu_betweenness(topo.handle, sample is not None, float(sample or 0.0),
                                                 seed is not None, int(seed or 0), out.ctypes.data))
    return out


def betweenness_weighted(topo: Topology, weights, sample: float | None = None, seed: int | None = None) -> np.ndarray:
    """betweenness_weighted (algo/betweenness.rs:236-270)."""
    w = _f64(weights)
    out = np.empty(topo.n_nodes(), np.float64)
    _lib.check(_lib.load().ursa_gpu_betweenness_weighted(topo.handle, w.ctypes.data, w.size, sample is not None,
                                                          float(sample or 0.0), seed is not None, int(seed or 0),
                                                          out.ctypes.data))
    return out


def closeness(topo: Topology) -> np.ndarray:
    """closeness (algo/closeness.rs:69-135)."""
    out = np.empty(topo.n_nodes(), np.float64)
    _lib.check(_lib.load().ursa_gpu_closeness(topo.handle, out.ctypes.data))
    return out


def closeness_weighted(topo: Topology, weights) -> np.ndarray:
    """closeness_weighted (algo/closeness.rs:137-224)."""
    w = _f64(weights)
    out = np.empty(topo.n_nodes(), np.float64)
    _lib.check(_lib.load().ursa_gpu_closeness_weighted(topo.handle, w.ctypes.data, w.size, out.ctypes.data))
    return out


def avg_path_length(topo: Topology, sample=None) -> float:
    """avg_path_length (ursa-plan/src/stats.rs:142-150)."""
    out = C.c_double()
    _lib.check(_lib.load().ursa_gpu_avg_path_length(topo.handle, int(sample is not None),
                                                     float(sample or 0.0), C.byref(out)))
    return out.value


def diameter(topo: Topology, approximate: bool = True) -> int:
    """diameter (ursa-plan/src/stats.rs:152-167)."""
    out = C.c_int64()
    _lib.check(_lib.load().ursa_gpu_diameter(topo.handle, int(bool(approximate)), C.byref(out)))
    return out.value
