"""ctypes front end of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA path and the timed
CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU legs
use it.  The functions mirror ursa-core's kernel signatures
(ursa-core/src/algo/mod.rs:35-50) with numpy arrays in place of Vecs.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")

DIR = {"out": 0, "in": 1, "both": 2}


def build() -> str:
    """Compile liboracle.so with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        P = C.c_void_p
        u64, u32, i64, f64, i32 = C.c_uint64, C.c_uint32, C.c_int64, C.c_double, C.c_int
        L.orc_topo_build.restype = P
        L.orc_topo_build.argtypes = [u64, P, P, u64]
        L.orc_topo_free.argtypes = [P]
        L.orc_topo_n_nodes.restype = u64
        L.orc_topo_n_nodes.argtypes = [P]
        L.orc_topo_n_edges.restype = u64
        L.orc_topo_n_edges.argtypes = [P]
        L.orc_topo_csr.argtypes = [P, i32, P, P, P]
        L.orc_topo_undirected_len.restype = u64
        L.orc_topo_undirected_len.argtypes = [P]
        L.orc_topo_undirected.argtypes = [P, P, P]
        L.orc_degree.argtypes = [P, i32, P]
        L.orc_pagerank.restype = u32
        L.orc_pagerank.argtypes = [P, f64, u32, f64, P]
        L.orc_pagerank_weighted.restype = u32
        L.orc_pagerank_weighted.argtypes = [P, P, f64, u32, f64, P]
        L.orc_pagerank_deltas.restype = u32
        L.orc_pagerank_deltas.argtypes = [P, u32]
        L.orc_bfs_distances.argtypes = [P, u32, i32, P]
        L.orc_shortest_path.restype = i64
        L.orc_shortest_path.argtypes = [P, u32, u32, i32, P]
        L.orc_dijkstra_distances.argtypes = [P, P, u32, i32, P]
        L.orc_shortest_path_weighted_with_cost.restype = i64
        L.orc_shortest_path_weighted_with_cost.argtypes = [P, P, u32, u32, i32, P, P]
        L.orc_k_hop.restype = u64
        L.orc_k_hop.argtypes = [P, P, u64, u32, i32, C.POINTER(P), C.POINTER(P)]
        L.orc_free.argtypes = [P]
        L.orc_connected_components_weak.argtypes = [P, P]
        L.orc_triangle_count.argtypes = [P, P]
        L.orc_triangle_count_nodes.argtypes = [P, P, u64, P]
        L.orc_clustering_coefficient.argtypes = [P, P]
        L.orc_betweenness.argtypes = [P, i32, f64, i32, u64, P]
        L.orc_betweenness_weighted.argtypes = [P, P, i32, f64, i32, u64, P]
        L.orc_betweenness_sources.argtypes = [P, P, P, u64, P]
        L.orc_shuffled_order.argtypes = [u64, u64, P]
        L.orc_sample_indices.restype = u64
        L.orc_sample_indices.argtypes = [u64, u64, i32, u64, P]
        L.orc_sample_sources.restype = u64
        L.orc_sample_sources.argtypes = [u64, i32, f64, i32, u64, P]
        L.orc_closeness.argtypes = [P, P]
        L.orc_closeness_sources.argtypes = [P, P, u64, P]
        L.orc_closeness_weighted.argtypes = [P, P, P]
        L.orc_avg_path_length.restype = f64
        L.orc_avg_path_length.argtypes = [P, i32, f64]
        L.orc_diameter.restype = i64
        L.orc_diameter.argtypes = [P, i32]
        L.orc_idmap_build.restype = u64
        L.orc_idmap_build.argtypes = [P, P, u64, P, P, P]
        L.orc_set_threads.argtypes = [i32]
        L.orc_get_threads.restype = i32
        _lib = L
    return _lib


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return lib().orc_get_threads()


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


class Topology:
    """Topology::build (ursa-core/src/topology.rs:276-298)."""

    def __init__(self, n_nodes: int, src, dst):
        src, dst = _u32(src), _u32(dst)
        if src.shape != dst.shape:
            raise ValueError("src/dst length mismatch")
        self._h = lib().orc_topo_build(int(n_nodes), _p(src), _p(dst), src.size)
        if not self._h:
            raise ValueError("invalid topology input (endpoint >= n_nodes or too many edges)")
        self.n = int(n_nodes)
        self.m = int(src.size)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_topo_free(h)
            self._h = None

    def csr(self, direction: str = "out"):
        off = np.empty(self.n + 1, np.uint64)
        tg = np.empty(self.m, np.uint32)
        eid = np.empty(self.m, np.uint32)
        lib().orc_topo_csr(self._h, DIR[direction], _p(off), _p(tg), _p(eid))
        return off, tg, eid

    def undirected(self):
        ms = lib().orc_topo_undirected_len(self._h)
        off = np.empty(self.n + 1, np.uint64)
        tg = np.empty(ms, np.uint32)
        lib().orc_topo_undirected(self._h, _p(off), _p(tg))
        return off, tg


def degree(t: Topology, direction: str = "out") -> np.ndarray:
    out = np.empty(t.n, np.uint32)
    lib().orc_degree(t._h, DIR[direction], _p(out))
    return out


def pagerank(t: Topology, damping=0.85, max_iter=30, tol=1e-6, return_iters=False):
    out = np.empty(t.n, np.float64)
    it = lib().orc_pagerank(t._h, damping, max_iter, tol, _p(out))
    return (out, it) if return_iters else out


def pagerank_deltas() -> np.ndarray:
    """L1 residual of every iteration of this thread's last pagerank call."""
    buf = np.empty(4096, np.float64)
    k = lib().orc_pagerank_deltas(_p(buf), buf.size)
    return buf[: min(k, buf.size)].copy()


def pagerank_weighted(t: Topology, weights, damping=0.85, max_iter=30, tol=1e-6, return_iters=False):
    w = _f64(weights)
    if w.size != t.m:
        raise ValueError("weights length must equal the edge count")
    out = np.empty(t.n, np.float64)
    it = lib().orc_pagerank_weighted(t._h, _p(w), damping, max_iter, tol, _p(out))
    return (out, it) if return_iters else out


def bfs_distances(t: Topology, source: int, direction: str = "out") -> np.ndarray:
    out = np.empty(t.n, np.int32)
    lib().orc_bfs_distances(t._h, source, DIR[direction], _p(out))
    return out


def shortest_path(t: Topology, source: int, target: int, direction: str = "out"):
    buf = np.empty(max(t.n, 1), np.uint32)
    ln = lib().orc_shortest_path(t._h, source, target, DIR[direction], _p(buf))
    return None if ln < 0 else [int(x) for x in buf[:ln]]


def dijkstra_distances(t: Topology, weights, source: int, direction: str = "out"):
    w = _f64(weights)
    out = np.empty(t.n, np.float64)
    lib().orc_dijkstra_distances(t._h, _p(w), source, DIR[direction], _p(out))
    return out


def shortest_path_weighted_with_cost(t: Topology, weights, source: int, target: int, direction="out"):
    w = _f64(weights)
    buf = np.empty(max(t.n, 1), np.uint32)
    cost = np.empty(max(t.n, 1), np.float64)
    ln = lib().orc_shortest_path_weighted_with_cost(t._h, _p(w), source, target, DIR[direction], _p(buf), _p(cost))
    if ln < 0:
        return None
    return [int(x) for x in buf[:ln]], [float(x) for x in cost[:ln]]


def shortest_path_weighted(t: Topology, weights, source: int, target: int, direction="out"):
    r = shortest_path_weighted_with_cost(t, weights, source, target, direction)
    return None if r is None else r[0]


def k_hop(t: Topology, seeds, k: int, direction: str = "out"):
    s = _u32(seeds)
    ps, pd = C.c_void_p(), C.c_void_p()
    cnt = lib().orc_k_hop(t._h, _p(s), s.size, k, DIR[direction], C.byref(ps), C.byref(pd))
    src = np.empty(cnt, np.uint32)
    dst = np.empty(cnt, np.uint32)
    if cnt:
        C.memmove(src.ctypes.data, ps.value, cnt * 4)
        C.memmove(dst.ctypes.data, pd.value, cnt * 4)
    if ps.value:
        lib().orc_free(ps)
    if pd.value:
        lib().orc_free(pd)
    return src, dst


def connected_components_weak(t: Topology) -> np.ndarray:
    out = np.empty(t.n, np.uint32)
    lib().orc_connected_components_weak(t._h, _p(out))
    return out


def triangle_count(t: Topology) -> np.ndarray:
    out = np.zeros(t.n, np.uint32)
    lib().orc_triangle_count(t._h, _p(out))
    return out


def triangle_count_nodes(t: Topology, nodes) -> np.ndarray:
    """triangle_count's values for the given nodes only (the reference counts
    each node on its own, triangle.rs:23-62)."""
    nodes = np.ascontiguousarray(nodes, np.uint32)
    assert nodes.size == 0 or int(nodes.max()) < t.n
    out = np.zeros(nodes.size, np.uint32)
    lib().orc_triangle_count_nodes(t._h, _p(nodes), nodes.size, _p(out))
    return out


def clustering_coefficient(t: Topology) -> np.ndarray:
    out = np.zeros(t.n, np.float64)
    lib().orc_clustering_coefficient(t._h, _p(out))
    return out


def betweenness(t: Topology, sample=None, seed=None) -> np.ndarray:
    out = np.zeros(t.n, np.float64)
    lib().orc_betweenness(t._h, sample is not None, float(sample or 0.0), seed is not None, int(seed or 0), _p(out))
    return out


def betweenness_weighted(t: Topology, weights, sample=None, seed=None) -> np.ndarray:
    w = _f64(weights)
    if w.size != t.m:
        raise ValueError("weights length must equal the edge count")
    out = np.zeros(t.n, np.float64)
    lib().orc_betweenness_weighted(
        t._h, _p(w), sample is not None, float(sample or 0.0), seed is not None, int(seed or 0), _p(out)
    )
    return out


def betweenness_sources(t: Topology, sources, weights=None) -> np.ndarray:
    s = _u32(sources)
    w = None if weights is None else _f64(weights)
    out = np.zeros(t.n, np.float64)
    lib().orc_betweenness_sources(t._h, _p(w), _p(s), s.size, _p(out))
    return out


def shuffled_order(n: int, seed: int) -> np.ndarray:
    out = np.empty(n, np.uint32)
    lib().orc_shuffled_order(n, seed, _p(out))
    return out


def sample_indices(r: int, k: int, seed=None) -> list[int]:
    out = np.empty(max(min(k, r), 1), np.uint64)
    cnt = lib().orc_sample_indices(r, k, seed is not None, int(seed or 0), _p(out))
    return [int(x) for x in out[:cnt]]


def sample_sources(n: int, sample=None, seed=None) -> np.ndarray:
    out = np.empty(max(n, 1), np.uint32)
    k = lib().orc_sample_sources(n, sample is not None, float(sample or 0.0), seed is not None, int(seed or 0), _p(out))
    return out[:k].copy()


def idmap_build(src, dst):
    """IdMap::from_edge_arrays / from_edge_batches for Int64 ids
    (ursa-core/src/id_map.rs:197-320): (to_user i64[n], dense_src u32[m],
    dense_dst u32[m]); chunked input is the same as its concatenation."""
    s = np.ascontiguousarray(np.asarray(src, dtype=np.int64))
    d = np.ascontiguousarray(np.asarray(dst, dtype=np.int64))
    if s.shape != d.shape:
        raise ValueError("src and dst columns must have the same length")
    ds = np.empty(s.size, np.uint32)
    dd = np.empty(s.size, np.uint32)
    users = np.empty(2 * s.size, np.int64)
    k = lib().orc_idmap_build(_p(s), _p(d), s.size, _p(ds), _p(dd), _p(users))
    return users[:k].copy(), ds, dd


def closeness(t: Topology) -> np.ndarray:
    """closeness (ursa-core/src/algo/closeness.rs:69-135)."""
    out = np.empty(t.n, np.float64)
    lib().orc_closeness(t._h, _p(out))
    return out


def closeness_sources(t: Topology, sources) -> np.ndarray:
    """closeness_one (closeness.rs:98-128) for the given sources only."""
    src = np.ascontiguousarray(np.asarray(sources, dtype=np.uint32))
    out = np.empty(src.size, np.float64)
    lib().orc_closeness_sources(t._h, _p(src), C.c_uint64(src.size), _p(out))
    return out


def closeness_weighted(t: Topology, weights) -> np.ndarray:
    """closeness_weighted (ursa-core/src/algo/closeness.rs:137-224)."""
    w = _f64(weights)
    out = np.empty(t.n, np.float64)
    lib().orc_closeness_weighted(t._h, _p(w), _p(out))
    return out


def avg_path_length(t: Topology, sample=None) -> float:
    """avg_path_length (ursa-plan/src/stats.rs:142-150)."""
    return float(lib().orc_avg_path_length(t._h, int(sample is not None), float(sample or 0.0)))


def diameter(t: Topology, approximate: bool = True) -> int:
    """diameter (ursa-plan/src/stats.rs:152-167)."""
    return int(lib().orc_diameter(t._h, int(bool(approximate))))
