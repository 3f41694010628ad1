"""Batched execution of many small independent graphs (the ursa_gpu_batch_*
entry points of include/ursa_gpu.h).

Per graph, a batch computes what ursa-core computes with one Topology::build
(ursa-core/src/topology.rs:276-298) followed by pagerank (algo/pagerank.rs:
98-124), connected_components_weak (algo/components.rs:58-68) and
triangle_count (algo/triangle.rs:40-62); the batch runs all of them for all
graphs in one launch of a captured CUDA graph.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import BATCH_COMPONENTS, BATCH_PAGERANK, BATCH_TRIANGLES, BatchConfig, PageRankParams

ALL = BATCH_PAGERANK | BATCH_COMPONENTS | BATCH_TRIANGLES


@dataclass
class BatchResults:
    """Per-node arrays concatenated graph after graph (node order), and
    per-graph pagerank statistics."""

    pagerank: np.ndarray      # f64[n_nodes]
    components: np.ndarray    # u32[n_nodes], minimum member local id
    triangles: np.ndarray     # u32[n_nodes]
    iterations: np.ndarray    # u32[n_graphs]
    last_delta: np.ndarray    # f64[n_graphs]
    node_offsets: np.ndarray  # u64[n_graphs + 1]

    def graph(self, g: int) -> dict:
        a, b = int(self.node_offsets[g]), int(self.node_offsets[g + 1])
        return {
            "pagerank": self.pagerank[a:b],
            "components": self.components[a:b],
            "triangles": self.triangles[a:b],
            "iterations": int(self.iterations[g]),
            "last_delta": float(self.last_delta[g]),
        }


class GraphBatch:
    """A device-resident batch of graphs.  node_counts[g] / edge_counts[g]
    give each graph's size; src/dst hold every graph's edge rows one graph
    after another with local ids."""

    def __init__(self, node_counts, edge_counts, src, dst):
        n = np.ascontiguousarray(np.asarray(node_counts, dtype=np.uint64))
        m = np.ascontiguousarray(np.asarray(edge_counts, dtype=np.uint64))
        if n.shape != m.shape:
            raise ValueError("node_counts and edge_counts differ in length")
        src = np.ascontiguousarray(np.asarray(src, dtype=np.uint32))
        dst = np.ascontiguousarray(np.asarray(dst, dtype=np.uint32))
        if src.shape != dst.shape or src.size != int(m.sum()):
            raise ValueError("src/dst must hold sum(edge_counts) rows")
        h = C.c_void_p()
        _lib.check(
            _lib.load().ursa_gpu_batch_build(n.size, n.ctypes.data, m.ctypes.data, src.ctypes.data,
                                            dst.ctypes.data, C.byref(h))
        )
        self._h = h
        self.node_counts = n
        self.edge_counts = m
        self.node_offsets = np.zeros(n.size + 1, np.uint64)
        np.cumsum(n, out=self.node_offsets[1:])

    @classmethod
    def from_graphs(cls, graphs):
        """graphs: iterable of (n, src, dst) with local ids."""
        graphs = list(graphs)
        n = [g[0] for g in graphs]
        m = [len(g[1]) for g in graphs]
        src = np.concatenate([np.asarray(g[1], np.uint32) for g in graphs]) if graphs else np.empty(0, np.uint32)
        dst = np.concatenate([np.asarray(g[2], np.uint32) for g in graphs]) if graphs else np.empty(0, np.uint32)
        return cls(n, m, src, dst)

    @property
    def handle(self):
        if not self._h:
            raise ValueError("batch already freed")
        return self._h

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.load().ursa_gpu_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def n_graphs(self) -> int:
        return int(_lib.load().ursa_gpu_batch_n_graphs(self.handle))

    def n_nodes(self) -> int:
        return int(_lib.load().ursa_gpu_batch_n_nodes(self.handle))

    def n_edges(self) -> int:
        return int(_lib.load().ursa_gpu_batch_n_edges(self.handle))

    def device_bytes(self) -> int:
        return int(_lib.load().ursa_gpu_batch_device_bytes(self.handle))

    @staticmethod
    def _p(params, damping, max_iter, tol) -> PageRankParams:
        if params is None:
            params = PageRankParams(0.85, 30, 1e-6)  # PageRankParams::default
            if damping is not None:
                params.damping = damping
            if max_iter is not None:
                params.max_iter = max_iter
            if tol is not None:
                params.tol = tol
        return params

    def run(self, params: PageRankParams | None = None, what: int = ALL, *, damping=None, max_iter=None,
            tol=None, stream: int | None = None) -> None:
        """One launch of the captured graph (synchronous unless a stream
        handle is given)."""
        p = self._p(params, damping, max_iter, tol)
        _lib.check(_lib.load().ursa_gpu_batch_run(self.handle, C.byref(p), what, stream))

    def tune(self, params: PageRankParams | None = None, what: int = ALL, **kw) -> tuple[dict, float]:
        """Autotune the bucket and tile shapes; returns (config, best ms)."""
        p = self._p(params, kw.get("damping"), kw.get("max_iter"), kw.get("tol"))
        cfg = BatchConfig()
        ms = C.c_float()
        _lib.check(_lib.load().ursa_gpu_batch_tune(self.handle, C.byref(p), what, C.byref(cfg), C.byref(ms)))
        return cfg.as_dict(), float(ms.value)

    def config(self) -> dict:
        cfg = BatchConfig()
        _lib.check(_lib.load().ursa_gpu_batch_get_config(self.handle, C.byref(cfg)))
        return cfg.as_dict()

    def set_config(self, cap, threads, tc_tile: int = 32, tc_threads: int = 256) -> None:
        cfg = BatchConfig()
        cfg.n_buckets = len(cap)
        for i, (c, t) in enumerate(zip(cap, threads)):
            cfg.cap[i] = c
            cfg.threads[i] = t
        cfg.tc_tile = tc_tile
        cfg.tc_threads = tc_threads
        _lib.check(_lib.load().ursa_gpu_batch_set_config(self.handle, C.byref(cfg)))

    def results(self) -> BatchResults:
        N, G = self.n_nodes(), self.n_graphs()
        pr = np.empty(N, np.float64)
        cc = np.empty(N, np.uint32)
        tri = np.empty(N, np.uint32)
        it = np.empty(G, np.uint32)
        de = np.empty(G, np.float64)
        _lib.check(
            _lib.load().ursa_gpu_batch_results(self.handle, pr.ctypes.data, cc.ctypes.data, tri.ctypes.data,
                                              it.ctypes.data, de.ctypes.data)
        )
        return BatchResults(pr, cc, tri, it, de, self.node_offsets)

    def device_results(self) -> tuple[int, int, int]:
        a, b, c = C.c_void_p(), C.c_void_p(), C.c_void_p()
        _lib.check(_lib.load().ursa_gpu_batch_device_results(self.handle, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value
