"""The serving loop (the ursa_gpu_server_* entry points of include/ursa_gpu.h).

A Server keeps a resident Topology (shortest_path, hop and bfs queries) and
uploaded small graphs (pagerank queries) on the device and runs submitted
queries with continuous batching.  Query meanings follow the reference's
kernels: shortest_path (ursa-core/src/algo/bfs.rs:48-102), k_hop from one
seed (algo/hop.rs:52-130), bfs_distances (algo/bfs.rs:18-42) and pagerank
(algo/pagerank.rs:98-124).
"""

from __future__ import annotations

import atexit
import ctypes as C
import weakref
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (QUERY_BFS, QUERY_HOP, QUERY_PAGERANK, QUERY_SHORTEST_PATH, PageRankParams, Query, QueryInfo,
                   ServerConfig)

__all__ = ["Server", "Completed", "QUERY_SHORTEST_PATH", "QUERY_HOP", "QUERY_PAGERANK", "QUERY_BFS"]

# Servers still open at interpreter exit are closed before the CUDA runtime
# shuts down (a server's scheduler thread and resident kernels must not
# outlive it).
_open_servers: "weakref.WeakSet[Server]" = weakref.WeakSet()


@atexit.register
def _close_open_servers() -> None:
    for srv in list(_open_servers):
        try:
            srv.close()
        except Exception:
            pass


@dataclass
class Completed:
    ticket: int
    status: int
    type: int
    result: np.ndarray | None  # path / reached nodes (u32), distances (i32) or ranks (f64); None: no path
    iterations: int
    last_delta: float
    edges: int
    submit_us: float
    launch_us: float
    done_us: float

    @property
    def latency_us(self) -> float:
        return self.done_us - self.submit_us


class Server:
    def __init__(self, resident=None, *, path_lanes=4, path_slots=8, hop_lanes=4, hop_slots=8, pr_lanes=2,
                 pr_slots=32, pr_max_nodes=65536, hbm_reserve_bytes=8 << 30, upload_budget_bytes=0,
                 bfs_lanes=0, bfs_slots=16, heartbeat_limit_ns=0, heartbeat_period_us=0):
        cfg = ServerConfig(path_lanes, path_slots, hop_lanes, hop_slots, pr_lanes, pr_slots, pr_max_nodes,
                           hbm_reserve_bytes, upload_budget_bytes, bfs_lanes, bfs_slots, heartbeat_limit_ns,
                           heartbeat_period_us)
        h = C.c_void_p()
        self._resident = resident  # kept alive for the server's lifetime
        _lib.check(_lib.load().ursa_gpu_server_create(resident.handle if resident is not None else None,
                                                      C.byref(cfg), C.byref(h)))
        self._h = h
        _open_servers.add(self)

    @property
    def handle(self):
        if not self._h:
            raise ValueError("server already destroyed")
        return self._h

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.load().ursa_gpu_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- uploads
    def upload(self, n_nodes: int, src, dst) -> int:
        src = np.ascontiguousarray(np.asarray(src, dtype=np.uint32))
        dst = np.ascontiguousarray(np.asarray(dst, dtype=np.uint32))
        gid = C.c_uint32()
        _lib.check(_lib.load().ursa_gpu_server_upload(self.handle, n_nodes, src.ctypes.data, dst.ctypes.data,
                                                      src.size, C.byref(gid)))
        return gid.value

    def release(self, graph_id: int) -> None:
        _lib.check(_lib.load().ursa_gpu_server_release(self.handle, graph_id))

    # ---- queries
    def _submit(self, q: Query) -> int:
        t = C.c_uint64()
        _lib.check(_lib.load().ursa_gpu_server_submit(self.handle, C.byref(q), C.byref(t)))
        return t.value

    def shortest_path(self, source: int, target: int) -> int:
        return self._submit(Query(QUERY_SHORTEST_PATH, 0, source, target, 0, PageRankParams(0.85, 30, 1e-6)))

    def hop(self, seed: int, k: int = 2) -> int:
        return self._submit(Query(QUERY_HOP, 0, seed, 0, k, PageRankParams(0.85, 30, 1e-6)))

    def pagerank(self, graph_id: int, damping=0.85, max_iter=30, tol=1e-6) -> int:
        return self._submit(Query(QUERY_PAGERANK, graph_id, 0, 0, 0, PageRankParams(damping, max_iter, tol)))

    def bfs(self, source: int, direction: int = 0) -> int:
        """bfs_distances(source, direction): 0 = Out, 1 = In, 2 = Both."""
        return self._submit(Query(QUERY_BFS, 0, source, 0, 0, PageRankParams(0.85, 30, 1e-6), direction))

    def cancel(self, ticket: int) -> None:
        _lib.check(_lib.load().ursa_gpu_server_cancel(self.handle, ticket))

    def wait(self, ticket: int, timeout_s: float = 60.0) -> QueryInfo:
        info = QueryInfo()
        _lib.check(_lib.load().ursa_gpu_server_wait(self.handle, ticket, int(timeout_s * 1e6), C.byref(info)))
        return info

    def poll(self, cap: int = 4096) -> list[int]:
        buf = np.empty(cap, np.uint64)
        n = C.c_uint64()
        _lib.check(_lib.load().ursa_gpu_server_poll(self.handle, buf.ctypes.data, cap, C.byref(n)))
        return [int(x) for x in buf[: n.value]]

    def result(self, ticket: int, timeout_s: float = 60.0, out: np.ndarray | None = None) -> Completed:
        """Waits for the query and takes its result (the ticket is then forgotten).
        `out` (optional): a contiguous array of the result's dtype with at least
        info.result_len elements to receive it (e.g. one reused buffer for bfs
        answers, n i32 each); the result is then a view of its first
        result_len elements."""
        info = self.wait(ticket, timeout_s)
        L = _lib.load()
        n = max(int(info.result_len), 0)
        dtype = np.float64 if info.type == QUERY_PAGERANK else (np.int32 if info.type == QUERY_BFS else np.uint32)
        if out is not None and out.dtype == dtype and out.flags.c_contiguous and out.size >= n:
            out = out[:n]
        else:
            out = np.empty(n, dtype)
        _lib.check(L.ursa_gpu_server_result(self.handle, ticket, C.byref(info), out.ctypes.data if n else None, n))
        res = out
        if info.type == QUERY_SHORTEST_PATH and info.result_len < 0:
            res = None
        return Completed(ticket, info.status, info.type, res, info.iterations, info.last_delta, info.edges,
                         info.submit_us, info.launch_us, info.done_us)

    def stats(self) -> dict:
        st = _lib.ServerStats()
        _lib.check(_lib.load().ursa_gpu_server_get_stats(self.handle, C.byref(st)))
        return {k: int(getattr(st, k)) for k, _ in st._fields_}
