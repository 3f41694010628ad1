"""ctypes binding of libursa_gpu.so (the C ABI in include/ursa_gpu.h).

The library is loaded from this package directory only.  If it is missing,
importing the kernels raises: there is no CPU fallback on the product path.
"""

from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
GPU_SO = os.path.join(PKG, "libursa_gpu.so")

OK, EINVAL, ENOMEM, ECUDA, ETIMEOUT, ETRUNC, ENODEV, ECANCELED = range(8)
_STATUS = {
    EINVAL: "EINVAL",
    ENOMEM: "ENOMEM",
    ECUDA: "ECUDA",
    ETIMEOUT: "ETIMEOUT",
    ETRUNC: "ETRUNC",
    ENODEV: "ENODEV",
    ECANCELED: "ECANCELED",
}


class UrsaGpuError(RuntimeError):
    """A non-OK status from the C ABI (the Rust shim would panic! here)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS.get(status, status)}: {message}")
        self.status = status


class PageRankParams(C.Structure):
    """PageRankParams (ursa-core/src/algo/pagerank.rs:22-36)."""

    _fields_ = [("damping", C.c_double), ("max_iter", C.c_uint32), ("tol", C.c_double)]


class PageRankStats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("last_delta", C.c_double), ("device_ms", C.c_double)]


class BatchConfig(C.Structure):
    """ursa_gpu_batch_config: bucket capacities (nodes) and CTA size per
    bucket, and the triangle kernel's vertices per warp unit and CTA size."""

    _fields_ = [
        ("n_buckets", C.c_uint32),
        ("cap", C.c_uint32 * 3),
        ("threads", C.c_uint32 * 3),
        ("tc_tile", C.c_uint32),
        ("tc_threads", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        nb = self.n_buckets
        return {
            "n_buckets": nb,
            "cap": list(self.cap)[:nb],
            "threads": list(self.threads)[:nb],
            "tc_tile": self.tc_tile,
            "tc_threads": self.tc_threads,
        }


BATCH_PAGERANK, BATCH_COMPONENTS, BATCH_TRIANGLES = 1, 2, 4

QUERY_SHORTEST_PATH, QUERY_HOP, QUERY_PAGERANK, QUERY_BFS = 1, 2, 3, 4


class ServerConfig(C.Structure):
    _fields_ = [
        ("path_lanes", C.c_uint32),
        ("path_slots", C.c_uint32),
        ("hop_lanes", C.c_uint32),
        ("hop_slots", C.c_uint32),
        ("pr_lanes", C.c_uint32),
        ("pr_slots", C.c_uint32),
        ("pr_max_nodes", C.c_uint64),
        ("hbm_reserve_bytes", C.c_uint64),
        ("upload_budget_bytes", C.c_uint64),
        ("bfs_lanes", C.c_uint32),
        ("bfs_slots", C.c_uint32),
        ("heartbeat_limit_ns", C.c_uint64),
        ("heartbeat_period_us", C.c_uint64),
    ]


class Query(C.Structure):
    _fields_ = [
        ("type", C.c_uint32),
        ("graph", C.c_uint32),
        ("source", C.c_uint32),
        ("target", C.c_uint32),
        ("k", C.c_uint32),
        ("pr", PageRankParams),
        ("direction", C.c_uint32),
    ]


class QueryInfo(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("type", C.c_uint32),
        ("result_len", C.c_int64),
        ("iterations", C.c_uint32),
        ("last_delta", C.c_double),
        ("edges", C.c_uint64),
        ("submit_us", C.c_double),
        ("launch_us", C.c_double),
        ("done_us", C.c_double),
    ]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("submitted", "completed", "launches", "uploads_admitted",
                                           "uploads_rejected", "uploads_live", "upload_bytes", "pending",
                                           "wait_expiries")]

# Every exported symbol with its (restype, argtypes).
P, u32, u64, i32, i64, f64 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_int64, C.c_double
SIGNATURES = {
    "ursa_gpu_last_error": (C.c_char_p, []),
    "ursa_gpu_version": (i32, []),
    "ursa_gpu_launch_count": (u64, []),
    "ursa_gpu_set_device": (i32, [i32]),
    "ursa_gpu_thread_stream": (i32, [i32, P]),
    "ursa_gpu_topo_build": (i32, [u64, P, P, u64, C.POINTER(P)]),
    "ursa_gpu_topo_build_device": (i32, [u64, P, P, u64, P, C.POINTER(P)]),
    "ursa_gpu_topo_free": (None, [P]),
    "ursa_gpu_topo_n_nodes": (u64, [P]),
    "ursa_gpu_topo_n_edges": (u64, [P]),
    "ursa_gpu_topo_adjacency": (i32, [P, i32, P, P, P]),
    "ursa_gpu_topo_undirected_len": (i32, [P, C.POINTER(u64)]),
    "ursa_gpu_topo_undirected": (i32, [P, P, P]),
    "ursa_gpu_topo_prepare": (i32, [P, i32]),
    "ursa_gpu_topo_device_bytes": (u64, [P]),
    "ursa_gpu_degree": (i32, [P, i32, P]),
    "ursa_gpu_pagerank": (i32, [P, C.POINTER(PageRankParams), P, C.POINTER(PageRankStats)]),
    "ursa_gpu_pagerank_device": (i32, [P, C.POINTER(PageRankParams), P, P, C.POINTER(PageRankStats)]),
    "ursa_gpu_pagerank_weighted": (
        i32,
        [P, P, u64, C.POINTER(PageRankParams), P, C.POINTER(PageRankStats)],
    ),
    "ursa_gpu_bfs_distances": (i32, [P, u32, i32, P]),
    "ursa_gpu_bfs_distances_multi": (i32, [P, P, u64, i32, P]),
    "ursa_gpu_shortest_path": (i32, [P, u32, u32, i32, P, u64, C.POINTER(i64)]),
    "ursa_gpu_pool_cached_bytes": (i32, [i32, C.POINTER(u64)]),
    "ursa_gpu_pool_release": (i32, [i32]),
    "ursa_gpu_shortest_path_bidirectional": (i32, [P, u32, u32, P, u64, C.POINTER(i64)]),
    "ursa_gpu_dijkstra_distances": (i32, [P, P, u64, u32, i32, P]),
    "ursa_gpu_shortest_path_weighted_with_cost": (
        i32,
        [P, P, u64, u32, u32, i32, P, P, u64, C.POINTER(i64)],
    ),
    "ursa_gpu_k_hop": (i32, [P, P, u64, u32, i32, C.POINTER(P)]),
    "ursa_gpu_pairs_len": (u64, [P]),
    "ursa_gpu_pairs_copy": (i32, [P, P, P]),
    "ursa_gpu_pairs_free": (None, [P]),
    "ursa_gpu_connected_components_weak": (i32, [P, P]),
    "ursa_gpu_connected_components_weak_noalloc": (i32, [P, P, P]),
    "ursa_gpu_triangle_count": (i32, [P, P]),
    "ursa_gpu_clustering_coefficient": (i32, [P, P]),
    "ursa_gpu_betweenness": (i32, [P, i32, f64, i32, u64, P]),
    "ursa_gpu_betweenness_weighted": (i32, [P, P, u64, i32, f64, i32, u64, P]),
    "ursa_gpu_batch_build": (i32, [u64, P, P, P, P, C.POINTER(P)]),
    "ursa_gpu_batch_free": (None, [P]),
    "ursa_gpu_batch_n_graphs": (u64, [P]),
    "ursa_gpu_batch_n_nodes": (u64, [P]),
    "ursa_gpu_batch_n_edges": (u64, [P]),
    "ursa_gpu_batch_device_bytes": (u64, [P]),
    "ursa_gpu_batch_run": (i32, [P, C.POINTER(PageRankParams), u32, P]),
    "ursa_gpu_batch_tune": (
        i32,
        [P, C.POINTER(PageRankParams), u32, C.POINTER(BatchConfig), C.POINTER(C.c_float)],
    ),
    "ursa_gpu_batch_set_config": (i32, [P, C.POINTER(BatchConfig)]),
    "ursa_gpu_batch_get_config": (i32, [P, C.POINTER(BatchConfig)]),
    "ursa_gpu_batch_results": (i32, [P, P, P, P, P, P]),
    "ursa_gpu_batch_device_results": (i32, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P)]),
    "ursa_gpu_closeness": (i32, [P, P]),
    "ursa_gpu_closeness_device": (i32, [P, P, P, C.POINTER(C.c_float)]),
    "ursa_gpu_closeness_weighted": (i32, [P, P, u64, P]),
    "ursa_gpu_avg_path_length": (i32, [P, i32, f64, C.POINTER(f64)]),
    "ursa_gpu_diameter": (i32, [P, i32, C.POINTER(i64)]),
    "ursa_gpu_idmap_build": (i32, [u64, P, P, P, C.POINTER(P)]),
    "ursa_gpu_idmap_free": (None, [P]),
    "ursa_gpu_idmap_len": (u64, [P]),
    "ursa_gpu_idmap_n_edges": (u64, [P]),
    "ursa_gpu_idmap_user_ids": (i32, [P, P]),
    "ursa_gpu_idmap_dense_edges": (i32, [P, P, P]),
    "ursa_gpu_idmap_topology": (i32, [P, C.POINTER(P)]),
    "ursa_gpu_idmap_gather_user": (i32, [P, P, u64, P]),
    "ursa_gpu_query_batch": (i32, [P, P, P, u64, P]),
    "ursa_gpu_hop_batch": (i32, [P, P, P, u64, u32, i32, P]),
    "ursa_gpu_path_batch": (i32, [P, P, u32, u32, i32, P, u64, P]),
    "ursa_gpu_result_num_rows": (u64, [P]),
    "ursa_gpu_result_num_columns": (u64, [P]),
    "ursa_gpu_result_export": (i32, [P, P, P]),
    "ursa_gpu_result_free": (None, [P]),
    "ursa_gpu_idmap_lookup": (i32, [P, P, u64, P, P]),
    "ursa_gpu_server_create": (i32, [P, C.POINTER(ServerConfig), C.POINTER(P)]),
    "ursa_gpu_server_destroy": (None, [P]),
    "ursa_gpu_server_upload": (i32, [P, u64, P, P, u64, C.POINTER(u32)]),
    "ursa_gpu_server_release": (i32, [P, u32]),
    "ursa_gpu_server_submit": (i32, [P, C.POINTER(Query), C.POINTER(u64)]),
    "ursa_gpu_server_cancel": (i32, [P, u64]),
    "ursa_gpu_server_wait": (i32, [P, u64, u64, C.POINTER(QueryInfo)]),
    "ursa_gpu_server_poll": (i32, [P, P, u64, C.POINTER(u64)]),
    "ursa_gpu_server_result": (i32, [P, u64, C.POINTER(QueryInfo), P, u64]),
    "ursa_gpu_server_get_stats": (i32, [P, C.POINTER(ServerStats)]),
}

_lib = None


def load():
    """Load (once) and type the in-tree libursa_gpu.so."""
    global _lib
    if _lib is None:
        if not os.path.exists(GPU_SO):
            raise ImportError(
                f"{GPU_SO} is missing: build it with `python -m ursa_b200.build` "
                "(the GPU kernels have no CPU fallback)"
            )
        L = C.CDLL(GPU_SO)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != OK:
        raise UrsaGpuError(status, load().ursa_gpu_last_error().decode(errors="replace"))
