"""Arrow results (the ursa_gpu_*_batch entry points of include/ursa_gpu.h):
the "Arrow arrays out" half of the operator (ursa-plan/src/result.rs:144-261).

`query_batch`, `hop_batch` and `path_batch` return pyarrow RecordBatches with
the reference's schemas.  The columns are computed and id-translated on the
device and copied once into pinned host memory; the RecordBatch is imported
through the Arrow C Data Interface, so its buffers are that pinned block (no
further copy), kept alive until pyarrow releases the batch.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .topology import Direction, Topology

ALGOS = {
    "pagerank": 0,
    "connected_components": 1,
    "degree": 2,
    "triangle_count": 3,
    "clustering_coefficient": 4,
    "betweenness": 5,
    "closeness": 6,
    "label_propagation": 7,
    "louvain": 8,
}


class _Column(C.Structure):
    _fields_ = [
        ("name", C.c_char_p),
        ("algo", C.c_int),
        ("damping", C.c_double),
        ("max_iter", C.c_uint32),
        ("tol", C.c_double),
        ("strong", C.c_int),
        ("direction", C.c_int),
        ("has_sample", C.c_int),
        ("sample", C.c_double),
        ("has_seed", C.c_int),
        ("seed", C.c_uint64),
        ("weights", C.c_void_p),
        ("n_weights", C.c_uint64),
    ]


class ArrowSchema(C.Structure):
    """struct ArrowSchema of the Arrow C Data Interface."""


ArrowSchema._fields_ = [
    ("format", C.c_char_p),
    ("name", C.c_char_p),
    ("metadata", C.c_char_p),
    ("flags", C.c_int64),
    ("n_children", C.c_int64),
    ("children", C.POINTER(C.POINTER(ArrowSchema))),
    ("dictionary", C.POINTER(ArrowSchema)),
    ("release", C.c_void_p),
    ("private_data", C.c_void_p),
]


class ArrowArray(C.Structure):
    """struct ArrowArray of the Arrow C Data Interface."""


ArrowArray._fields_ = [
    ("length", C.c_int64),
    ("null_count", C.c_int64),
    ("offset", C.c_int64),
    ("n_buffers", C.c_int64),
    ("n_children", C.c_int64),
    ("buffers", C.POINTER(C.c_void_p)),
    ("children", C.POINTER(C.POINTER(ArrowArray))),
    ("dictionary", C.POINTER(ArrowArray)),
    ("release", C.c_void_p),
    ("private_data", C.c_void_p),
]


class OutputColumn:
    """OutputColumn::Algo (result.rs:28-35): a named node-valued column.

    algo: one of ALGOS; the keyword arguments are GraphAlgo's fields
    (ursa-plan/src/logical.rs:37-65); weights (one f64 per edge row) select
    the weighted form of pagerank, betweenness and closeness."""

    def __init__(self, name: str, algo: str, *, damping: float = 0.85, max_iter: int = 30, tol: float = 1e-6,
                 strong: bool = False, direction=Direction.Out, sample=None, seed=None, weights=None):
        if algo not in ALGOS:
            raise ValueError(f"unknown algorithm {algo!r}")
        self.name, self.algo = name, algo
        self.damping, self.max_iter, self.tol = float(damping), int(max_iter), float(tol)
        self.strong, self.direction = bool(strong), Direction.of(direction)
        self.sample, self.seed = sample, seed
        self.weights = None if weights is None else np.ascontiguousarray(np.asarray(weights, dtype=np.float64))

    def _struct(self) -> _Column:
        w = self.weights
        return _Column(self.name.encode(), ALGOS[self.algo], self.damping, self.max_iter, self.tol, int(self.strong),
                       int(self.direction), int(self.sample is not None), float(self.sample or 0.0),
                       int(self.seed is not None), int(self.seed or 0),
                       None if w is None else w.ctypes.data, 0 if w is None else w.size)


def _import(handle: int):
    """Exports a result and imports it into pyarrow without copying."""
    import pyarrow as pa

    L = _lib.load()
    schema, array = ArrowSchema(), ArrowArray()
    try:
        _lib.check(L.ursa_gpu_result_export(handle, C.addressof(schema), C.addressof(array)))
        return pa.RecordBatch._import_from_c(C.addressof(array), C.addressof(schema))
    finally:
        L.ursa_gpu_result_free(handle)


def _ids_handle(ids):
    return None if ids is None else ids.handle


def query_batch(topo: Topology, ids, columns):
    """query_batch (result.rs:160-168): ("id", column...) over every node.
    ids: the IdMap the topology was built from (Int64 id column), or None
    (UInt32 dense ids)."""
    cols = [c._struct() for c in columns]
    arr = (_Column * max(len(cols), 1))(*cols)
    h = C.c_void_p()
    _lib.check(_lib.load().ursa_gpu_query_batch(topo.handle, _ids_handle(ids), C.addressof(arr), len(cols),
                                                C.byref(h)))
    return _import(h.value)


def hop_batch(topo: Topology, ids, seeds, k: int, direction=Direction.Out):
    """hop_batch (result.rs:180-199): ("src", "dst") = (seed, reached)."""
    s = np.ascontiguousarray(np.asarray(seeds, dtype=np.uint32))
    h = C.c_void_p()
    _lib.check(_lib.load().ursa_gpu_hop_batch(topo.handle, _ids_handle(ids), s.ctypes.data if s.size else None,
                                              s.size, int(k), int(Direction.of(direction)), C.byref(h)))
    return _import(h.value)


def path_batch(topo: Topology, ids, source: int, target: int, direction=Direction.Out, weights=None):
    """path_batch (result.rs:216-261): ("src", "dst", "hop", "cost"), one row
    per path edge."""
    w = None if weights is None else np.ascontiguousarray(np.asarray(weights, dtype=np.float64))
    h = C.c_void_p()
    _lib.check(_lib.load().ursa_gpu_path_batch(topo.handle, _ids_handle(ids), int(source), int(target),
                                               int(Direction.of(direction)), None if w is None else w.ctypes.data,
                                               0 if w is None else w.size, C.byref(h)))
    return _import(h.value)
