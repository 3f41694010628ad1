"""Host mirror of ursa-core's Topology (ursa-core/src/topology.rs:251-431).

`Topology.build(n_nodes, src_dense, dst_dense)` uploads the dense endpoint
columns and builds the out-CSR on the device; `out()`, `incoming()` and
`undirected()` download the pub fields on demand (the transpose and the
undirected CSR are built lazily on the device and cached, like the
reference's OnceLock fields).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from enum import IntEnum

import numpy as np

from . import _lib


class Direction(IntEnum):
    """Direction (topology.rs:28-32)."""

    Out = 0
    In = 1
    Both = 2

    @classmethod
    def of(cls, d) -> "Direction":
        if isinstance(d, Direction):
            return d
        if isinstance(d, str):
            return {"out": cls.Out, "in": cls.In, "both": cls.Both}[d.lower()]
        return cls(int(d))


@dataclass
class Adjacency:
    """One direction's CSR (topology.rs:36-47)."""

    offsets: np.ndarray  # u64, n + 1
    targets: np.ndarray  # u32, m
    edge_ids: np.ndarray  # u32, m

    def neighbors(self, u: int) -> np.ndarray:
        return self.targets[self.offsets[u] : self.offsets[u + 1]]

    def edge_ids_of(self, u: int) -> np.ndarray:
        return self.edge_ids[self.offsets[u] : self.offsets[u + 1]]

    def degree(self, u: int) -> int:
        return int(self.offsets[u + 1] - self.offsets[u])


@dataclass
class UndirectedCsr:
    """Sorted, deduplicated undirected adjacency (topology.rs:222-244)."""

    offsets: np.ndarray  # u64, n + 1
    targets: np.ndarray  # u32

    def neighbors(self, u: int) -> np.ndarray:
        return self.targets[self.offsets[u] : self.offsets[u + 1]]

    def degree(self, u: int) -> int:
        return int(self.offsets[u + 1] - self.offsets[u])


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


class Topology:
    """Device-resident topology; freed when the object is dropped."""

    def __init__(self, handle: int, n: int, m: int):
        self._h = handle
        self._n = n
        self._m = m

    @classmethod
    def build(cls, n_nodes: int, src_dense, dst_dense) -> "Topology":
        """Topology::build (topology.rs:276-298)."""
        src, dst = _u32(src_dense), _u32(dst_dense)
        if src.shape != dst.shape:
            raise ValueError("src/dst length mismatch")
        L = _lib.load()
        h = C.c_void_p()
        _lib.check(L.ursa_gpu_topo_build(int(n_nodes), src.ctypes.data, dst.ctypes.data, src.size, C.byref(h)))
        return cls(h.value, int(n_nodes), int(src.size))

    @classmethod
    def build_device(cls, n_nodes: int, d_src, d_dst, stream: int = 0) -> "Topology":
        """Build from device-resident u32 endpoint tensors (torch, contiguous)."""
        if d_src.numel() != d_dst.numel():
            raise ValueError("src/dst length mismatch")
        L = _lib.load()
        h = C.c_void_p()
        _lib.check(
            L.ursa_gpu_topo_build_device(
                int(n_nodes), d_src.data_ptr(), d_dst.data_ptr(), d_src.numel(), stream or None, C.byref(h)
            )
        )
        return cls(h.value, int(n_nodes), int(d_src.numel()))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                _lib.load().ursa_gpu_topo_free(h)
            except Exception:
                pass
            self._h = None

    def free(self) -> None:
        self.__del__()

    @property
    def handle(self) -> int:
        return self._h

    def n_nodes(self) -> int:
        return self._n

    def n_edges(self) -> int:
        return self._m

    def _adj(self, d: int) -> Adjacency:
        off = np.empty(self._n + 1, np.uint64)
        tg = np.empty(self._m, np.uint32)
        eid = np.empty(self._m, np.uint32)
        _lib.check(_lib.load().ursa_gpu_topo_adjacency(self._h, d, off.ctypes.data, tg.ctypes.data, eid.ctypes.data))
        return Adjacency(off, tg, eid)

    def out(self) -> Adjacency:
        """Topology::out (topology.rs:335-337)."""
        return self._adj(0)

    def incoming(self) -> Adjacency:
        """Topology::incoming (topology.rs:343-348)."""
        return self._adj(1)

    def undirected(self) -> UndirectedCsr:
        """Topology::undirected (topology.rs:353-355)."""
        L = _lib.load()
        ln = C.c_uint64()
        _lib.check(L.ursa_gpu_topo_undirected_len(self._h, C.byref(ln)))
        off = np.empty(self._n + 1, np.uint64)
        tg = np.empty(ln.value, np.uint32)
        _lib.check(L.ursa_gpu_topo_undirected(self._h, off.ctypes.data, tg.ctypes.data))
        return UndirectedCsr(off, tg)

    def prepare(self, transpose: bool = True, undirected: bool = False) -> None:
        what = (1 if transpose else 0) | (2 if undirected else 0)
        _lib.check(_lib.load().ursa_gpu_topo_prepare(self._h, what))

    def device_bytes(self) -> int:
        return int(_lib.load().ursa_gpu_topo_device_bytes(self._h))
