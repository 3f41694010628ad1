"""Node-id interning on the device (the ursa_gpu_idmap_* entry points of
include/ursa_gpu.h): IdMap for Int64 ids (ursa-core/src/id_map.rs:197-440).

`IdMap.from_edge_batches(chunks)` interns the edges' user ids in first-seen
order (per edge, src before dst, chunk after chunk) exactly as the reference
does, and `topology()` builds the Topology from the device-resident dense
columns without a host round trip.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .topology import Topology


def _i64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64))


class IdMap:
    def __init__(self, handle: int):
        self._h = handle

    @classmethod
    def from_edge_batches(cls, chunks) -> "IdMap":
        """chunks: iterable of (src, dst) Int64 columns of equal length
        (IdMap::from_edge_batches, id_map.rs:220-292)."""
        chunks = [(_i64(s), _i64(d)) for s, d in chunks]
        for s, d in chunks:
            if s.shape != d.shape:
                raise ValueError("src and dst columns must have the same length")
        n = len(chunks)
        srcp = (C.c_void_p * max(n, 1))(*[s.ctypes.data for s, _ in chunks])
        dstp = (C.c_void_p * max(n, 1))(*[d.ctypes.data for _, d in chunks])
        lens = np.array([s.size for s, _ in chunks] or [0], np.uint64)
        h = C.c_void_p()
        _lib.check(_lib.load().ursa_gpu_idmap_build(n, C.cast(srcp, C.c_void_p), C.cast(dstp, C.c_void_p),
                                                   lens.ctypes.data, C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_edge_arrays(cls, src, dst) -> "IdMap":
        """IdMap::from_edge_arrays (id_map.rs:197-205)."""
        return cls.from_edge_batches([(src, dst)])

    @property
    def handle(self) -> int:
        if not self._h:
            raise ValueError("idmap already freed")
        return self._h

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.load().ursa_gpu_idmap_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self) -> int:
        return int(_lib.load().ursa_gpu_idmap_len(self.handle))

    def n_edges(self) -> int:
        return int(_lib.load().ursa_gpu_idmap_n_edges(self.handle))

    def user_id_array(self) -> np.ndarray:
        """IdMap::user_id_array (id_map.rs:359): user ids in dense order."""
        out = np.empty(len(self), np.int64)
        _lib.check(_lib.load().ursa_gpu_idmap_user_ids(self.handle, out.ctypes.data))
        return out

    def dense_edges(self) -> tuple[np.ndarray, np.ndarray]:
        m = self.n_edges()
        s = np.empty(m, np.uint32)
        d = np.empty(m, np.uint32)
        _lib.check(_lib.load().ursa_gpu_idmap_dense_edges(self.handle, s.ctypes.data, d.ctypes.data))
        return s, d

    def topology(self) -> Topology:
        """Topology::build(len, dense src, dense dst) from the device columns."""
        h = C.c_void_p()
        _lib.check(_lib.load().ursa_gpu_idmap_topology(self.handle, C.byref(h)))
        return Topology(h.value, len(self), self.n_edges())

    def gather_user(self, dense) -> np.ndarray:
        """IdMap::gather_user (id_map.rs:381-398)."""
        d = np.ascontiguousarray(np.asarray(dense, dtype=np.uint32))
        out = np.empty(d.size, np.int64)
        _lib.check(_lib.load().ursa_gpu_idmap_gather_user(self.handle, d.ctypes.data, d.size, out.ctypes.data))
        return out

    def dense_from_array(self, ids) -> list:
        """IdMap::dense_from_array (id_map.rs:402-440) for Int64 ids: a list of
        dense ids, None where the id is not in the map."""
        a = _i64(ids)
        dense = np.empty(a.size, np.uint32)
        found = np.empty(a.size, np.uint8)
        if a.size:
            _lib.check(_lib.load().ursa_gpu_idmap_lookup(self.handle, a.ctypes.data, a.size, dense.ctypes.data,
                                                         found.ctypes.data))
        return [int(x) if f else None for x, f in zip(dense, found)]
