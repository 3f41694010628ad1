"""ursa_b200 -- B200 (sm_100a) implementation of ursa-core's CSR topology and
graph kernels behind a C ABI (include/ursa_gpu.h).

The Python modules mirror the reference's Rust API for tests and tools:
`Topology` (ursa-core/src/topology.rs) and the kernels of ursa-core/src/algo.
"""

from ._lib import PageRankParams, PageRankStats, UrsaGpuError  # noqa: F401
from .topology import Adjacency, Direction, Topology, UndirectedCsr  # noqa: F401
from . import algo  # noqa: F401


def pool_cached_bytes(device: int = 0) -> int:
    """Device bytes the library's memory pool holds but no buffer uses."""
    import ctypes as C

    v = C.c_uint64()
    _lib.check(_lib.load().ursa_gpu_pool_cached_bytes(device, C.byref(v)))
    return int(v.value)


def pool_release(device: int = 0) -> None:
    """Returns the pool's cached device memory to the driver."""
    _lib.check(_lib.load().ursa_gpu_pool_release(device))


from . import _lib  # noqa: E402

__all__ = [
    "pool_cached_bytes",
    "pool_release",
    "Adjacency",
    "Direction",
    "PageRankParams",
    "PageRankStats",
    "Topology",
    "UndirectedCsr",
    "UrsaGpuError",
    "algo",
]
