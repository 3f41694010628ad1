"""ursa_b200 -- B200 (sm_100a) implementation of ursa-core's CSR topology and
graph kernels behind a C ABI (include/ursa_gpu.h).

The Python modules mirror the reference's Rust API for tests and tools:
`Topology` (ursa-core/src/topology.rs) and the kernels of ursa-core/src/algo.
"""

from ._lib import PageRankParams, PageRankStats, UrsaGpuError  # noqa: F401
from .topology import Adjacency, Direction, Topology, UndirectedCsr  # noqa: F401
from . import algo  # noqa: F401

__all__ = [
    "Adjacency",
    "Direction",
    "PageRankParams",
    "PageRankStats",
    "Topology",
    "UndirectedCsr",
    "UrsaGpuError",
    "algo",
]
