"""Parity of the device CSR build, transpose, undirected CSR and degree with
the oracle (ursa-core/src/topology.rs, algo/degree.rs): byte-identical."""

import numpy as np
import pytest

from cases import medium_cases, small_cases

pytestmark = pytest.mark.gpu


def _pair(orc, n, s, d):
    from ursa_b200 import Topology

    return Topology.build(n, s, d), orc.Topology(n, s, d)


def _assert_same_csr(g, o):
    go, gt, ge = g.offsets, g.targets, g.edge_ids
    oo, ot, oe = o
    assert np.array_equal(go, oo)
    assert np.array_equal(gt, ot)
    assert np.array_equal(ge, oe)


@pytest.mark.parametrize("case", small_cases() + medium_cases(), ids=lambda c: c[0])
def test_csr_transpose_undirected_degree(orc, case):
    from ursa_b200 import algo

    _, n, s, d = case
    g, o = _pair(orc, n, s, d)
    _assert_same_csr(g.out(), o.csr("out"))
    _assert_same_csr(g.incoming(), o.csr("in"))
    gu = g.undirected()
    ou_off, ou_tg = o.undirected()
    assert np.array_equal(gu.offsets, ou_off) and np.array_equal(gu.targets, ou_tg)
    for dirn in ("out", "in", "both"):
        assert np.array_equal(algo.degree(g, dirn), orc.degree(o, dirn))


def test_rmat16_full(orc):
    from ursa_b200 import Topology, gen

    n, s, d = gen.rmat(16, 16, 1)
    g, o = Topology.build(n, s, d), orc.Topology(n, s, d)
    _assert_same_csr(g.out(), o.csr("out"))
    _assert_same_csr(g.incoming(), o.csr("in"))
    gu = g.undirected()
    ou = o.undirected()
    assert np.array_equal(gu.offsets, ou[0]) and np.array_equal(gu.targets, ou[1])


def test_rmat22_build_properties():
    """Full-size R-MAT-22: the CSR is a stable grouping of the input rows
    (size-independent checks: offsets monotone, every row placed once, each
    segment's rows ascending, targets match the rows' endpoints)."""
    from ursa_b200 import Topology, gen

    n, s, d = gen.rmat(22, 16, 2)
    g = Topology.build(n, s, d)
    for adj, key, other in ((g.out(), s, d), (g.incoming(), d, s)):
        off, tg, eid = adj.offsets, adj.targets, adj.edge_ids
        assert off[0] == 0 and off[-1] == s.size and np.all(np.diff(off.astype(np.int64)) >= 0)
        assert np.array_equal(np.sort(eid), np.arange(s.size, dtype=np.uint32))
        assert np.array_equal(tg, other[eid])
        owner = np.repeat(np.arange(n, dtype=np.uint32), np.diff(off.astype(np.int64)))
        assert np.array_equal(key[eid], owner)
        # stable: within each segment edge ids ascend
        step = np.diff(eid.astype(np.int64))
        same = owner[1:] == owner[:-1]
        assert np.all(step[same] > 0)


def test_invalid_endpoints_rejected():
    from ursa_b200 import Topology, UrsaGpuError

    with pytest.raises(UrsaGpuError, match="out of range"):
        Topology.build(3, [0, 5], [1, 2])


def test_build_twice_identical():
    from ursa_b200 import Topology
    from cases import random_graph

    n, s, d = random_graph(10_000, 200_000, 11)
    a = Topology.build(n, s, d).incoming()
    b = Topology.build(n, s, d).incoming()
    assert np.array_equal(a.targets, b.targets) and np.array_equal(a.edge_ids, b.edge_ids)


def test_pool_keeps_freed_blocks_until_released():
    """Freed device buffers stay cached in the pool (the next build maps
    nothing new) until ursa_gpu_pool_release returns them to the driver."""
    import ursa_b200
    from ursa_b200 import Topology, gen

    import torch

    n, s, d = gen.rmat(16, 16, 9)
    g = Topology.build(n, s, d)
    g.prepare(transpose=True)
    g.free()
    torch.cuda.synchronize()  # the frees are stream-ordered
    before = ursa_b200.pool_cached_bytes(0)
    assert before >= 8 * s.size  # at least the freed CSR arrays
    ursa_b200.pool_release(0)
    # chunks that still hold live buffers stay reserved; everything else went back
    assert ursa_b200.pool_cached_bytes(0) < before
