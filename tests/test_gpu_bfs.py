"""BFS family on the GPU vs the oracle (ursa-core/src/algo/bfs.rs, hop.rs).

All three are exact: bfs_distances levels, k_hop pairs in the reference's
emission order (seed order, then discovery order), and shortest_path node
sequences (first-discoverer parents)."""

import numpy as np
import pytest

from cases import medium_cases, random_graph, small_cases

pytestmark = pytest.mark.gpu

DIRS = ("out", "in", "both")


def _pair(orc, n, s, d):
    from ursa_b200 import Topology

    return Topology.build(n, s, d), orc.Topology(n, s, d)


def _sources(n, k, seed):
    rng = np.random.default_rng(seed)
    return [int(x) for x in rng.integers(0, max(n, 1), k)] if n else [0]


@pytest.mark.parametrize("case", small_cases() + medium_cases(), ids=lambda c: c[0])
def test_bfs_distances_exact(orc, case):
    from ursa_b200 import algo

    _, n, s, d = case
    g, o = _pair(orc, n, s, d)
    for dirn in DIRS:
        for src in _sources(n, 3, len(s)) + [n + 5]:  # includes an out-of-range source
            assert np.array_equal(algo.bfs_distances(g, src, dirn), orc.bfs_distances(o, src, dirn)), (dirn, src)


def test_bfs_goldens():
    from ursa_b200 import Topology, algo

    t = Topology.build(5, [0, 1, 2, 1], [1, 2, 3, 4])  # bfs.rs:270-298
    assert list(algo.bfs_distances(t, 0)) == [0, 1, 2, 3, 2]
    d = algo.bfs_distances(t, 3)
    assert d[3] == 0 and d[0] == -1 and d[1] == -1
    d = algo.bfs_distances(t, 3, "both")
    assert d[0] == 3 and d[4] == 3


@pytest.mark.parametrize("case", small_cases() + medium_cases(), ids=lambda c: c[0])
def test_k_hop_exact_order(orc, case):
    from ursa_b200 import algo

    _, n, s, d = case
    g, o = _pair(orc, n, s, d)
    seeds = _sources(n, 4, 7) + [n + 3]
    if n:
        seeds.append(seeds[0])  # repeated seed emits its pairs again
    for dirn in DIRS:
        for k in (1, 2, 3):
            gs, gd = algo.k_hop(g, seeds, k, dirn)
            os_, od = orc.k_hop(o, seeds, k, dirn)
            assert np.array_equal(gs, os_) and np.array_equal(gd, od), (dirn, k)


def test_k_hop_goldens():
    from ursa_b200 import Topology, algo

    t = Topology.build(5, [0, 1, 2, 1], [1, 2, 3, 4])  # hop.rs:535-580

    def pairs(r):
        return sorted(zip(r[0].tolist(), r[1].tolist()))

    assert pairs(algo.k_hop(t, [0], 1)) == [(0, 1)]
    assert pairs(algo.k_hop(t, [0], 2)) == [(0, 1), (0, 2), (0, 4)]
    assert pairs(algo.k_hop(t, [0], 10)) == [(0, 1), (0, 2), (0, 3), (0, 4)]
    assert pairs(algo.k_hop(t, [3], 2, "in")) == [(3, 1), (3, 2)]
    assert pairs(algo.k_hop(t, [0, 2], 1)) == [(0, 1), (2, 3)]
    assert algo.k_hop(t, [99], 3)[0].size == 0
    assert algo.k_hop(t, [0], 0)[0].size == 0
    assert algo.k_hop(t, [], 2)[0].size == 0


@pytest.mark.parametrize("case", small_cases() + medium_cases(), ids=lambda c: c[0])
def test_shortest_path_exact(orc, case):
    from ursa_b200 import algo

    _, n, s, d = case
    g, o = _pair(orc, n, s, d)
    srcs = _sources(n, 3, 11)
    tgts = _sources(n, 3, 12) + [n + 1]
    for dirn in DIRS:
        for a in srcs:
            for b in tgts:
                assert algo.shortest_path(g, a, b, dirn) == orc.shortest_path(o, a, b, dirn), (dirn, a, b)


def test_shortest_path_goldens():
    from ursa_b200 import Topology, algo

    t = Topology.build(5, [0, 1, 2, 1], [1, 2, 3, 4])  # bfs.rs:300-332
    assert algo.shortest_path(t, 0, 3) == [0, 1, 2, 3]
    assert algo.shortest_path(t, 0, 4) == [0, 1, 4]
    assert algo.shortest_path(t, 2, 2) == [2]
    assert algo.shortest_path(t, 3, 0) is None
    assert algo.shortest_path(t, 0, 99) is None
    assert algo.shortest_path(t, 3, 0, "in") == [3, 2, 1, 0]
    t2 = Topology.build(4, [0, 1, 0], [1, 3, 3])  # bfs.rs:340
    assert algo.shortest_path(t2, 0, 3) == [0, 3]


def test_bfs_rmat20_sources(orc):
    """R-MAT-20 with the C1-style seeded source choice (sample_indices over
    nodes with out-degree > 0): distances exact from 8 sources, both
    traversal modes exercised (the frontier grows past the switch point)."""
    from ursa_b200 import algo, gen

    n, s, d = gen.rmat(20, 16, 1)
    g, o = _pair(orc, n, s, d)
    outdeg = np.bincount(s, minlength=n)
    cand = np.nonzero(outdeg > 0)[0]
    pick = orc.sample_indices(cand.size, 8, 1)
    for i in pick:
        src = int(cand[i])
        for dirn in ("out", "both"):
            assert np.array_equal(algo.bfs_distances(g, src, dirn), orc.bfs_distances(o, src, dirn))


@pytest.mark.parametrize("direction", DIRS)
def test_bfs_distances_multi(orc, direction):
    """Many sources in one traversal: each row equals the oracle's
    bfs_distances; 300 sources fill a 256-wide batch and a partial one, and
    an unknown source gives a row of -1."""
    from ursa_b200 import Topology, algo

    n, s, d = random_graph(1500, 6000, 17)
    g, o = Topology.build(n, s, d), orc.Topology(n, s, d)
    srcs = list(range(0, 1500, 5)) + [n + 3]
    got = algo.bfs_distances_multi(g, srcs, direction)
    assert got.shape == (len(srcs), n)
    for i, x in enumerate(srcs):
        assert np.array_equal(got[i], orc.bfs_distances(o, x, direction)), (direction, x)


@pytest.mark.parametrize("direction", DIRS)
def test_bfs_distances_multi_hubs(orc, direction):
    """Hubs in every direction: node 0 has 2,499 in-edges, node 1 has 1,800
    out-edges (split scans for out, in and both traversals)."""
    from ursa_b200 import Topology, algo

    rng = np.random.default_rng(23)
    s = list(range(2, 2500)) + [1] * 1800 + rng.integers(2, 2600, 4000).tolist()
    d = [0] * 2498 + list(range(700, 2500)) + rng.integers(2, 2600, 4000).tolist()
    n = 2600
    g, o = Topology.build(n, s, d), orc.Topology(n, s, d)
    srcs = list(range(0, n, 7))
    got = algo.bfs_distances_multi(g, srcs, direction)
    for i, x in enumerate(srcs):
        assert np.array_equal(got[i], orc.bfs_distances(o, x, direction)), (direction, x)
