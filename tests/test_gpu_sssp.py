"""Weighted shortest paths on the GPU vs the oracle (ursa-core/src/algo/bfs.rs:
126-259).  Distances are bit-exact (the same left-to-right f64 path sums as
Dijkstra); paths are identical with positive weights (parent = the first
settled tight predecessor) and their costs are the settled distances."""

import math

import numpy as np
import pytest

from cases import medium_cases, small_cases

pytestmark = pytest.mark.gpu

DIRS = ("out", "in", "both")


def _pair(orc, n, s, d):
    from ursa_b200 import Topology

    return Topology.build(n, s, d), orc.Topology(n, s, d)


def _weights(m, seed, lo=1.0, hi=10.0):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, m).astype(np.float32).astype(np.float64)


def _nodes(n, k, seed):
    rng = np.random.default_rng(seed)
    return [int(x) for x in rng.integers(0, max(n, 1), k)]


@pytest.mark.parametrize("case", small_cases() + medium_cases(), ids=lambda c: c[0])
def test_dijkstra_distances_exact(orc, case):
    from ursa_b200 import algo

    _, n, s, d = case
    g, o = _pair(orc, n, s, d)
    w = _weights(len(s), 3)
    for dirn in DIRS:
        for src in _nodes(n, 2, 5) + [n + 2]:
            got = algo.dijkstra_distances(g, w, src, dirn)
            ref = orc.dijkstra_distances(o, w, src, dirn)
            assert np.array_equal(got.view(np.uint64), ref.view(np.uint64)), (dirn, src)


@pytest.mark.parametrize("case", small_cases() + medium_cases(), ids=lambda c: c[0])
def test_weighted_path_exact(orc, case):
    from ursa_b200 import algo

    _, n, s, d = case
    g, o = _pair(orc, n, s, d)
    w = _weights(len(s), 4)
    for dirn in DIRS:
        for a in _nodes(n, 2, 6):
            for b in _nodes(n, 3, 7) + [n + 1]:
                got = algo.shortest_path_weighted_with_cost(g, w, a, b, dirn)
                ref = orc.shortest_path_weighted_with_cost(o, w, a, b, dirn)
                assert got == ref, (dirn, a, b)


def test_weighted_goldens():
    from ursa_b200 import Topology, algo

    t = Topology.build(4, [0, 1, 0], [1, 3, 3])  # bfs.rs:334-387
    assert algo.shortest_path_weighted(t, [1.0, 1.0, 5.0], 0, 3) == [0, 1, 3]
    assert algo.shortest_path_weighted(t, [5.0, 5.0, 1.0], 0, 3) == [0, 3]
    assert algo.shortest_path_weighted(t, [1.0, 1.0, 5.0], 2, 2) == [2]
    assert algo.shortest_path_weighted(t, [1.0, 1.0, 5.0], 0, 2) is None
    assert algo.shortest_path_weighted_with_cost(t, [1.0, 1.0, 5.0], 0, 3) == ([0, 1, 3], [0.0, 1.0, 2.0])
    assert algo.shortest_path_weighted_with_cost(t, [1.0, 1.0, 5.0], 0, 0) == ([0], [0.0])
    t2 = Topology.build(4, [0, 1, 0, 0], [1, 3, 3, 3])
    assert algo.shortest_path_weighted_with_cost(t2, [1.0, 1.0, 5.0, 0.5], 0, 3) == ([0, 3], [0.0, 0.5])
    d = algo.dijkstra_distances(t, [1.0, 1.0, 5.0], 0)
    assert list(d[[0, 1, 3]]) == [0.0, 1.0, 2.0] and math.isinf(d[2])


def test_zero_weights_give_min_cost_paths(orc):
    """With zero-weight edges the settle order among equal distances depends
    on discovery order; the device path is then a valid minimum-cost path
    with the same cost (distances stay exact)."""
    from ursa_b200 import algo
    from cases import random_graph

    n, s, d = random_graph(500, 3000, 9)
    rng = np.random.default_rng(9)
    w = rng.integers(0, 3, s.size).astype(np.float64)
    g, o = _pair(orc, n, s, d)
    got_d = algo.dijkstra_distances(g, w, 0)
    assert np.array_equal(got_d, orc.dijkstra_distances(o, w, 0))
    for b in range(1, 60):
        got = algo.shortest_path_weighted_with_cost(g, w, 0, b)
        ref = orc.shortest_path_weighted_with_cost(o, w, 0, b)
        assert (got is None) == (ref is None)
        if got is None:
            continue
        path, cost = got
        assert path[0] == 0 and path[-1] == b and cost[-1] == ref[1][-1]
        # every hop is a real edge whose weight adds up exactly
        edges = {}
        for i in range(s.size):
            k = (int(s[i]), int(d[i]))
            edges[k] = min(edges.get(k, math.inf), w[i])
        for i in range(len(path) - 1):
            assert cost[i] + edges[(path[i], path[i + 1])] == cost[i + 1]


def test_poisson_weighted_c3_sample(orc):
    """The C3 graph family (Poisson(16) out-degree, f32 weights in [1,10)) at
    2^16 nodes: exact distances and paths from seeded sources."""
    from ursa_b200 import algo, gen

    n, s, d = gen.poisson(1 << 16, 16.0, 3)
    w = gen.weights_f32(s.size, 1.0, 10.0, 3).astype(np.float64)
    g, o = _pair(orc, n, s, d)
    for src in _nodes(n, 3, 13):
        assert np.array_equal(algo.dijkstra_distances(g, w, src), orc.dijkstra_distances(o, w, src))
        for b in _nodes(n, 3, src):
            assert algo.shortest_path_weighted_with_cost(g, w, src, b) == \
                orc.shortest_path_weighted_with_cost(o, w, src, b)
