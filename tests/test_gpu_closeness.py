"""Closeness and the path statistics on the device vs the oracle
(ursa-core/src/algo/closeness.rs:69-224, ursa-plan/src/stats.rs:82-167).

Bit-exact: unweighted closeness (integer folds, one f64 division per node),
avg_path_length and diameter (integer distance totals below 2^53), and
weighted closeness (exact Dijkstra distances, node-order f64 sums).
"""

import numpy as np
import pytest

from cases import random_graph, small_cases

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.asarray(a, np.float64).view(np.uint64)


def _cases():
    from ursa_b200 import gen

    out = [(name, n, s, d) for name, n, s, d in small_cases()]
    out.append(("rand_300", *random_graph(300, 1200, 4)))
    out.append(("rand_2000", *random_graph(2000, 6000, 5)))  # more than 64 sources per batch
    n, s, d = gen.rmat(11, 8, 9)
    out.append(("rmat11", n, s, d))
    chain = 130
    out.append(("chain130", chain, list(range(chain - 1)), list(range(1, chain))))  # 129 levels
    # hubs: in-degree 2,499 and 1,200 (split scans over several warps), a
    # tail leaving the hub, random edges among the spokes
    rng = np.random.default_rng(12)
    hs = list(range(1, 2500)) + list(range(1300, 2500)) + [0] + list(range(2500, 2599))
    hd = [0] * 2499 + [1] * 1200 + [2500] + list(range(2501, 2600))
    rs, rd = rng.integers(1, 2500, 3000), rng.integers(1, 2500, 3000)
    out.append(("hubs", 2600, hs + rs.tolist(), hd + rd.tolist()))
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_closeness_exact(orc, case):
    from ursa_b200 import Topology, algo

    _, n, s, d = case
    got = algo.closeness(Topology.build(n, s, d))
    ref = orc.closeness(orc.Topology(n, s, d))
    assert np.array_equal(_bits(got), _bits(ref))


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_path_stats_exact(orc, case):
    from ursa_b200 import Topology, algo

    _, n, s, d = case
    g, o = Topology.build(n, s, d), orc.Topology(n, s, d)
    for sample in (None, 0.1, 0.5, 1.0):
        assert _bits([algo.avg_path_length(g, sample)])[0] == _bits([orc.avg_path_length(o, sample)])[0], sample
    for approx in (False, True):
        assert algo.diameter(g, approx) == orc.diameter(o, approx)


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_closeness_weighted_exact(orc, case):
    from ursa_b200 import Topology, algo

    _, n, s, d = case
    rng = np.random.default_rng(n)
    w = rng.uniform(0.0, 4.0, len(s))
    if len(w):
        w[rng.integers(0, len(w), max(1, len(w) // 10))] = 0.0  # zero-cost edges
    got = algo.closeness_weighted(Topology.build(n, s, d), w)
    ref = orc.closeness_weighted(orc.Topology(n, s, d), w)
    assert np.array_equal(_bits(got), _bits(ref))


def test_reference_goldens():
    from ursa_b200 import Topology, algo

    c = algo.closeness(Topology.build(4, [0, 1, 2], [1, 2, 3]))
    assert list(c) == [0.5, 2.0 / 3.0, 1.0, 0.0]  # closeness.rs directed line
    assert algo.closeness(Topology.build(0, [], [])).size == 0
    c = algo.closeness_weighted(Topology.build(3, [0, 1, 0], [1, 2, 2]), [1.0, 1.0, 5.0])
    assert abs(c[0] - 2.0 / 3.0) < 1e-12 and abs(c[1] - 1.0) < 1e-12
    tri = Topology.build(3, [0, 1, 2], [1, 2, 0])
    assert algo.avg_path_length(tri) == 1.5 and algo.diameter(tri, False) == 2  # stats.rs
    two = Topology.build(4, [0, 2], [1, 3])
    assert algo.avg_path_length(two) == 1.0 and algo.diameter(two, False) == 1


def test_closeness_device_output(orc):
    """ursa_gpu_closeness_device: same bits as the host form, device time > 0."""
    import ctypes as C

    import torch

    from ursa_b200 import Topology, _lib, algo, gen

    n, s, d = gen.rmat(12, 8, 3)
    g = Topology.build(n, s, d)
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    ms = C.c_float()
    _lib.check(_lib.load().ursa_gpu_closeness_device(g.handle, out.data_ptr(), None, C.byref(ms)))
    assert np.array_equal(_bits(out.cpu().numpy()), _bits(algo.closeness(g)))
    assert ms.value > 0.0


def test_negative_weights_rejected():
    """evaluate_weight rejects negative weights before any Dijkstra-family
    kernel (ursa-plan/src/weight.rs:88-93); the C ABI does the same."""
    import ctypes as C

    from ursa_b200 import Topology, _lib

    L = _lib.load()
    g = Topology.build(3, [0, 1], [1, 2])
    w = np.array([1.0, -0.5])
    out = np.empty(3)
    assert L.ursa_gpu_closeness_weighted(g.handle, w.ctypes.data, 2, out.ctypes.data) == 1
    assert L.ursa_gpu_dijkstra_distances(g.handle, w.ctypes.data, 2, 0, 0, out.ctypes.data) == 1
    path, cost, ln = np.empty(3, np.uint32), np.empty(3), C.c_int64()
    assert L.ursa_gpu_shortest_path_weighted_with_cost(g.handle, w.ctypes.data, 2, 0, 2, 0, path.ctypes.data,
                                                       cost.ctypes.data, 3, C.byref(ln)) == 1
    assert L.ursa_gpu_betweenness_weighted(g.handle, w.ctypes.data, 2, 0, 0.0, 0, 0, out.ctypes.data) == 1
    w0 = np.array([1.0, -0.0])  # negative zero is not negative
    assert L.ursa_gpu_closeness_weighted(g.handle, w0.ctypes.data, 2, out.ctypes.data) == 0
