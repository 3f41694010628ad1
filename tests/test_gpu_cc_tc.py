"""Weak connected components, triangle count and clustering coefficient on
the GPU vs the oracle (ursa-core/src/algo/components.rs, triangle.rs,
clustering.rs).

  * components: identical partitions; the device labels each component by its
    minimum member id, so it equals the oracle's labels canonicalised that way;
  * triangle_count: bit-exact u32 counts;
  * clustering_coefficient: bit-exact f64 (same formula and operation order).
"""

import numpy as np
import pytest

from cases import canon, medium_cases, small_cases

pytestmark = pytest.mark.gpu


def _pair(orc, n, s, d):
    from ursa_b200 import Topology

    return Topology.build(n, s, d), orc.Topology(n, s, d)


@pytest.mark.parametrize("case", small_cases() + medium_cases(), ids=lambda c: c[0])
def test_components_exact_partition(orc, case):
    from ursa_b200 import algo

    _, n, s, d = case
    g, o = _pair(orc, n, s, d)
    got = algo.connected_components_weak(g)
    ref = orc.connected_components_weak(o)
    assert np.array_equal(got, canon(ref))
    assert np.array_equal(canon(got), got)  # already min-member labels


@pytest.mark.parametrize("case", small_cases() + medium_cases(), ids=lambda c: c[0])
def test_triangles_and_clustering_exact(orc, case):
    from ursa_b200 import algo

    _, n, s, d = case
    g, o = _pair(orc, n, s, d)
    assert np.array_equal(algo.triangle_count(g), orc.triangle_count(o))
    got = algo.clustering_coefficient(g)
    ref = orc.clustering_coefficient(o)
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))


def test_goldens():
    from ursa_b200 import Topology, algo

    T = lambda n, s, d: list(algo.triangle_count(Topology.build(n, s, d)))  # noqa: E731
    assert T(3, [0, 0, 1, 2], [1, 2, 2, 0]) == [1, 1, 1]  # triangle.rs:251-281
    assert T(3, [0, 1], [1, 2]) == [0, 0, 0]
    assert T(4, [0, 0, 0, 1, 1, 2], [1, 2, 3, 2, 3, 3]) == [3, 3, 3, 3]
    assert T(3, [0, 0, 1, 2, 0, 0], [1, 2, 2, 0, 0, 1]) == [1, 1, 1]
    C = lambda n, s, d: algo.clustering_coefficient(Topology.build(n, s, d))  # noqa: E731
    assert list(C(3, [0, 0, 1, 2], [1, 2, 2, 0])) == [1.0, 1.0, 1.0]  # clustering.rs:328-357
    assert list(C(3, [0, 1], [1, 2])) == [0.0, 0.0, 0.0]
    cc = C(4, [0, 0, 0, 1], [1, 2, 3, 2])
    assert abs(cc[0] - 1.0 / 3.0) < 1e-12
    lab = algo.connected_components_weak(Topology.build(5, [0, 1, 3], [1, 2, 4]))  # components.rs:144-153
    assert list(lab) == [0, 0, 0, 3, 3]


def test_networkx_fixture(orc):
    import json
    import os

    from ursa_b200 import Topology, algo

    with open(os.path.join(os.path.dirname(__file__), "golden", "networkx_gnp100.json")) as f:
        g = json.load(f)
    dense = {k: v for k, v in g["dense_ids"]}
    t = Topology.build(len(dense), [dense[a] for a, _ in g["edges"]], [dense[b] for _, b in g["edges"]])
    tc = algo.triangle_count(t)
    cl = algo.clustering_coefficient(t)
    for k, v in g["triangles"].items():
        assert tc[dense[int(k)]] == v
    for k, v in g["clustering"].items():
        assert abs(cl[dense[int(k)]] - v) < 1e-9


def test_rmat18_exact(orc):
    from ursa_b200 import algo, gen

    n, s, d = gen.rmat(18, 16, 1)
    g, o = _pair(orc, n, s, d)
    assert np.array_equal(algo.triangle_count(g), orc.triangle_count(o))
    assert np.array_equal(algo.connected_components_weak(g), canon(orc.connected_components_weak(o)))


def test_triangles_long_oriented_lists_exact(orc):
    """Oriented lists of every length class the counting kernel has: a
    1,100-clique (its lowest-ranked member has 1,099 higher neighbours, above
    the 1,024 a shared-memory table holds), a 400-clique (lists of 257..399),
    hub stars and a sparse random part, all against the oracle."""
    from ursa_b200 import algo

    rng = np.random.default_rng(11)
    src, dst = [], []
    for base, k in ((0, 1100), (1100, 400)):
        a, b = np.triu_indices(k, 1)
        src.append(a + base)
        dst.append(b + base)
    n = 6000
    m = 30_000
    src.append(rng.integers(1500, n, m))
    dst.append(rng.integers(1500, n, m))
    for hub in (1500, 1501, 0):
        leaves = rng.choice(np.arange(1500, n), 900, replace=False)
        src.append(np.full(leaves.size, hub))
        dst.append(leaves)
    s = np.concatenate(src).astype(np.uint32)
    d = np.concatenate(dst).astype(np.uint32)
    g, o = _pair(orc, n, s, d)
    got = algo.triangle_count(g)
    assert np.array_equal(got, orc.triangle_count(o))
    assert got[0] >= 1099 * 1098 // 2  # the clique's own triangles at node 0
    assert np.array_equal(algo.clustering_coefficient(g), orc.clustering_coefficient(o))


def test_rmat22_properties():
    """Full-size R-MAT-22: component labels are min-member ids (label[u] <= u,
    label[label[u]] == label[u]) and every edge joins one component;
    triangle counts sum to a multiple of 3."""
    from ursa_b200 import Topology, algo, gen

    n, s, d = gen.rmat(22, 16, 2)
    g = Topology.build(n, s, d)
    lab = algo.connected_components_weak(g).astype(np.int64)
    assert np.all(lab <= np.arange(n)) and np.array_equal(lab[lab], lab)
    assert np.array_equal(lab[s], lab[d])
    tri = algo.triangle_count(g).astype(np.int64)
    assert tri.sum() % 3 == 0 and tri.sum() > 0
