"""Brandes betweenness on the GPU vs the oracle (ursa-core/src/algo/
betweenness.rs).  Sources (all, or the seeded sample) are the reference's;
shortest-path counts are exact integers; the dependency sums run in another
order than the reference's predecessor lists, so values agree to f64
rounding: |got - ref| <= 1e-9 * max(1, |ref|) per node (stated tolerance)."""

import json
import os

import numpy as np
import pytest

from cases import medium_cases, random_graph, small_cases

pytestmark = pytest.mark.gpu
RTOL = 1e-9


def close(got, ref):
    got, ref = np.asarray(got), np.asarray(ref)
    return got.shape == ref.shape and bool(np.all(np.abs(got - ref) <= RTOL * np.maximum(1.0, np.abs(ref))))


def _pair(orc, n, s, d):
    from ursa_b200 import Topology

    return Topology.build(n, s, d), orc.Topology(n, s, d)


SMALL = small_cases() + [c for c in medium_cases() if c[0] in ("rand_2000_100000", "hub_out_5000", "rmat14")]


@pytest.mark.parametrize("case", SMALL, ids=lambda c: c[0])
def test_betweenness_exact_sources(orc, case):
    from ursa_b200 import algo

    _, n, s, d = case
    if n > 20000:
        pytest.skip("all-source Brandes on the CPU oracle is too slow here")
    g, o = _pair(orc, n, s, d)
    assert close(algo.betweenness(g), orc.betweenness(o))


@pytest.mark.parametrize("case", SMALL, ids=lambda c: c[0])
def test_betweenness_sampled(orc, case):
    from ursa_b200 import algo

    _, n, s, d = case
    g, o = _pair(orc, n, s, d)
    for frac, seed in ((0.25, 42), (0.01, None), (1e-9, 7)):
        assert close(algo.betweenness(g, frac, seed), orc.betweenness(o, frac, seed)), (frac, seed)


@pytest.mark.parametrize("case", SMALL, ids=lambda c: c[0])
def test_betweenness_weighted(orc, case):
    from ursa_b200 import algo

    _, n, s, d = case
    w = np.random.default_rng(3).uniform(1.0, 10.0, len(s)).astype(np.float32).astype(np.float64)
    g, o = _pair(orc, n, s, d)
    frac = None if n <= 2000 else 0.02
    assert close(algo.betweenness_weighted(g, w, frac, 5), orc.betweenness_weighted(o, w, frac, 5))


def test_goldens():
    from ursa_b200 import Topology, algo

    line = Topology.build(5, [0, 1, 2, 3], [1, 2, 3, 4])  # betweenness.rs:368-375
    assert list(algo.betweenness(line)) == [0.0, 3.0, 4.0, 3.0, 0.0]
    assert list(algo.betweenness(line, None, 99)) == [0.0, 3.0, 4.0, 3.0, 0.0]
    dia = Topology.build(4, [0, 0, 1, 2], [1, 2, 3, 3])  # :377-387
    bc = algo.betweenness(dia)
    assert bc[0] == 0.0 and bc[3] == 0.0 and abs(bc[1] - 0.5) < 1e-12 and abs(bc[2] - 0.5) < 1e-12
    even = algo.betweenness_weighted(dia, [1.0, 1.0, 1.0, 1.0])  # :389-402
    assert abs(even[1] - 0.5) < 1e-12 and abs(even[2] - 0.5) < 1e-12
    cheap = algo.betweenness_weighted(dia, [1.0, 5.0, 1.0, 5.0])
    assert abs(cheap[1] - 1.0) < 1e-12 and abs(cheap[2]) < 1e-12
    n = 80  # :420-439
    cyc = algo.betweenness(Topology.build(n, list(range(n)), [(i + 1) % n for i in range(n)]))
    assert np.all(np.abs(cyc - cyc[0]) < 1e-9) and cyc[0] > 0
    ring = Topology.build(7, [0, 1, 2, 3, 4, 5, 6, 0, 2], [1, 2, 3, 4, 5, 6, 0, 3, 5])  # :441-460
    assert np.array_equal(algo.betweenness(ring, 0.5, 7), algo.betweenness(ring, 0.5, 7))
    assert algo.betweenness(Topology.build(0, [], [])).size == 0


def test_networkx_fixture():
    from ursa_b200 import Topology, algo

    with open(os.path.join(os.path.dirname(__file__), "golden", "networkx_gnp100.json")) as f:
        gx = json.load(f)
    dense = {k: v for k, v in gx["dense_ids"]}
    t = Topology.build(len(dense), [dense[a] for a, _ in gx["edges"]], [dense[b] for _, b in gx["edges"]])
    bc = algo.betweenness(t)
    for k, v in gx["betweenness"].items():  # test_networkx_reference.py:62-68
        assert abs(bc[dense[int(k)]] - v) < 1e-6


def test_weighted_length_mismatch():
    from ursa_b200 import Topology, UrsaGpuError, algo

    with pytest.raises(UrsaGpuError, match="weights length"):
        algo.betweenness_weighted(Topology.build(3, [0, 1], [1, 2]), [1.0])


def test_c3_family_sampled(orc):
    """The C3 family (Poisson(16) out-degree, f32 weights in [1,10)) at 2^15
    nodes with a seeded 2^-9 sample (64 sources), plain and weighted."""
    from ursa_b200 import algo, gen

    n, s, d = gen.poisson(1 << 15, 16.0, 3)
    w = gen.weights_f32(s.size, 1.0, 10.0, 3).astype(np.float64)
    g, o = _pair(orc, n, s, d)
    frac = 2.0 ** -9
    assert close(algo.betweenness(g, frac, 3), orc.betweenness(o, frac, 3))
    assert close(algo.betweenness_weighted(g, w, frac, 3), orc.betweenness_weighted(o, w, frac, 3))


def test_determinism_graph(orc):
    # ursa-core/tests/determinism_threads.rs:68-94 graphs (LCG n=300 m=2500; n=400 m=4000)
    from test_oracle_golden import lcg_graph

    from ursa_b200 import algo

    s, d = lcg_graph(300, 2500)
    g, o = _pair(orc, 300, s, d)
    assert close(algo.betweenness(g), orc.betweenness(o))
    s, d = lcg_graph(400, 4000)
    g, o = _pair(orc, 400, s, d)
    got = algo.betweenness(g, 0.25, 42)
    assert close(got, orc.betweenness(o, 0.25, 42))
    assert np.array_equal(got, algo.betweenness(g, 0.25, 42))
