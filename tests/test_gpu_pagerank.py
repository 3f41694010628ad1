"""PageRank on the GPU vs the f64 oracle (ursa-core/src/algo/pagerank.rs).

The device sums each row's f32 shares with compensated (TwoSum) f32
accumulation and keeps the update, residual and dangling mass in f64.
Tolerances (stated here, asserted per run):
  * fixed iteration count (tol = 0): max relative error <= 2e-6 and
    L1 error <= 1e-6;
  * convergence runs (tol > 0): the same iteration count as the oracle and
    the fixed-count bound.  The residual is summed exactly on the device
    (128-bit fixed point, each term truncated at 2^-96), so a count may
    differ by one only where the oracle's own residual at the earlier count
    lies within NEAR_TOL (relative) of tol -- the f32 shares move the device
    residual by far less than that; such a case is then held to L1 <= 3 * tol
    and max relative error <= 1e-3 (one power step apart).
"""

import numpy as np
import pytest

from cases import hub_graph, medium_cases, random_graph, small_cases

pytestmark = pytest.mark.gpu

MAXREL_FIXED = 2e-6
L1_FIXED = 1e-6
NEAR_TOL = 1e-3


def errors(got, ref):
    l1 = float(np.abs(got - ref).sum())
    denom = np.maximum(np.abs(ref), 1e-300)
    maxrel = float((np.abs(got - ref) / denom).max()) if ref.size else 0.0
    return l1, maxrel


def run_pair(orc, n, s, d, damping=0.85, max_iter=30, tol=1e-6, weights=None):
    from ursa_b200 import PageRankStats, Topology, algo

    g = Topology.build(n, s, d)
    o = orc.Topology(n, s, d)
    st = PageRankStats()
    if weights is None:
        got = algo.pagerank(g, damping=damping, max_iter=max_iter, tol=tol, stats=st)
        ref, it = orc.pagerank(o, damping, max_iter, tol, return_iters=True)
    else:
        got = algo.pagerank_weighted(g, weights, damping=damping, max_iter=max_iter, tol=tol, stats=st)
        ref, it = orc.pagerank_weighted(o, weights, damping, max_iter, tol, return_iters=True)
    run_pair.deltas = orc.pagerank_deltas()  # the oracle's residual per iteration
    return got, ref, st.iterations, it


def check(got, ref, it_gpu, it_ref, tol):
    l1, maxrel = errors(got, ref)
    if tol == 0 or it_gpu == it_ref:
        assert it_gpu == it_ref
        assert l1 <= L1_FIXED and maxrel <= MAXREL_FIXED, (l1, maxrel)
    else:
        assert abs(it_gpu - it_ref) == 1, (it_gpu, it_ref)
        d = run_pair.deltas[min(it_gpu, it_ref) - 1]
        assert abs(d - tol) <= NEAR_TOL * tol, (it_gpu, it_ref, d)
        assert l1 <= 3 * tol and maxrel <= 1e-3, (l1, maxrel)


@pytest.mark.parametrize("case", small_cases() + medium_cases(), ids=lambda c: c[0])
def test_pagerank_fixed_iterations(orc, case):
    _, n, s, d = case
    got, ref, a, b = run_pair(orc, n, s, d, max_iter=40, tol=0.0)
    check(got, ref, a, b, 0.0)


@pytest.mark.parametrize("case", small_cases() + medium_cases(), ids=lambda c: c[0])
def test_pagerank_default_params(orc, case):
    _, n, s, d = case
    got, ref, a, b = run_pair(orc, n, s, d)  # PageRankParams::default
    check(got, ref, a, b, 1e-6)


def test_pagerank_goldens():
    from ursa_b200 import Topology, algo

    pr = algo.pagerank(Topology.build(4, [0, 1, 3, 2], [2, 2, 2, 0]))  # pagerank.rs:275-285
    assert abs(pr.sum() - 1.0) < 1e-6
    assert all(i == 2 or v < pr[2] for i, v in enumerate(pr))
    assert algo.pagerank(Topology.build(0, [], [])).size == 0  # :287-291
    t = Topology.build(3, [0, 0, 1, 2], [1, 2, 0, 0])  # :293-310
    uni = algo.pagerank_weighted(t, [1.0, 1.0, 1.0, 1.0])
    assert abs(uni[1] - uni[2]) < 1e-9
    w = algo.pagerank_weighted(t, [1.0, 9.0, 1.0, 1.0])
    assert w[2] > w[1] and abs(w.sum() - 1.0) < 1e-6
    z = algo.pagerank_weighted(Topology.build(2, [0], [1]), [0.0])  # :312-319
    assert abs(z.sum() - 1.0) < 1e-6


def test_pagerank_max_iter_zero_and_edgeless():
    from ursa_b200 import Topology, algo

    g = Topology.build(5, [0, 1], [1, 2])
    assert np.array_equal(algo.pagerank(g, max_iter=0), np.full(5, 0.2))
    e = algo.pagerank(Topology.build(4, [], []), max_iter=10, tol=0.0)
    assert np.allclose(e, 0.25, rtol=0, atol=1e-15)


def test_pagerank_bit_reproducible():
    from ursa_b200 import Topology, algo
    from ursa_b200 import gen

    n, s, d = gen.rmat(15, 16, 3)
    g = Topology.build(n, s, d)
    a = algo.pagerank(g, max_iter=50, tol=1e-9)
    for _ in range(3):
        assert np.array_equal(algo.pagerank(g, max_iter=50, tol=1e-9), a)


@pytest.mark.parametrize("case", small_cases()[:10] + medium_cases(), ids=lambda c: c[0])
def test_pagerank_weighted(orc, case):
    _, n, s, d = case
    rng = np.random.default_rng(len(s))
    w = rng.uniform(1.0, 10.0, len(s)).astype(np.float32).astype(np.float64)
    got, ref, a, b = run_pair(orc, n, s, d, max_iter=30, tol=0.0, weights=w)
    check(got, ref, a, b, 0.0)


def test_pagerank_weighted_zero_weights(orc):
    n, s, d = random_graph(3000, 30_000, 5)
    rng = np.random.default_rng(5)
    w = rng.uniform(0.0, 3.0, s.size)
    w[rng.random(s.size) < 0.3] = 0.0  # zero-strength nodes become dangling
    got, ref, a, b = run_pair(orc, n, s, d, max_iter=25, tol=0.0, weights=w)
    check(got, ref, a, b, 0.0)


def test_pagerank_plain_then_weighted_on_one_topology(orc):
    """The execution plan is cached on the topology and built without the
    original edge ids until a weighted call needs them; the weighted call
    then builds a plan with them, and later plain calls keep using it."""
    from ursa_b200 import Topology, algo, gen

    n, s, d = gen.rmat(16, 16, 7)
    rng = np.random.default_rng(7)
    w = rng.uniform(1.0, 10.0, s.size).astype(np.float32).astype(np.float64)
    g = Topology.build(n, s, d)
    o = orc.Topology(n, s, d)
    ref_plain = orc.pagerank(o, 0.85, 20, 0.0)
    ref_w = orc.pagerank_weighted(o, w, 0.85, 20, 0.0)
    for weighted in (False, True, False, True):
        if weighted:
            got, ref = algo.pagerank_weighted(g, w, max_iter=20, tol=0.0), ref_w
        else:
            got, ref = algo.pagerank(g, max_iter=20, tol=0.0), ref_plain
        l1, maxrel = errors(got, ref)
        assert l1 <= L1_FIXED and maxrel <= MAXREL_FIXED, (weighted, l1, maxrel)
    g.free()


def test_pagerank_weighted_length_mismatch():
    from ursa_b200 import Topology, UrsaGpuError, algo

    with pytest.raises(UrsaGpuError, match="weights length"):
        algo.pagerank_weighted(Topology.build(3, [0, 1], [1, 2]), [1.0])


def test_pagerank_rmat20_vs_oracle(orc):
    from ursa_b200 import gen

    n, s, d = gen.rmat(20, 16, 2)
    got, ref, a, b = run_pair(orc, n, s, d, max_iter=100, tol=1e-6)
    check(got, ref, a, b, 1e-6)
    got, ref, a, b = run_pair(orc, n, s, d, max_iter=20, tol=0.0)
    check(got, ref, a, b, 0.0)


def test_pagerank_rmat22_properties():
    """Full-size R-MAT-22 (C2): converges within max_iter, mass is conserved
    (sum of ranks = 1 up to the f32 share rounding), run-to-run identical."""
    from ursa_b200 import PageRankStats, Topology, algo, gen

    n, s, d = gen.rmat(22, 16, 2)
    g = Topology.build(n, s, d)
    st = PageRankStats()
    pr = algo.pagerank(g, damping=0.85, max_iter=100, tol=1e-6, stats=st)
    assert 1 < st.iterations < 100 and st.last_delta < 1e-6
    assert abs(pr.sum() - 1.0) < 1e-5
    assert np.all(pr > 0)
    assert np.array_equal(pr, algo.pagerank(g, damping=0.85, max_iter=100, tol=1e-6))


def test_pagerank_hub_chunks_exact_structure(orc):
    # A hub whose in-degree spans many chunks, plus many hubs just above the
    # hub threshold, exercises the chunk-arrival finalisation.
    n, s, d = hub_graph(200_000, 9, True, 0)
    rng = np.random.default_rng(1)
    extra_s = rng.integers(0, n, 400_000, dtype=np.uint32)
    extra_d = (rng.integers(0, 300, 400_000) + 1).astype(np.uint32)  # 300 rows with ~1333 in-edges
    s = np.concatenate([s, extra_s])
    d = np.concatenate([d, extra_d])
    got, ref, a, b = run_pair(orc, n, s, d, max_iter=30, tol=0.0)
    check(got, ref, a, b, 0.0)
