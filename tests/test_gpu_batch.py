"""Batched execution of many small graphs (ursa_gpu_batch_*) vs the oracle.

Per graph of a batch, the device computes pagerank, weak components and
triangle counts; each is compared with the oracle run on that graph alone
(ursa-core/src/algo/pagerank.rs:98-124, components.rs:58-68,
triangle.rs:40-62):
  * components: the oracle's partition, labelled by minimum member (local) id;
  * triangle counts: bit-exact;
  * pagerank: the plain kernel's bounds -- with a fixed iteration count
    (tol = 0) max relative error <= 2e-6 and L1 <= 1e-6; with tol > 0 the
    iteration count may differ by one, then L1 <= 3 * tol and max relative
    error <= 1e-3.
Results must not depend on the launch configuration nor on the batch's
other graphs (bit-identical), which the tests check directly.
"""

import numpy as np
import pytest

from cases import canon, hub_graph, random_graph, small_cases

pytestmark = pytest.mark.gpu

MAXREL_FIXED = 2e-6
L1_FIXED = 1e-6


def _graphs():
    gs = [(n, np.asarray(s, np.uint32), np.asarray(d, np.uint32)) for _, n, s, d in small_cases()]
    gs.append(random_graph(2000, 30_000, 11))
    gs.append(random_graph(300, 9_000, 12))
    gs.append(hub_graph(5000, 1, True, 20000))
    gs.append(hub_graph(3000, 2, False, 5000))
    gs.append(random_graph(70_000, 400_000, 13))  # above every shared-memory capacity
    gs.append((0, np.empty(0, np.uint32), np.empty(0, np.uint32)))  # empty graph
    from ursa_b200 import gen

    n, k, s, d = gen.rmat_batch(24, median=600.0, hi=8000, seed0=500)
    off = np.concatenate([[0], np.cumsum(k)]).astype(np.int64)
    for i in range(len(n)):
        gs.append((int(n[i]), s[off[i]:off[i + 1]], d[off[i]:off[i + 1]]))
    return gs


@pytest.fixture(scope="module")
def graphs():
    return _graphs()


@pytest.fixture(scope="module")
def batch(graphs):
    from ursa_b200.batch import GraphBatch

    return GraphBatch.from_graphs(graphs)


def _errors(got, ref):
    l1 = float(np.abs(got - ref).sum())
    maxrel = float((np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)).max()) if ref.size else 0.0
    return l1, maxrel


def _check_all(orc, graphs, res, max_iter, tol):
    for g, (n, s, d) in enumerate(graphs):
        r = res.graph(g)
        o = orc.Topology(n, s, d)
        ref, it = orc.pagerank(o, 0.85, max_iter, tol, return_iters=True)
        l1, maxrel = _errors(r["pagerank"], ref)
        if tol == 0 or r["iterations"] == it:
            assert r["iterations"] == it, (g, r["iterations"], it)
            assert l1 <= L1_FIXED and maxrel <= MAXREL_FIXED, (g, n, l1, maxrel)
        else:
            assert abs(r["iterations"] - it) <= 1, (g, r["iterations"], it)
            assert l1 <= 3 * tol and maxrel <= 1e-3, (g, l1, maxrel)
        assert np.array_equal(r["components"], canon(orc.connected_components_weak(o))), g
        assert np.array_equal(r["triangles"], orc.triangle_count(o)), g


def test_batch_fixed_iterations_vs_oracle(orc, graphs, batch):
    batch.run(max_iter=25, tol=0.0)
    _check_all(orc, graphs, batch.results(), 25, 0.0)


def test_batch_converged_vs_oracle(orc, graphs, batch):
    batch.run(max_iter=100, tol=1e-6)
    _check_all(orc, graphs, batch.results(), 100, 1e-6)


def _snapshot(batch):
    r = batch.results()
    return r.pagerank.copy(), r.components.copy(), r.triangles.copy(), r.iterations.copy(), r.last_delta.copy()


def _same(a, b):
    return (np.array_equal(a[0].view(np.uint64), b[0].view(np.uint64)) and np.array_equal(a[1], b[1])
            and np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])
            and np.array_equal(a[4].view(np.uint64), b[4].view(np.uint64)))


def test_results_independent_of_configuration(batch):
    batch.set_config([4096, 16384, 57344], [256, 512, 1024], 32, 256)
    batch.run(max_iter=100, tol=1e-6)
    ref = _snapshot(batch)
    for cap, th, tile, tct in [
        ([57344], [1024], 1, 128),
        ([64, 1024, 8192], [128, 256, 512], 256, 512),  # most graphs keep global shares
        ([2048, 30000], [512, 128], 7, 256),
        ([16], [128], 4096, 128),  # every graph above the capacity
    ]:
        batch.set_config(cap, th, tile, tct)
        batch.run(max_iter=100, tol=1e-6)
        assert _same(_snapshot(batch), ref), (cap, th, tile, tct)
    batch.set_config([4096, 16384, 57344], [256, 512, 1024], 32, 256)


def test_results_independent_of_batch_composition(graphs, batch):
    from ursa_b200.batch import GraphBatch

    batch.run(max_iter=60, tol=1e-7)
    whole = batch.results()
    for g in [0, 8, len(graphs) - 1, len(graphs) - 20]:
        alone = GraphBatch.from_graphs([graphs[g]])
        alone.run(max_iter=60, tol=1e-7)
        a = alone.results().graph(0)
        w = whole.graph(g)
        assert np.array_equal(a["pagerank"].view(np.uint64), w["pagerank"].view(np.uint64)), g
        assert np.array_equal(a["components"], w["components"]), g
        assert np.array_equal(a["triangles"], w["triangles"]), g
        assert a["iterations"] == w["iterations"], g
        alone.close()


def test_matches_plain_single_graph_path(graphs, batch):
    """Components and triangle counts equal the plain kernels' output; the
    plain and batched pageranks agree within twice the oracle bound."""
    from ursa_b200 import Topology, algo

    batch.run(max_iter=30, tol=0.0)
    res = batch.results()
    for g in [1, 5, 8, 15, 16, 17, 18, 20, 30]:
        n, s, d = graphs[g]
        if n == 0:
            continue
        t = Topology.build(n, s, d)
        r = res.graph(g)
        assert np.array_equal(r["components"], algo.connected_components_weak(t)), g
        assert np.array_equal(r["triangles"], algo.triangle_count(t)), g
        l1, maxrel = _errors(r["pagerank"], algo.pagerank(t, max_iter=30, tol=0.0))
        assert l1 <= 2 * L1_FIXED and maxrel <= 2 * MAXREL_FIXED, (g, l1, maxrel)


def test_algorithm_subsets(graphs, batch):
    from ursa_b200.batch import BATCH_COMPONENTS, BATCH_PAGERANK, BATCH_TRIANGLES

    batch.run(max_iter=20, tol=0.0)
    full = _snapshot(batch)
    batch.run(max_iter=20, tol=0.0, what=BATCH_TRIANGLES)
    assert np.array_equal(batch.results().triangles, full[2])
    batch.run(max_iter=20, tol=0.0, what=BATCH_COMPONENTS)
    assert np.array_equal(batch.results().components, full[1])
    batch.run(max_iter=20, tol=0.0, what=BATCH_PAGERANK)
    assert np.array_equal(batch.results().pagerank.view(np.uint64), full[0].view(np.uint64))


def test_tuner_picks_a_valid_config_and_keeps_results(batch):
    batch.run(max_iter=40, tol=1e-6)
    before = _snapshot(batch)
    cfg, ms = batch.tune(max_iter=40, tol=1e-6)
    assert ms > 0
    assert 1 <= cfg["n_buckets"] <= 3 and 1 <= cfg["tc_tile"] <= 4096
    assert all(t in (128, 256, 512, 1024) for t in cfg["threads"])
    assert cfg["tc_threads"] in (128, 256, 512)
    assert batch.config() == cfg
    batch.run(max_iter=40, tol=1e-6)
    assert _same(_snapshot(batch), before)


def test_max_iter_zero_returns_uniform(graphs):
    from ursa_b200.batch import GraphBatch

    b = GraphBatch.from_graphs(graphs[:6])
    b.run(max_iter=0, tol=1e-6)
    r = b.results()
    for g in range(6):
        n = graphs[g][0]
        assert np.all(r.graph(g)["pagerank"] == 1.0 / n)
        assert r.graph(g)["iterations"] == 0


def test_rmat_batch_sample(orc):
    """A slice of the batched R-MAT family (log-normal sizes, per-graph edge
    factor 8..32, seed 100 + i) at its real sizes."""
    from ursa_b200 import gen
    from ursa_b200.batch import GraphBatch

    n, k, s, d = gen.rmat_batch(40)
    b = GraphBatch(n, k, s, d)
    b.tune(max_iter=100, tol=1e-6)
    b.run(max_iter=100, tol=1e-6)
    res = b.results()
    off = np.concatenate([[0], np.cumsum(k)]).astype(np.int64)
    graphs = [(int(n[i]), s[off[i]:off[i + 1]], d[off[i]:off[i + 1]]) for i in range(len(n))]
    _check_all(orc, graphs, res, 100, 1e-6)


def test_bad_local_id_is_rejected():
    from ursa_b200 import UrsaGpuError
    from ursa_b200.batch import GraphBatch

    with pytest.raises(UrsaGpuError, match="EINVAL"):
        GraphBatch([3, 2], [1, 1], [0, 2], [1, 0])  # graph 1 has 2 nodes: id 2 is out of range


def test_empty_batch():
    from ursa_b200.batch import GraphBatch

    b = GraphBatch([], [], [], [])
    b.run()
    r = b.results()
    assert r.pagerank.size == 0 and r.iterations.size == 0
