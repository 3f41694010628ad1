"""Pin the CPU oracle against every golden value the reference's own tests hold
for the hot path: ursa-core's inline unit tests (topology.rs, degree.rs,
pagerank.rs, bfs.rs, hop.rs, components.rs, triangle.rs, clustering.rs,
betweenness.rs, rng.rs), the thread-count determinism test
(ursa-core/tests/determinism_threads.rs), the Python end-to-end goldens
(tests/test_native_kernels.py, test_weighted.py, test_scan_and_pipeline.py,
test_determinism_and_scan.py, test_graph_algorithms.py) and the NetworkX
cross-check (tests/test_networkx_reference.py), through a committed fixture.
"""

import json
import math
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def diamond(orc):
    # topology.rs:438-440
    return orc.Topology(3, [0, 0, 1, 2], [1, 2, 2, 0])


def path5(orc):
    # bfs.rs:266-268 / hop.rs:525-527: 0->1->2->3 plus 1->4
    return orc.Topology(5, [0, 1, 2, 1], [1, 2, 3, 4])


def nbrs(off, tg, u):
    return [int(x) for x in tg[off[u] : off[u + 1]]]


# ---------------------------------------------------------------- topology.rs
def test_parallel_build_is_byte_identical_to_serial(orc):
    # topology.rs:443-469 (random keys; serial = 1 thread, parallel = 2/3/8)
    rng = np.random.default_rng(0xC0FFEE)
    for n, m in [(2000, 100_000), (50_000, 300_000), (16, 80_000)]:
        keys = rng.integers(0, n, m, dtype=np.uint32)
        other = rng.integers(0, n, m, dtype=np.uint32)
        orc.set_threads(1)
        ref = orc.Topology(n, keys, other).csr("out")
        for th in (2, 3, 8):
            orc.set_threads(th)
            got = orc.Topology(n, keys, other).csr("out")
            for a, b in zip(ref, got):
                assert np.array_equal(a, b)
    orc.set_threads(1)


def test_out_adjacency_groups_by_source(orc):
    off, tg, _ = diamond(orc).csr("out")  # topology.rs:472-478
    assert nbrs(off, tg, 0) == [1, 2]
    assert nbrs(off, tg, 1) == [2]
    assert nbrs(off, tg, 2) == [0]
    assert off[1] - off[0] == 2


def test_transpose_is_correct(orc):
    off, tg, _ = diamond(orc).csr("in")  # topology.rs:481-489, 516-532
    assert sorted(nbrs(off, tg, 2)) == [0, 1]
    assert nbrs(off, tg, 0) == [2]
    assert nbrs(off, tg, 1) == [0]


def test_edge_ids_track_original_rows(orc):
    off, _, eid = diamond(orc).csr("out")  # topology.rs:492-498
    assert sorted(int(x) for x in eid[off[0] : off[1]]) == [0, 1]


def test_undirected_sorted_deduped_self_loop_free(orc):
    t = orc.Topology(3, [0, 0, 1, 2, 1, 0], [1, 2, 2, 0, 1, 1])  # topology.rs:501-513
    off, tg = t.undirected()
    assert nbrs(off, tg, 0) == [1, 2]
    assert nbrs(off, tg, 1) == [0, 2]
    assert nbrs(off, tg, 2) == [0, 1]


# ------------------------------------------------------------------ degree.rs
def test_degree_directions(orc):
    t = diamond(orc)  # degree.rs:35-41, test_native_kernels.py:44-48
    assert degree_list(orc, t, "out") == [2, 1, 1]
    assert degree_list(orc, t, "in") == [1, 1, 2]
    assert degree_list(orc, t, "both") == [3, 2, 3]


def degree_list(orc, t, d):
    return [int(x) for x in orc.degree(t, d)]


# ---------------------------------------------------------------- pagerank.rs
def test_pagerank_sums_to_one_and_hub_highest(orc):
    t = orc.Topology(4, [0, 1, 3, 2], [2, 2, 2, 0])  # pagerank.rs:175-185
    pr = orc.pagerank(t)
    assert abs(pr.sum() - 1.0) < 1e-6
    assert all(i == 2 or v < pr[2] for i, v in enumerate(pr))


def test_pagerank_empty(orc):
    assert orc.pagerank(orc.Topology(0, [], [])).size == 0  # pagerank.rs:187-191


def test_weighted_pagerank_shifts_rank(orc):
    t = orc.Topology(3, [0, 0, 1, 2], [1, 2, 0, 0])  # pagerank.rs:193-210
    uni = orc.pagerank_weighted(t, [1.0, 1.0, 1.0, 1.0])
    assert abs(uni[1] - uni[2]) < 1e-9
    w = orc.pagerank_weighted(t, [1.0, 9.0, 1.0, 1.0])
    assert w[2] > w[1]
    assert abs(w.sum() - 1.0) < 1e-6
    # test_weighted.py:43-62: amount*fx = [5, 6, 1, 1]
    w2 = orc.pagerank_weighted(t, [5.0, 6.0, 1.0, 1.0])
    assert w2[2] > w2[1]
    # unweighted: symmetric 1 and 2 (test_weighted.py:38)
    u = orc.pagerank(t)
    assert abs(u[1] - u[2]) < 1e-9


def test_zero_weight_out_edges_are_dangling(orc):
    t = orc.Topology(2, [0], [1])  # pagerank.rs:212-219
    pr = orc.pagerank_weighted(t, [0.0])
    assert abs(pr.sum() - 1.0) < 1e-6


def test_pagerank_bit_reproducible_across_threads(orc):
    # determinism_threads.rs:19-66: LCG graph n=400 m=4000, tol 1e-12, 100 iters
    src, dst = lcg_graph(400, 4000)
    ref = None
    for th in (1, 2, 3, 4, 8):
        orc.set_threads(th)
        t = orc.Topology(400, src, dst)
        pr = orc.pagerank(t, 0.85, 100, 1e-12)
        if ref is None:
            ref = pr
        assert np.array_equal(pr, ref)
    orc.set_threads(1)


def lcg_graph(n, m):
    # determinism_threads.rs:19-35
    state = 0x9E3779B97F4A7C15
    mask = (1 << 64) - 1
    src, dst = [], []
    for _ in range(m):
        state = (state * 6364136223846793005 + 1442695040888963407) & mask
        src.append((state >> 33) % n)
        state = (state * 6364136223846793005 + 1442695040888963407) & mask
        dst.append((state >> 33) % n)
    return np.array(src, np.uint32), np.array(dst, np.uint32)


# --------------------------------------------------------------------- bfs.rs
def test_bfs_distances_along_a_path(orc):
    d = orc.bfs_distances(path5(orc), 0, "out")  # bfs.rs:270-279
    assert list(d) == [0, 1, 2, 3, 2]


def test_bfs_unreachable_is_negative_one(orc):
    d = orc.bfs_distances(path5(orc), 3, "out")  # bfs.rs:281-289
    assert d[3] == 0 and d[0] == -1 and d[1] == -1


def test_bfs_both_direction(orc):
    d = orc.bfs_distances(path5(orc), 3, "both")  # bfs.rs:291-298
    assert d[0] == 3 and d[4] == 3


def test_bfs_out_of_range_source(orc):
    assert list(orc.bfs_distances(path5(orc), 99, "out")) == [-1] * 5  # bfs.rs:21-23


def test_shortest_path_cases(orc):
    t = path5(orc)  # bfs.rs:300-332
    assert orc.shortest_path(t, 0, 3) == [0, 1, 2, 3]
    assert orc.shortest_path(t, 0, 4) == [0, 1, 4]
    assert orc.shortest_path(t, 2, 2) == [2]
    assert orc.shortest_path(t, 3, 0) is None
    assert orc.shortest_path(t, 0, 99) is None
    assert orc.shortest_path(t, 3, 0, "in") == [3, 2, 1, 0]


def test_weighted_shortest_path_cases(orc):
    t = orc.Topology(4, [0, 1, 0], [1, 3, 3])  # bfs.rs:334-387
    assert orc.shortest_path(t, 0, 3) == [0, 3]
    assert orc.shortest_path_weighted(t, [1.0, 1.0, 5.0], 0, 3) == [0, 1, 3]
    assert orc.shortest_path_weighted(t, [5.0, 5.0, 1.0], 0, 3) == [0, 3]
    assert orc.shortest_path_weighted(t, [1.0, 1.0, 5.0], 2, 2) == [2]
    assert orc.shortest_path_weighted(t, [1.0, 1.0, 5.0], 0, 2) is None
    assert orc.shortest_path_weighted_with_cost(t, [1.0, 1.0, 5.0], 0, 3) == ([0, 1, 3], [0.0, 1.0, 2.0])
    assert orc.shortest_path_weighted_with_cost(t, [1.0, 1.0, 5.0], 0, 0) == ([0], [0.0])
    t2 = orc.Topology(4, [0, 1, 0, 0], [1, 3, 3, 3])
    assert orc.shortest_path_weighted_with_cost(t2, [1.0, 1.0, 5.0, 0.5], 0, 3) == ([0, 3], [0.0, 0.5])


def test_dijkstra_distances(orc):
    t = orc.Topology(4, [0, 1, 0], [1, 3, 3])
    d = orc.dijkstra_distances(t, [1.0, 1.0, 5.0], 0)
    assert list(d[[0, 1, 3]]) == [0.0, 1.0, 2.0]
    assert math.isinf(d[2])
    assert all(math.isinf(x) for x in orc.dijkstra_distances(t, [1.0, 1.0, 5.0], 77))


def test_scan_pipeline_path_goldens(orc):
    # test_scan_and_pipeline.py:384-420, test_weighted.py:65-80
    t = orc.Topology(4, [0, 1, 2], [1, 2, 3])
    assert orc.shortest_path(t, 0, 3) == [0, 1, 2, 3]
    assert orc.shortest_path(t, 3, 0) is None
    assert orc.shortest_path(t, 3, 0, "in") == [3, 2, 1, 0]
    tw = orc.Topology(3, [0, 1, 0], [1, 2, 2])
    assert orc.shortest_path_weighted_with_cost(tw, [1.0, 1.0, 5.0], 0, 2) == ([0, 1, 2], [0.0, 1.0, 2.0])


# --------------------------------------------------------------------- hop.rs
def pairs(s, d):
    return sorted(zip((int(x) for x in s), (int(y) for y in d)))


def test_k_hop_goldens(orc):
    t = path5(orc)  # hop.rs:535-580
    assert pairs(*orc.k_hop(t, [0], 1)) == [(0, 1)]
    assert pairs(*orc.k_hop(t, [0], 2)) == [(0, 1), (0, 2), (0, 4)]
    assert pairs(*orc.k_hop(t, [0], 10)) == [(0, 1), (0, 2), (0, 3), (0, 4)]
    assert pairs(*orc.k_hop(t, [3], 2, "in")) == [(3, 1), (3, 2)]
    assert pairs(*orc.k_hop(t, [0, 2], 1)) == [(0, 1), (2, 3)]
    s, d = orc.k_hop(t, [99], 3)
    assert s.size == 0 and d.size == 0
    s, d = orc.k_hop(t, [0], 0)
    assert s.size == 0
    # repeated seed emits its pairs again (hop.rs:41-44)
    s, d = orc.k_hop(t, [0, 0], 1)
    assert list(s) == [0, 0] and list(d) == [1, 1]


def test_k_hop_python_goldens(orc):
    # test_scan_and_pipeline.py:331-368
    t = orc.Topology(5, [0, 1, 2, 1], [1, 2, 3, 4])
    s, d = orc.k_hop(t, [0], 2)
    assert set(int(x) for x in d) == {1, 2, 4}
    t2 = orc.Topology(4, [0, 1, 2], [1, 2, 3])
    assert set(int(x) for x in orc.k_hop(t2, [3], 2, "in")[1]) == {1, 2}
    t3 = orc.Topology(4, [1, 2, 3], [0, 0, 0])
    s, d = orc.k_hop(t3, [1, 2, 3], 1)
    assert list(s) == [1, 2, 3] and list(d) == [0, 0, 0]


# -------------------------------------------------------------- components.rs
def canon(labels):
    """Relabel each component by its minimum member id."""
    labels = np.asarray(labels)
    mins = {}
    for i, l in enumerate(labels):
        mins.setdefault(int(l), i)
    return np.array([mins[int(l)] for l in labels], dtype=np.uint32)


def test_components_two(orc):
    cc = orc.connected_components_weak(orc.Topology(5, [0, 1, 3], [1, 2, 4]))  # components.rs:144-153
    assert cc[0] == cc[1] == cc[2] and cc[3] == cc[4] and cc[0] != cc[3]
    assert list(canon(cc)) == [0, 0, 0, 3, 3]


def test_components_chain(orc):
    cc = orc.connected_components_weak(orc.Topology(3, [0, 1], [1, 2]))  # components.rs:170-176
    assert cc[0] == cc[1] == cc[2]


# ------------------------------------------------------- triangle/clustering
def test_triangle_goldens(orc):
    T = orc.triangle_count  # triangle.rs:251-281
    assert list(T(orc.Topology(3, [0, 0, 1, 2], [1, 2, 2, 0]))) == [1, 1, 1]
    assert list(T(orc.Topology(3, [0, 1], [1, 2]))) == [0, 0, 0]
    assert list(T(orc.Topology(4, [0, 0, 0, 1, 1, 2], [1, 2, 3, 2, 3, 3]))) == [3, 3, 3, 3]
    assert list(T(orc.Topology(3, [0, 0, 1, 2, 0, 0], [1, 2, 2, 0, 0, 1]))) == [1, 1, 1]


def test_triangle_count_nodes_equals_full_count(orc):
    """The per-node restatement (used to check large graphs on a sample of
    nodes) gives triangle_count's values for the listed nodes, in any order."""
    rng = np.random.default_rng(5)
    n, m = 2000, 30_000
    t = orc.Topology(n, rng.integers(0, n, m).astype(np.uint32), rng.integers(0, n, m).astype(np.uint32))
    full = orc.triangle_count(t)
    nodes = rng.choice(n, 700, replace=False)
    assert np.array_equal(orc.triangle_count_nodes(t, nodes), full[nodes])
    assert orc.triangle_count_nodes(t, []).size == 0


def test_clustering_goldens(orc):
    C = orc.clustering_coefficient  # clustering.rs:328-357
    assert list(C(orc.Topology(3, [0, 0, 1, 2], [1, 2, 2, 0]))) == [1.0, 1.0, 1.0]
    assert list(C(orc.Topology(3, [0, 1], [1, 2]))) == [0.0, 0.0, 0.0]
    cc = C(orc.Topology(4, [0, 0, 0], [1, 2, 3]))
    assert cc[0] == 0.0 and cc[1] == 0.0
    cc = C(orc.Topology(4, [0, 0, 0, 1], [1, 2, 3, 2]))
    assert abs(cc[0] - 1.0 / 3.0) < 1e-12


# ------------------------------------------------------------ betweenness.rs
def test_betweenness_line(orc):
    t = orc.Topology(5, [0, 1, 2, 3], [1, 2, 3, 4])  # betweenness.rs:368-375
    assert list(orc.betweenness(t)) == [0.0, 3.0, 4.0, 3.0, 0.0]
    # exact ignores the seed (test_determinism_and_scan.py:69-75)
    assert list(orc.betweenness(t, None, 99)) == [0.0, 3.0, 4.0, 3.0, 0.0]


def test_betweenness_diamond(orc):
    bc = orc.betweenness(orc.Topology(4, [0, 0, 1, 2], [1, 2, 3, 3]))  # :377-387
    assert bc[0] == 0.0 and bc[3] == 0.0
    assert abs(bc[1] - 0.5) < 1e-12 and abs(bc[2] - 0.5) < 1e-12


def test_betweenness_weighted_cheap_route(orc):
    t = orc.Topology(4, [0, 0, 1, 2], [1, 2, 3, 3])  # :389-402, test_weighted.py:129-142
    even = orc.betweenness_weighted(t, [1.0, 1.0, 1.0, 1.0])
    assert abs(even[1] - 0.5) < 1e-12 and abs(even[2] - 0.5) < 1e-12
    cheap = orc.betweenness_weighted(t, [1.0, 5.0, 1.0, 5.0])
    assert abs(cheap[1] - 1.0) < 1e-12 and abs(cheap[2]) < 1e-12


def test_betweenness_sample_bounded(orc):
    t = orc.Topology(5, [0, 1, 2, 3], [1, 2, 3, 4])  # :404-412
    bc = orc.betweenness(t, 0.5, 7)
    assert all(x >= 0 and math.isfinite(x) for x in bc)
    assert bc[2] >= bc[0]


def test_betweenness_cycle_uniform_across_chunks(orc):
    n = 80  # :420-439
    t = orc.Topology(n, list(range(n)), [(i + 1) % n for i in range(n)])
    bc = orc.betweenness(t)
    assert all(abs(x - bc[0]) < 1e-9 for x in bc) and bc[0] > 0


def test_betweenness_sampled_seed_reproducible(orc):
    t = orc.Topology(7, [0, 1, 2, 3, 4, 5, 6, 0, 2], [1, 2, 3, 4, 5, 6, 0, 3, 5])  # :441-460
    assert np.array_equal(orc.betweenness(t, 0.5, 7), orc.betweenness(t, 0.5, 7))
    a = orc.sample_sources(7, 0.5, 1)
    b = orc.sample_sources(7, 0.5, 2)
    assert len(a) == len(b) and list(a) != list(b)


def test_betweenness_thread_count_independent(orc):
    # determinism_threads.rs:68-94
    src, dst = lcg_graph(300, 2500)
    src4, dst4 = lcg_graph(400, 4000)
    ref_full = ref_samp = None
    for th in (1, 2, 3, 4, 8):
        orc.set_threads(th)
        full = orc.betweenness(orc.Topology(300, src, dst))
        samp = orc.betweenness(orc.Topology(400, src4, dst4), 0.25, 42)
        if ref_full is None:
            ref_full, ref_samp = full, samp
        assert np.array_equal(full, ref_full)
        assert np.array_equal(samp, ref_samp)
    orc.set_threads(1)


# --------------------------------------------------------------------- rng.rs
def test_rng_goldens(orc):
    o = orc.shuffled_order(100, 42)  # rng.rs:74-120
    assert sorted(int(x) for x in o) == list(range(100))
    assert list(orc.shuffled_order(50, 7)) == list(orc.shuffled_order(50, 7))
    assert list(orc.shuffled_order(50, 7)) != list(orc.shuffled_order(50, 8))
    s = orc.sample_indices(100, 10, 7)
    assert len(s) == 10 and all(i < 100 for i in s) and all(a < b for a, b in zip(s, s[1:]))
    assert orc.sample_indices(100, 10, 7) == orc.sample_indices(100, 10, 7)
    assert orc.sample_indices(100, 10, 7) != orc.sample_indices(100, 10, 8)
    assert orc.sample_indices(100, 10) == orc.sample_indices(100, 10)
    assert orc.sample_indices(4, 1000, 1) == [0, 1, 2, 3]
    assert orc.sample_indices(0, 5, 1) == []


def test_splitmix_first_value(orc):
    # SplitMix64 from state 0 (rng.rs:21-28): the first output is the published
    # splitmix64 test value 0xE220A8397B1DCDAF.  shuffled_order(2, s) swaps
    # iff next(s ^ 0xD1B5...) % 2 == 1; choose s so the folded state is 0.
    seed = 0xD1B54A32D192ED03
    first = 0xE220A8397B1DCDAF
    assert list(orc.shuffled_order(2, seed)) == ([1, 0] if first % 2 == 0 else [0, 1])


# ------------------------------------------------------- NetworkX cross-check
@pytest.fixture(scope="module")
def nxg(orc):
    with open(os.path.join(GOLDEN, "networkx_gnp100.json")) as f:
        g = json.load(f)
    dense = {k: v for k, v in g["dense_ids"]}
    src = [dense[a] for a, _ in g["edges"]]
    dst = [dense[b] for _, b in g["edges"]]
    t = orc.Topology(len(dense), src, dst)
    return g, dense, t


def test_networkx_pagerank(orc, nxg):
    g, dense, t = nxg  # test_networkx_reference.py:53-59
    pr = orc.pagerank(t, 0.85, 500, 1e-12)
    for k, v in g["pagerank"].items():
        assert abs(pr[dense[int(k)]] - v) < 1e-6


def test_networkx_betweenness(orc, nxg):
    g, dense, t = nxg  # :62-68
    bc = orc.betweenness(t)
    for k, v in g["betweenness"].items():
        assert abs(bc[dense[int(k)]] - v) < 1e-6


def test_networkx_triangles_clustering(orc, nxg):
    g, dense, t = nxg  # :82-97
    tc = orc.triangle_count(t)
    cl = orc.clustering_coefficient(t)
    for k, v in g["triangles"].items():
        assert tc[dense[int(k)]] == v
    for k, v in g["clustering"].items():
        assert abs(cl[dense[int(k)]] - v) < 1e-9


def test_networkx_weak_components(orc, nxg):
    g, dense, t = nxg
    cc = orc.connected_components_weak(t)
    inv = {v: k for k, v in dense.items()}
    groups = {}
    for i, l in enumerate(cc):
        groups.setdefault(int(l), []).append(inv[i])
    assert sorted(sorted(x) for x in groups.values()) == g["weak_components"]


def test_idmap_goldens(orc):
    """IdMap interning, the reference's own cases (id_map.rs:469-575)."""
    users, sd, dd = orc.idmap_build([10, 10, 20, 30], [20, 30, 30, 10])  # :470-477
    assert list(users) == [10, 20, 30]
    assert list(sd) == [0, 0, 1, 2] and list(dd) == [1, 2, 2, 0]
    # chunks intern like their concatenation (:529-550): the oracle takes
    # the concatenation, the device path is tested chunk by chunk
    users, sd, dd = orc.idmap_build([], [])  # :569-573
    assert users.size == 0 and sd.size == 0 and dd.size == 0
    # first-seen order over src, dst interleaved (from_ids order, :460-467)
    users, _, _ = orc.idmap_build([100, 100, 7], [7, 42, 100])
    assert list(users) == [100, 7, 42]


def test_closeness_goldens(orc):
    """algo/closeness.rs tests."""
    T = orc.Topology
    c = orc.closeness(T(3, [0, 1, 2], [1, 2, 0]))  # directed triangle
    assert all(abs(x - 2.0 / 3.0) < 1e-12 for x in c)
    c = orc.closeness(T(4, [0, 1, 2], [1, 2, 3]))  # directed line
    assert abs(c[0] - 0.5) < 1e-12 and abs(c[1] - 2.0 / 3.0) < 1e-12 and abs(c[2] - 1.0) < 1e-12 and c[3] == 0.0
    assert orc.closeness(T(0, [], [])).size == 0
    c = orc.closeness(T(100, list(range(100)), [(i + 1) % 100 for i in range(100)]))
    assert all(abs(x - c[0]) < 1e-12 for x in c) and c[0] > 0.0
    c = orc.closeness_weighted(T(3, [0, 1, 0], [1, 2, 2]), [1.0, 1.0, 5.0])
    assert abs(c[0] - 2.0 / 3.0) < 1e-12 and abs(c[1] - 1.0) < 1e-12
    c = orc.closeness_weighted(T(3, [0, 1], [1, 2]), [0.0, 1.0])  # zero-weight reachable node counted
    assert abs(c[0] - 2.0) < 1e-12 and abs(c[1] - 1.0) < 1e-12
    c = orc.closeness_weighted(T(3, [0, 0], [1, 2]), [0.0, 0.0])
    assert c[0] == 0.0


def test_path_stats_goldens(orc):
    """ursa-plan/src/stats.rs tests."""
    T = orc.Topology
    tri = T(3, [0, 1, 2], [1, 2, 0])
    assert abs(orc.avg_path_length(tri) - 1.5) < 1e-12
    assert orc.diameter(tri, False) == 2 and orc.diameter(tri, True) <= 2
    assert orc.diameter(T(4, [0, 1, 2], [1, 2, 3]), False) == 3
    two = T(4, [0, 2], [1, 3])
    assert abs(orc.avg_path_length(two) - 1.0) < 1e-12 and orc.diameter(two, False) == 1


def test_closeness_sources_matches_full(orc):
    from cases import random_graph

    n, s, d = random_graph(500, 2000, 11)
    t = orc.Topology(n, s, d)
    full = orc.closeness(t)
    src = np.array([0, 7, 499, 250, 7], np.uint32)
    assert np.array_equal(orc.closeness_sources(t, src), full[src])
