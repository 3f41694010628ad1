"""Arrow results (ursa_gpu_query_batch / hop_batch / path_batch) vs the
reference's result.rs (ursa-plan/src/result.rs:144-261).

Each column of a batch is bit-identical to the standalone kernel call on the
same topology (the kernels are the same; every one is deterministic), the id
columns are the oracle's IdMap user ids gathered dense -> user, and the
schemas are the reference's (names, types, no nullable field).
"""

import gc

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _graph(scale=11, seed=21):
    from ursa_b200 import gen
    from ursa_b200.idmap import IdMap

    n, s, d = gen.rmat(scale, 8, seed)
    label = np.random.default_rng(seed).permutation(np.arange(n, dtype=np.int64) * 7919 - 10**12)
    us, ud = label[s], label[d]
    ids = IdMap.from_edge_arrays(us, ud)
    return ids, ids.topology(), us, ud


def test_multi_column_batch_is_aligned():
    """result.rs:317-335: (id, deg, pr) over the diamond."""
    import pyarrow as pa

    from ursa_b200.idmap import IdMap
    from ursa_b200.result import OutputColumn, query_batch

    ids = IdMap.from_edge_arrays([0, 0, 1, 2], [1, 2, 2, 0])
    b = query_batch(ids.topology(), ids, [OutputColumn("deg", "degree", direction="out"),
                                          OutputColumn("pr", "pagerank", damping=0.85, max_iter=30, tol=1e-6)])
    assert b.num_columns == 3 and b.num_rows == 3
    assert b.schema.names == ["id", "deg", "pr"]
    assert b.schema.types == [pa.int64(), pa.uint32(), pa.float64()]
    assert not any(f.nullable for f in b.schema)
    assert b.column(0).to_pylist() == [0, 1, 2]
    assert b.column(1).to_pylist() == [2, 1, 1]


def test_query_batch_columns_match_kernels(orc):
    import pyarrow as pa

    from ursa_b200 import algo
    from ursa_b200.result import OutputColumn, query_batch

    ids, g, us, ud = _graph()
    users, _, _ = orc.idmap_build(us, ud)
    w = np.random.default_rng(5).uniform(0.1, 3.0, g.n_edges())
    cols = [
        OutputColumn("deg_in", "degree", direction="in"),
        OutputColumn("deg_both", "degree", direction="both"),
        OutputColumn("pr", "pagerank", damping=0.85, max_iter=100, tol=1e-9),
        OutputColumn("prw", "pagerank", damping=0.85, max_iter=100, tol=1e-9, weights=w),
        OutputColumn("cc", "connected_components"),
        OutputColumn("tri", "triangle_count"),
        OutputColumn("clust", "clustering_coefficient"),
        OutputColumn("bc", "betweenness", sample=0.1, seed=7),
        OutputColumn("bcw", "betweenness", sample=0.1, seed=7, weights=w),
        OutputColumn("clo", "closeness"),
        OutputColumn("clow", "closeness", weights=w),
    ]
    b = query_batch(g, ids, cols)
    assert b.num_rows == g.n_nodes() and b.schema.names == ["id"] + [c.name for c in cols]
    assert np.array_equal(b.column(0).to_numpy(), users)
    want = {
        "deg_in": algo.degree(g, "in"),
        "deg_both": algo.degree(g, "both"),
        "pr": algo.pagerank(g, damping=0.85, max_iter=100, tol=1e-9),
        "prw": algo.pagerank_weighted(g, w, damping=0.85, max_iter=100, tol=1e-9),
        "cc": algo.connected_components_weak(g),
        "tri": algo.triangle_count(g),
        "clust": algo.clustering_coefficient(g),
        "bc": algo.betweenness(g, 0.1, 7),
        "bcw": algo.betweenness_weighted(g, w, 0.1, 7),
        "clo": algo.closeness(g),
        "clow": algo.closeness_weighted(g, w),
    }
    for c in cols:
        got = b.column(c.name).to_numpy()
        ref = np.asarray(want[c.name])
        assert got.dtype == ref.dtype, c.name
        assert np.array_equal(got.view(np.uint8), ref.view(np.uint8)), c.name
    assert b.schema.field("tri").type == pa.uint32() and b.schema.field("clo").type == pa.float64()


def test_query_batch_without_idmap_and_empty():
    import pyarrow as pa

    from ursa_b200 import Topology
    from ursa_b200.result import OutputColumn, query_batch

    g = Topology.build(4, [0, 1, 2], [1, 2, 3])
    b = query_batch(g, None, [OutputColumn("clo", "closeness")])
    assert b.schema.field("id").type == pa.uint32()
    assert b.column(0).to_pylist() == [0, 1, 2, 3]
    assert b.column(1).to_pylist() == [0.5, 2.0 / 3.0, 1.0, 0.0]  # closeness.rs directed line
    e = query_batch(Topology.build(0, [], []), None, [OutputColumn("pr", "pagerank")])
    assert e.num_rows == 0 and e.schema.names == ["id", "pr"]
    assert query_batch(g, None, []).schema.names == ["id"]


def test_host_side_algorithms_are_refused():
    from ursa_b200 import Topology
    from ursa_b200._lib import UrsaGpuError
    from ursa_b200.result import OutputColumn, query_batch

    g = Topology.build(3, [0, 1], [1, 2])
    for col in (OutputColumn("scc", "connected_components", strong=True), OutputColumn("lp", "label_propagation"),
                OutputColumn("lv", "louvain"), OutputColumn("bcw", "closeness", weights=[1.0, -1.0])):
        with pytest.raises(UrsaGpuError):
            query_batch(g, None, [col])


def test_hop_batch(orc):
    import pyarrow as pa

    from ursa_b200 import algo
    from ursa_b200.result import hop_batch

    ids, g, us, ud = _graph()
    users, _, _ = orc.idmap_build(us, ud)
    seeds = [0, 5, 17, 5]
    b = hop_batch(g, ids, seeds, 2, "out")
    sa, ra = algo.k_hop(g, seeds, 2, "out")
    assert b.schema.names == ["src", "dst"] and b.schema.types == [pa.int64(), pa.int64()]
    assert np.array_equal(b.column(0).to_numpy(), users[sa])
    assert np.array_equal(b.column(1).to_numpy(), users[ra])
    assert hop_batch(g, ids, seeds, 0).num_rows == 0  # hop.rs:55-57


def test_path_batch(orc):
    import pyarrow as pa

    from ursa_b200 import algo
    from ursa_b200.result import path_batch

    ids, g, us, ud = _graph()
    users, _, _ = orc.idmap_build(us, ud)
    dist = algo.bfs_distances(g, 0, "out")
    far = int(np.argmax(dist))
    path = algo.shortest_path(g, 0, far, "out")
    b = path_batch(g, ids, 0, far, "out")
    assert b.schema.names == ["src", "dst", "hop", "cost"]
    assert b.schema.types == [pa.int64(), pa.int64(), pa.int64(), pa.float64()]
    assert b.num_rows == len(path) - 1
    assert np.array_equal(b.column("src").to_numpy(), users[np.asarray(path[:-1])])
    assert np.array_equal(b.column("dst").to_numpy(), users[np.asarray(path[1:])])
    assert b.column("hop").to_pylist() == list(range(len(path) - 1))
    assert b.column("cost").to_pylist() == [float(i + 1) for i in range(len(path) - 1)]
    w = np.random.default_rng(9).uniform(0.5, 2.0, g.n_edges())
    wp, wc = algo.shortest_path_weighted_with_cost(g, w, 0, far, "out")
    bw = path_batch(g, ids, 0, far, "out", weights=w)
    assert np.array_equal(bw.column("dst").to_numpy(), users[np.asarray(wp[1:])])
    assert np.array_equal(bw.column("cost").to_numpy(), np.asarray(wc[1:]))
    unreachable = int(np.flatnonzero(dist < 0)[0]) if (dist < 0).any() else None
    if unreachable is not None:
        assert path_batch(g, ids, 0, unreachable).num_rows == 0
    assert path_batch(g, ids, 3, 3).num_rows == 0  # a one-node path has no edge


def test_buffers_outlive_the_handle_and_the_batch():
    """The pinned block stays alive while any exported array uses it; a
    column taken out of the batch outlives the batch."""
    from ursa_b200.result import OutputColumn, query_batch

    ids, g, _, _ = _graph(10, 3)
    b = query_batch(g, ids, [OutputColumn("deg", "degree")])
    col = b.column("deg")
    ref = col.to_numpy().copy()
    del b
    gc.collect()
    for _ in range(3):  # churn the pinned pool with other results
        query_batch(g, ids, [OutputColumn("pr", "pagerank")])
    assert np.array_equal(col.to_numpy(), ref)


def test_gather_user_on_device(orc):
    from ursa_b200._lib import UrsaGpuError

    ids, g, us, ud = _graph(9, 4)
    users, _, _ = orc.idmap_build(us, ud)
    dense = np.random.default_rng(1).integers(0, len(users), 1000).astype(np.uint32)
    assert np.array_equal(ids.gather_user(dense), users[dense])
    with pytest.raises(UrsaGpuError):
        ids.gather_user([len(users)])
