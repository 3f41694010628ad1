"""Node-id interning on the device (ursa_gpu_idmap_*) vs the oracle's
restatement of IdMap::from_edge_batches (ursa-core/src/id_map.rs:197-440).

Bit-exact: the user ids in dense order, the dense edge columns, lookups
(None for unknown ids) and gathers; a topology built from the device
columns equals Topology::build over the dense columns.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

I64_MIN, I64_MAX = np.iinfo(np.int64).min, np.iinfo(np.int64).max


def _check(orc, src, dst, chunks=None):
    from ursa_b200.idmap import IdMap

    m = IdMap.from_edge_batches(chunks) if chunks is not None else IdMap.from_edge_arrays(src, dst)
    users, sd, dd = orc.idmap_build(src, dst)
    assert len(m) == users.size
    assert np.array_equal(m.user_id_array(), users)
    gs, gd = m.dense_edges()
    assert np.array_equal(gs, sd) and np.array_equal(gd, dd)
    return m


def test_reference_goldens(orc):
    m = _check(orc, [10, 10, 20, 30], [20, 30, 30, 10])  # id_map.rs:470-477
    assert list(m.dense_edges()[0]) == [0, 0, 1, 2] and list(m.dense_edges()[1]) == [1, 2, 2, 0]
    # the same graph split across two chunks interns identically (:529-550)
    c = _check(orc, [10, 10, 20, 30], [20, 30, 30, 10], chunks=[([10, 10], [20, 30]), ([20, 30], [30, 10])])
    assert list(c.user_id_array()) == [10, 20, 30]


def test_empty_map(orc):
    from ursa_b200.idmap import IdMap

    m = IdMap.from_edge_batches([])  # :569-573
    assert len(m) == 0 and m.n_edges() == 0
    m2 = IdMap.from_edge_arrays([], [])
    assert len(m2) == 0


def test_length_mismatch_is_rejected():
    from ursa_b200.idmap import IdMap

    with pytest.raises(ValueError):
        IdMap.from_edge_arrays([1, 2, 3], [1, 2])  # :576-583


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_ids_with_extremes(orc, seed):
    rng = np.random.default_rng(seed)
    pool = np.concatenate([rng.integers(I64_MIN, I64_MAX, 5000, dtype=np.int64),
                           np.array([-1, 0, 1, I64_MIN, I64_MAX, -2], np.int64)])
    src = pool[rng.integers(0, pool.size, 40_000)]
    dst = pool[rng.integers(0, pool.size, 40_000)]
    m = _check(orc, src, dst)
    cuts = sorted(rng.integers(0, src.size, 5))
    chunks = [(a, b) for a, b in zip(np.split(src, cuts), np.split(dst, cuts))]
    c = _check(orc, src, dst, chunks=chunks)
    assert np.array_equal(c.user_id_array(), m.user_id_array())


def test_lookup_and_gather(orc):
    from ursa_b200.idmap import IdMap

    src = np.array([5, -1, 9, I64_MAX], np.int64)
    dst = np.array([-1, 9, 5, 7], np.int64)
    m = IdMap.from_edge_arrays(src, dst)
    users = m.user_id_array()
    assert list(users) == [5, -1, 9, I64_MAX, 7]
    assert m.dense_from_array([7, 5, 12345, -1, I64_MIN]) == [4, 0, None, 1, None]
    assert m.dense_from_array([]) == []
    assert list(m.gather_user([4, 0, 1])) == [7, 5, -1]


def test_topology_from_device_columns(orc):
    from ursa_b200 import Topology, gen
    from ursa_b200.idmap import IdMap

    n, s, d = gen.rmat(14, 8, 3)
    rng = np.random.default_rng(7)
    label = rng.permutation(np.arange(n, dtype=np.int64) * 7919 - 10**12)
    src, dst = label[s], label[d]
    m = _check(orc, src, dst)
    t = m.topology()
    ds, dd = m.dense_edges()
    ref = Topology.build(len(m), ds, dd)
    for direction in ("out", "in"):
        a, b = t.out() if direction == "out" else t.incoming(), ref.out() if direction == "out" else ref.incoming()
        assert np.array_equal(a.offsets, b.offsets)
        assert np.array_equal(a.targets, b.targets)
        assert np.array_equal(a.edge_ids, b.edge_ids)


def test_rmat20_scale(orc):
    """R-MAT-20 edges (about 16M rows) under scrambled 64-bit ids."""
    from ursa_b200 import gen

    n, s, d = gen.rmat(20, 16, 5)
    rng = np.random.default_rng(11)
    label = rng.integers(I64_MIN, I64_MAX, n, dtype=np.int64)
    _check(orc, label[s], label[d])
