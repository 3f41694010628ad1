"""The serving loop (ursa_gpu_server_*) vs the oracle and the plain kernels.

  * shortest_path: None exactly when the oracle's shortest_path is None
    (ursa-core/src/algo/bfs.rs:48-102); otherwise a valid path over
    out-edges from source to target with the oracle's hop count;
  * hop: k_hop(&[seed], k) of the oracle and of the plain kernel, pair for
    pair in the reference's emission order (algo/hop.rs:52-130);
  * bfs: bfs_distances(source, direction) of the oracle, exactly, in every
    direction (ursa-core/src/algo/bfs.rs:18-42), out-of-range sources all -1;
  * pagerank on uploaded graphs: the oracle within the plain kernel's bounds
    (fixed iterations: max relative error <= 2e-6, L1 <= 1e-6);
  * the one-query bidirectional shortest_path entry point returns exactly a
    server's path (the same algorithm, no batching);
  * alone == in the mix: every query's result is bit-identical when it runs
    by itself and when it runs among hundreds of concurrent queries of all
    types;
  * cancellation, upload admission by budget, release;
  * bounded waits: with the heartbeat stalled from the host, the slot
    kernels give up after the configured limit, the server counts the
    expiry, and the next query relaunches the lane.
"""

import numpy as np
import pytest

from cases import random_graph

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def resident():
    from ursa_b200 import Topology, gen

    n, s, d = gen.rmat(14, 8, 21)
    # a few extra components: a chain (long paths) and a pair
    chain = np.arange(n, n + 40, dtype=np.uint32)
    s = np.concatenate([s, chain[:-1], np.array([n + 41], np.uint32)])
    d = np.concatenate([d, chain[1:], np.array([n + 40], np.uint32)])
    n2 = n + 42
    return n2, s, d, Topology.build(n2, s, d)


@pytest.fixture(scope="module")
def otopo(orc, resident):
    n, s, d, _ = resident
    return orc.Topology(n, s, d)


def _server(resident, **kw):
    from ursa_b200.serve import Server

    opts = dict(path_lanes=3, path_slots=8, hop_lanes=3, hop_slots=8, pr_lanes=2, pr_slots=16,
                pr_max_nodes=1 << 16, hbm_reserve_bytes=1 << 30, bfs_lanes=2, bfs_slots=8)
    opts.update(kw)
    return Server(resident[3], **opts)


def _path_queries(n, seed=5, count=120):
    rng = np.random.default_rng(seed)
    q = [(int(a), int(b)) for a, b in zip(rng.integers(0, n, count), rng.integers(0, n, count))]
    q += [(7, 7), (n + 5, 3), (3, n + 5), (n - 42, n - 3), (n - 3, n - 42), (n - 1, n - 2), (n - 2, n - 1)]
    return q


def _check_path(orc, otopo, out, s, t, path):
    ref = orc.shortest_path(otopo, s, t)
    if ref is None:
        assert path is None, (s, t, path)
        return
    assert path is not None, (s, t)
    assert len(path) == len(ref), (s, t, len(path), len(ref))
    assert int(path[0]) == s and int(path[-1]) == t
    off, tgt = out
    for a, b in zip(path[:-1], path[1:]):
        assert b in tgt[off[a]:off[a + 1]], (s, t, a, b)


def test_shortest_path_vs_oracle(orc, resident, otopo):
    n = resident[0]
    off, tgt = otopo.csr("out")[:2]
    with _server(resident) as srv:
        qs = _path_queries(n)
        tickets = [srv.shortest_path(a, b) for a, b in qs]
        for (a, b), tk in zip(qs, tickets):
            r = srv.result(tk)
            assert r.status == 0
            _check_path(orc, otopo, (off, tgt), a, b, r.result)


def test_hop_matches_plain_and_oracle(orc, resident, otopo):
    from ursa_b200 import algo

    n, _, _, topo = resident
    rng = np.random.default_rng(9)
    seeds = [int(x) for x in rng.integers(0, n, 60)] + [0, 1, n - 42, n + 3]
    with _server(resident) as srv:
        for k in (1, 2, 3):
            tickets = [srv.hop(x, k) for x in seeds]
            for x, tk in zip(seeds, tickets):
                r = srv.result(tk)
                assert r.status == 0
                _, plain = algo.k_hop(topo, [x], k)
                _, ref = orc.k_hop(otopo, [x], k)
                assert np.array_equal(r.result, plain), (x, k)
                assert np.array_equal(r.result, ref), (x, k)


def test_bfs_vs_oracle(orc, resident, otopo):
    from ursa_b200 import algo

    n, _, _, topo = resident
    rng = np.random.default_rng(17)
    srcs = [int(x) for x in rng.integers(0, n, 40)] + [0, n - 42, n - 1, n + 7]
    names = {0: "out", 1: "in", 2: "both"}
    with _server(resident) as srv:
        for d in (0, 1, 2):
            tickets = [srv.bfs(x, d) for x in srcs]
            for x, tk in zip(srcs, tickets):
                r = srv.result(tk)
                assert r.status == 0 and r.result.dtype == np.int32 and r.result.size == n
                if x >= n:
                    assert np.all(r.result == -1)
                    continue
                ref = orc.bfs_distances(otopo, x, names[d])
                assert np.array_equal(r.result, ref), (x, d)
                if d == 0 and x % 5 == 0:
                    assert np.array_equal(r.result, algo.bfs_distances(topo, x, "out")), x


def test_bidirectional_plain_call_equals_server_path(orc, resident, otopo):
    from ursa_b200 import algo

    n, _, _, topo = resident
    off, tgt = otopo.csr("out")[:2]
    qs = _path_queries(n, seed=11, count=60)
    with _server(resident) as srv:
        tickets = [srv.shortest_path(a, b) for a, b in qs]
        for (a, b), tk in zip(qs, tickets):
            r = srv.result(tk)
            plain = algo.shortest_path_bidirectional(topo, a, b)
            if r.result is None:
                assert plain is None, (a, b)
            else:
                assert plain == [int(x) for x in r.result], (a, b)
            _check_path(orc, otopo, (off, tgt), a, b, None if plain is None else np.array(plain, np.uint32))


def test_heartbeat_expiry_is_counted_and_recovered(resident):
    """The scheduler bumps the heartbeat only every 10 s here, and the slot
    kernels wait at most 50 ms for a bump: they return on their own, the
    server counts the expiry, and a later query relaunches the lane."""
    import time

    from ursa_b200 import algo

    n, _, _, topo = resident
    with _server(resident, path_lanes=1, path_slots=2, hop_lanes=1, hop_slots=2,
                 heartbeat_limit_ns=50_000_000, heartbeat_period_us=10_000_000) as srv:
        r = srv.result(srv.hop(3, 2))
        assert r.status == 0
        deadline = time.time() + 5.0
        while srv.stats()["wait_expiries"] == 0 and time.time() < deadline:
            time.sleep(0.05)
        assert srv.stats()["wait_expiries"] >= 1
        r2 = srv.result(srv.hop(5, 2))
        assert r2.status == 0
        assert np.array_equal(r2.result, algo.k_hop(topo, [5], 2)[1])


def _uploads(count=12, seed=31):
    from ursa_b200 import gen

    n, k, s, d = gen.rmat_batch(count, median=800.0, hi=20000, seed0=seed)
    off = np.concatenate([[0], np.cumsum(k)]).astype(np.int64)
    gs = [(int(n[i]), s[off[i]:off[i + 1]], d[off[i]:off[i + 1]]) for i in range(count)]
    gs.append(random_graph(3000, 40000, 7))
    gs.append((5, np.array([0, 1, 3], np.uint32), np.array([1, 2, 4], np.uint32)))
    return gs


def test_pagerank_on_uploads_vs_oracle(orc, resident):
    gs = _uploads()
    with _server(resident) as srv:
        ids = [srv.upload(*g) for g in gs]
        tickets = [srv.pagerank(i, max_iter=25, tol=0.0) for i in ids]
        for g, tk in zip(gs, tickets):
            r = srv.result(tk)
            assert r.status == 0 and r.iterations == 25
            ref = orc.pagerank(orc.Topology(*g), 0.85, 25, 0.0)
            l1 = float(np.abs(r.result - ref).sum())
            maxrel = float((np.abs(r.result - ref) / np.maximum(np.abs(ref), 1e-300)).max())
            assert l1 <= 1e-6 and maxrel <= 2e-6, (l1, maxrel)
        for i in ids:
            srv.release(i)
        assert srv.stats()["uploads_live"] == 0


def _same(a, b):
    if a.result is None or b.result is None:
        return a.result is None and b.result is None
    return a.result.dtype == b.result.dtype and np.array_equal(a.result.view(np.uint8), b.result.view(np.uint8))


def test_alone_equals_in_mix(resident):
    """Each query run by itself (nothing else on the server) gives the
    bit-identical result it gives among hundreds of concurrent queries."""
    n = resident[0]
    gs = _uploads(8, seed=77)
    rng = np.random.default_rng(123)
    with _server(resident, path_slots=4, hop_slots=4, pr_slots=4) as srv:
        ids = [srv.upload(*g) for g in gs]
        mix = []
        for i in range(360):
            r = rng.random()
            if r < 0.42:
                mix.append(("path", int(rng.integers(0, n)), int(rng.integers(0, n))))
            elif r < 0.5:
                mix.append(("bfs", int(rng.integers(0, n)), int(rng.integers(0, 3))))
            elif r < 0.8:
                mix.append(("hop", int(rng.integers(0, n)), 2))
            else:
                mix.append(("pr", ids[int(rng.integers(0, len(ids)))], 0))

        def submit(q):
            if q[0] == "path":
                return srv.shortest_path(q[1], q[2])
            if q[0] == "hop":
                return srv.hop(q[1], q[2])
            if q[0] == "bfs":
                return srv.bfs(q[1], q[2])
            return srv.pagerank(q[1], max_iter=100, tol=1e-7)

        alone = [srv.result(submit(q)) for q in mix]
        before = srv.stats()["launches"]
        tickets = [submit(q) for q in mix]
        together = [srv.result(t) for t in tickets]
        launches = srv.stats()["launches"] - before
        for q, a, b in zip(mix, alone, together):
            assert a.status == 0 and b.status == 0, q
            assert _same(a, b), q
            assert a.iterations == b.iterations, q
        # the mix really ran batched: queries shared launches, and launches
        # of different lanes were on the GPU at the same time
        assert launches < len(mix) / 2, launches
        spans = sorted((b.launch_us, b.done_us) for b in together)
        overlapping = sum(1 for x, y in zip(spans[:-1], spans[1:]) if y[0] < x[1])
        assert overlapping > 0
        for i in ids:
            srv.release(i)


def test_cancel_pending_queries(resident):
    n = resident[0]
    with _server(resident, path_lanes=1, path_slots=1, hop_lanes=1, hop_slots=1) as srv:
        rng = np.random.default_rng(3)
        tickets = [srv.hop(int(x), 3) for x in rng.integers(0, n, 200)]
        for t in tickets[100:]:
            srv.cancel(t)
        results = [srv.result(t) for t in tickets]
        cancelled = [r for r in results if r.status == 7]
        assert len(cancelled) >= 50
        assert all(r.status in (0, 7) for r in results)


def test_upload_admission_by_budget(resident):
    from ursa_b200 import UrsaGpuError

    g = _uploads(1, seed=5)[0]
    with _server(resident, upload_budget_bytes=48 * len(g[1]) + 96 * g[0] + (1 << 20) + 1000) as srv:
        a = srv.upload(*g)
        with pytest.raises(UrsaGpuError, match="ENOMEM"):
            srv.upload(*g)
        assert srv.stats()["uploads_rejected"] == 1
        t = srv.pagerank(a)
        srv.release(a)  # waits for the query holding it
        assert srv.result(t).status == 0
        b = srv.upload(*g)  # admitted again once the first is gone
        srv.release(b)


def test_bad_queries_are_rejected(resident):
    from ursa_b200 import UrsaGpuError

    with _server(resident) as srv:
        with pytest.raises(UrsaGpuError, match="EINVAL"):
            srv.pagerank(12345)
        with pytest.raises(UrsaGpuError, match="EINVAL"):
            srv.upload((1 << 16) + 1, [0], [1])
