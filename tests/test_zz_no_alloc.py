"""The allocation-free connected-components entry point.

Callers such as a serving loop that has promised all free HBM to resident
graphs, or a host runtime that owns every device byte through its own pool,
cannot let the library allocate during a query.  This checks, through the C
ABI, that ursa_gpu_connected_components_weak_noalloc gives exactly the labels
of the allocating entry point on two calls in a row (the shared scratch
array keeps the previous call's contents, so the second call must not see
them), and that graphs above its 4,194,304-node limit are refused.

The file sorts last so a run that stops at the first failure has already run
every other test.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_labels(g, n, stream=None):
    """Labels through the allocation-free entry point; stream is a torch
    stream whose handle is passed (the caller's stream), or None for the
    library's own stream for this thread."""
    import torch

    from ursa_b200 import _lib

    out = torch.full((max(n, 1),), 0xFFFFFFF, dtype=torch.int32, device="cuda:0")
    torch.cuda.synchronize()
    h = None if stream is None else stream.cuda_stream
    _lib.check(_lib.load().ursa_gpu_connected_components_weak_noalloc(g.handle, out.data_ptr(), h))
    return out[:n].cpu().numpy().view(np.uint32)


def _canon(labels):
    _, first, inv = np.unique(np.asarray(labels, np.int64), return_index=True, return_inverse=True)
    return first[inv]


def test_noalloc_matches_allocating_entry_point_twice():
    from ursa_b200 import Topology, algo, gen

    n1, s1, d1 = gen.rmat(16, 16, 1)  # larger graph first
    rng = np.random.default_rng(5)
    n2 = 5000
    s2 = rng.integers(0, n2, 3000, dtype=np.uint32)
    d2 = rng.integers(0, n2, 3000, dtype=np.uint32)
    for n, s, d in ((n1, s1, d1), (n2, s2, d2)):
        g = Topology.build(n, s, d)
        ref = algo.connected_components_weak(g)
        got = _noalloc_labels(g, n)
        assert np.array_equal(got, ref)
        assert np.array_equal(_noalloc_labels(g, n), ref)  # and again, same graph


def test_noalloc_rejects_oversized_graph():
    import torch

    from ursa_b200 import Topology, UrsaGpuError, _lib

    n = (1 << 22) + 1
    g = Topology.build(n, [0, 1], [1, 2])
    out = torch.zeros(n, dtype=torch.int32, device="cuda")  # a valid buffer all the same
    with pytest.raises(UrsaGpuError, match="at most 4194304"):
        _lib.check(_lib.load().ursa_gpu_connected_components_weak_noalloc(g.handle, out.data_ptr(), None))
    assert int(out.abs().sum()) == 0  # nothing was written


def test_noalloc_on_callers_stream():
    import torch

    from ursa_b200 import Topology, algo, gen

    n, s, d = gen.rmat(15, 16, 4)
    g = Topology.build(n, s, d)
    ref = algo.connected_components_weak(g)
    st = torch.cuda.Stream(device="cuda:0")
    assert np.array_equal(_noalloc_labels(g, n, st), ref)
    assert np.array_equal(_noalloc_labels(g, n, st), ref)


def test_noalloc_at_the_node_limit_matches_oracle(orc):
    """Exactly 4,194,304 nodes (R-MAT scale 22, seed 2): the last entry of the
    scratch array is used; the partition equals the oracle's."""
    from ursa_b200 import Topology, gen

    n, s, d = gen.rmat(22, 16, 2)
    assert n == 1 << 22
    g = Topology.build(n, s, d)
    ref = _canon(orc.connected_components_weak(orc.Topology(n, s, d)))
    assert np.array_equal(_noalloc_labels(g, n), ref)
    assert np.array_equal(_noalloc_labels(g, n), ref)


def test_noalloc_selects_the_topologys_device():
    """With another device current on the calling thread, the call still runs
    on the topology's device (needs two visible GPUs)."""
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible GPUs")
    from ursa_b200 import Topology, algo, gen

    n, s, d = gen.rmat(12, 16, 1)
    g = Topology.build(n, s, d)  # on device 0
    ref = algo.connected_components_weak(g)
    st = torch.cuda.Stream(device="cuda:0")
    torch.cuda.set_device(1)
    try:
        assert np.array_equal(_noalloc_labels(g, n, st), ref)
    finally:
        torch.cuda.set_device(0)
