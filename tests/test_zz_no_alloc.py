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


def _noalloc_labels(g, n):
    import torch

    from ursa_b200 import _lib

    out = torch.full((max(n, 1),), 0xFFFFFFF, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    _lib.check(_lib.load().ursa_gpu_connected_components_weak_noalloc(g.handle, out.data_ptr(), None))
    return out[:n].cpu().numpy().view(np.uint32)


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
