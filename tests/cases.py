"""Shared graph cases for the parity tests: the reference's hand-built golden
graphs, edge cases (empty, edgeless, self-loops, duplicates, hubs above the
chunking thresholds) and seeded random / R-MAT graphs."""

import numpy as np

from ursa_b200 import gen


def small_cases():
    """(name, n, src, dst) tuples from the reference's unit tests."""
    return [
        ("diamond", 3, [0, 0, 1, 2], [1, 2, 2, 0]),  # topology.rs:438-440
        ("path5", 5, [0, 1, 2, 1], [1, 2, 3, 4]),  # bfs.rs:266-268
        ("hub_sink", 4, [0, 1, 3, 2], [2, 2, 2, 0]),  # pagerank.rs:278
        ("selfloop_dup", 3, [0, 0, 1, 2, 1, 0], [1, 2, 2, 0, 1, 1]),  # topology.rs:503
        ("two_components", 5, [0, 1, 3], [1, 2, 4]),  # components.rs:147
        ("k4", 4, [0, 0, 0, 1, 1, 2], [1, 2, 3, 2, 3, 3]),  # triangle.rs:268-270
        ("line5", 5, [0, 1, 2, 3], [1, 2, 3, 4]),  # betweenness.rs:372
        ("diamond_bc", 4, [0, 0, 1, 2], [1, 2, 3, 3]),  # betweenness.rs:381
        ("cycle80", 80, list(range(80)), [(i + 1) % 80 for i in range(80)]),  # betweenness.rs:426-429
        ("ring7_chords", 7, [0, 1, 2, 3, 4, 5, 6, 0, 2], [1, 2, 3, 4, 5, 6, 0, 3, 5]),
        ("single_edge", 2, [0], [1]),
        ("isolated_nodes", 6, [1, 3], [3, 1]),
        ("edgeless", 4, [], []),
        ("single_node", 1, [], []),
        ("only_selfloops", 3, [0, 1, 1], [0, 1, 1]),
    ]


def random_graph(n, m, seed):
    rng = np.random.default_rng(seed)
    return n, rng.integers(0, n, m, dtype=np.uint32), rng.integers(0, n, m, dtype=np.uint32)


def hub_graph(n_leaves, seed=0, in_hub=True, extra=0):
    """A star plus random edges: the hub's degree crosses the hub thresholds."""
    rng = np.random.default_rng(seed)
    n = n_leaves + 1
    leaves = np.arange(1, n, dtype=np.uint32)
    hub = np.zeros(n_leaves, np.uint32)
    src, dst = (leaves, hub) if in_hub else (hub, leaves)
    if extra:
        src = np.concatenate([src, rng.integers(0, n, extra, dtype=np.uint32)])
        dst = np.concatenate([dst, rng.integers(0, n, extra, dtype=np.uint32)])
    return n, src.astype(np.uint32), dst.astype(np.uint32)


def medium_cases():
    out = []
    for n, m, seed in [(2000, 100_000, 1), (50_000, 300_000, 2), (16, 80_000, 3), (1, 10, 4)]:
        out.append((f"rand_{n}_{m}", *random_graph(n, m, seed)))
    out.append(("hub_in_5000", *hub_graph(5000, 1, True, 20000)))
    out.append(("hub_in_300000", *hub_graph(300_000, 2, True, 50000)))
    out.append(("hub_out_5000", *hub_graph(5000, 3, False, 20000)))
    n, s, d = gen.rmat(14, 16, 7)
    out.append(("rmat14", n, s, d))
    return out


def canon(labels):
    """Relabel components by their minimum member id."""
    labels = np.asarray(labels, dtype=np.int64)
    n = labels.size
    if n == 0:
        return labels.astype(np.uint32)
    first = {}
    out = np.empty(n, np.uint32)
    for i in range(n):
        out[i] = first.setdefault(int(labels[i]), i)
    return out
