"""Generate tests/golden/networkx_gnp100.json.

This restates the reference's NetworkX cross-check
(tests/test_networkx_reference.py:33-129 in cldixon/ursa): a seeded directed
G(n=100, p=0.05, seed=42) graph, with PageRank, unnormalised betweenness,
triangles and clustering computed by NetworkX.  The fixture is committed so
the oracle (and through it the CUDA path) is pinned without NetworkX on the
machine that runs the tests.

Run:  python tests/golden/make_networkx_golden.py
"""

import json
import os

import networkx as nx


def main() -> None:
    src = nx.gnp_random_graph(100, 0.05, seed=42, directed=True)
    edges = [(int(a), int(b)) for a, b in src.edges()]
    gd = nx.DiGraph()
    gd.add_edges_from(edges)
    gu = nx.Graph()
    gu.add_edges_from(edges)
    # The reference frame interns ids in first-seen order alternating src then
    # dst per row (ursa-core/src/id_map.rs:220-300); the dense index of a user
    # id is therefore its first-appearance rank in that walk.
    dense = {}
    for a, b in edges:
        for x in (a, b):
            if x not in dense:
                dense[x] = len(dense)
    out = {
        "generator": "networkx.gnp_random_graph(100, 0.05, seed=42, directed=True)",
        "networkx_version": nx.__version__,
        "edges": edges,
        "dense_ids": [[k, v] for k, v in dense.items()],
        "pagerank": {str(k): v for k, v in nx.pagerank(gd, alpha=0.85, tol=1e-12, max_iter=1000).items()},
        "betweenness": {
            str(k): v for k, v in nx.betweenness_centrality(gd, normalized=False, endpoints=False).items()
        },
        "triangles": {str(k): v for k, v in nx.triangles(gu).items()},
        "clustering": {str(k): v for k, v in nx.clustering(gu).items()},
        "weak_components": sorted(sorted(int(x) for x in c) for c in nx.weakly_connected_components(gd)),
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "networkx_gnp100.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)
    print("wrote", path, len(edges), "edges")


if __name__ == "__main__":
    main()
