"""The BFS oracle against the reference's own DOBFS.

tests/golden/bfs_golden.json holds, per graph and per source the
reference's SourcePicker yields, the depths along the reference's DOBFS
parent pointers (tests/golden/make_golden.py --bfs).  The oracle's serial
search (the reference verifier's) must give exactly those depths on the
graphs the host builder makes.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from gapbs_b200.graph import make_graph
from conftest import GOLDEN

with open(os.path.join(GOLDEN, "bfs_golden.json")) as fh:
    CASES = json.load(fh)["cases"]


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_depths_match_reference_trees(name):
    e = CASES[name]
    g = make_graph(e["args"].format(graphs=os.path.join(GOLDEN, "graphs")))
    odeg = np.diff(g.out_offsets)
    for run in e["runs"]:
        d = oracle.bfs_depths(g, run["source"])
        assert hashlib.sha256(d.tobytes()).hexdigest() == run["depth_sha256"]
        if "depths" in run:
            assert d.tolist() == run["depths"]
        assert int((d >= 0).sum()) == run["reached"]
        assert int(odeg[d >= 0].sum()) == run["tree_edges"]


def test_verifier_rejects_broken_trees():
    g = make_graph("-g 10")
    src = 351
    d = oracle.bfs_depths(g, src)
    # a valid tree built from the depths: any in-neighbour one level up
    parent = np.full(g.num_nodes, -1, np.int32)
    for v in range(g.num_nodes):
        if v == src:
            parent[v] = src
        elif d[v] > 0:
            nb = g.in_neigh(v)
            parent[v] = next(u for u in nb if d[u] == d[v] - 1)
    assert oracle.bfs_verify(g, src, parent)
    bad = parent.copy()
    v = int(np.nonzero(d == 2)[0][0])
    bad[v] = src if d[v] != 1 else bad[v]  # a parent two levels up
    assert not oracle.bfs_verify(g, src, bad)
    bad = parent.copy()
    bad[int(np.nonzero(d >= 1)[0][0])] = -1  # a reached vertex without parent
    assert not oracle.bfs_verify(g, src, bad)
