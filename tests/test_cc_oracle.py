"""The connected-components oracle against the reference's own Afforest.

tests/golden/cc_golden.json holds the reference's labels (src/cc.cc, run by
tests/golden/make_golden.py --cc); the serial restatement in oracle/ must
reproduce them exactly on the graphs the host builder makes, and its labels
must be the smallest vertex id of each component.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from gapbs_b200.graph import Graph, make_graph
from conftest import GOLDEN

with open(os.path.join(GOLDEN, "cc_golden.json")) as fh:
    CASES = json.load(fh)["cases"]


def graph_for(args):
    return make_graph(args.format(graphs=os.path.join(GOLDEN, "graphs")))


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference(name):
    e = CASES[name]
    g = graph_for(e["args"])
    comp = oracle.cc_afforest(g)
    assert comp.size == e["num_nodes"]
    assert hashlib.sha256(comp.tobytes()).hexdigest() == e["labels_sha256"]
    if "labels" in e:
        assert comp.tolist() == e["labels"]
    assert np.unique(comp).size == e["components"]


def test_labels_are_component_minima():
    rng = np.random.default_rng(9)
    g = Graph.from_edges(rng.integers(0, 3000, 2500), rng.integers(0, 3000, 2500), symmetrize=True)
    comp = oracle.cc_afforest(g)
    n = g.num_nodes
    # union-find over the edge list, independent of the restatement
    parent = np.arange(n)

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    src = np.repeat(np.arange(n), np.diff(g.out_offsets))
    for u, v in zip(src, g.out_neighbors):
        ru, rv = find(u), find(v)
        if ru != rv:
            parent[max(ru, rv)] = min(ru, rv)
    expect = np.array([find(x) for x in range(n)], np.int32)
    assert np.array_equal(comp, expect)
