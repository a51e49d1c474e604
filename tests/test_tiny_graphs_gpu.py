"""The smallest inputs every engine path must take: graphs without edges (the
builder drops self-loops, so an edge list of one self-loop gives N vertices
and no edges), a single vertex, two vertices, and directed graphs whose only
vertex with out-edges has no in-edges.

PageRank against the oracle (sweep count, scores within the plain-PR
tolerance), connected components against the oracle's Afforest labels, BFS
against the oracle's depths and the reference's verifier, batched PPR against
single-vector solves.
"""
import numpy as np
import pytest

import oracle
from gapbs_b200 import PageRankEngine
from gapbs_b200.graph import Graph
from conftest import gpu_available
from helpers import depths_from_parents

pytestmark = pytest.mark.gpu

GRAPHS = {
    "edgeless5": ([4], [4], True),
    "single": ([0], [0], True),
    "edgeless5_directed": ([4], [4], False),
    "pair": ([0], [1], True),
    "pair_directed": ([0], [1], False),
    "two_cycle_directed": ([0, 1], [1, 0], False),
    "source_only_out": ([0, 0, 0, 1], [1, 2, 3, 2], False),
}


@pytest.fixture(scope="module")
def engine():
    if not gpu_available():
        pytest.skip("no CUDA device")
    eng = PageRankEngine(0)
    yield eng
    eng.close()


def build(name):
    u, v, sym = GRAPHS[name]
    return Graph.from_edges(np.array(u), np.array(v), symmetrize=sym)


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_pagerank(engine, name):
    g = build(name)
    engine.upload(g)
    res = engine.run(20, 1e-4)
    s64, k64, _ = oracle.pr_pull_f64(g, 20, 1e-4)
    _, k32, _ = oracle.pr_pull_f32(g, 20, 1e-4)
    assert int(res.sweeps[0]) == k32
    assert np.all(np.abs(res.scores - s64) <= 2e-5 * np.abs(s64) + 1e-10)


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_connected_components(engine, name):
    g = build(name)
    engine.upload(g)
    assert np.array_equal(engine.connected_components(), oracle.cc_afforest(g))


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_bfs_from_every_vertex(engine, name):
    g = build(name)
    engine.upload(g)
    for src in range(g.num_nodes):
        parent = engine.bfs(src)
        assert oracle.bfs_verify(g, src, parent)
        assert np.array_equal(depths_from_parents(parent, src), oracle.bfs_depths(g, src))


@pytest.mark.parametrize("name", ["edgeless5", "pair", "source_only_out"])
def test_batched_ppr_matches_single(engine, name):
    g = build(name)
    engine.upload(g)
    n = g.num_nodes
    tele = np.zeros((n, 4), np.float32)
    for c in range(4):
        tele[c % n, c] = 1.0
    batched = engine.run(20, 1e-4, teleport=tele)
    for c in range(4):
        single = engine.run(20, 1e-4, teleport=np.ascontiguousarray(tele[:, c:c + 1]))
        assert int(batched.sweeps[c]) == int(single.sweeps[0])
        np.testing.assert_allclose(batched.scores[:, c], single.scores[:, 0], rtol=1e-6, atol=1e-9)
