"""Seeded random graphs through every engine path, against the oracle.

Small edge lists with duplicates, self-loops, isolated vertices and several
components, directed and symmetrized, of sizes that put rows in every degree
bin: PageRank (sweep count and the per-vertex tolerance of the plain-PR
tests), connected components (the reference's labels, which the oracle's
Afforest reproduces), and BFS from several sources (the reference's verifier
and exact depths).
"""
import numpy as np
import pytest

import oracle
from gapbs_b200 import PageRankEngine
from gapbs_b200.graph import Graph
from conftest import gpu_available
from helpers import depths_from_parents

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    if not gpu_available():
        pytest.skip("no CUDA device")
    eng = PageRankEngine(0)
    yield eng
    eng.close()


def random_graph(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 3000))
    m = int(rng.integers(1, 8 * n))
    # skewed endpoints (a few hubs), some duplicates and self-loops
    u = (rng.pareto(1.2, m) * n / 20).astype(np.int64) % n
    v = rng.integers(0, n, m)
    if seed % 3 == 0:  # a second component far from the first
        u = np.concatenate([u, n + rng.integers(0, 50, 200)])
        v = np.concatenate([v, n + rng.integers(0, 50, 200)])
    return Graph.from_edges(u.astype(np.int32), v.astype(np.int32), symmetrize=seed % 2 == 0)


@pytest.mark.parametrize("seed", range(24))
def test_random_graph_all_paths(engine, seed):
    g = random_graph(seed)
    engine.upload(g)
    res = engine.run(20, 1e-4)
    s64, _, _ = oracle.pr_pull_f64(g, 20, 1e-4)
    _, k32, _ = oracle.pr_pull_f32(g, 20, 1e-4)
    assert int(res.sweeps[0]) == k32
    assert np.all(np.abs(res.scores - s64) <= 2e-5 * np.abs(s64) + 1e-10)
    assert np.array_equal(engine.connected_components(), oracle.cc_afforest(g))
    rng = np.random.default_rng(seed + 1000)
    for src in rng.integers(0, g.num_nodes, 3):
        src = int(src)
        parent = engine.bfs(src)
        assert oracle.bfs_verify(g, src, parent)
        assert np.array_equal(depths_from_parents(parent, src), oracle.bfs_depths(g, src))
