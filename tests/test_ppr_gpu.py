"""GPU parity of personalized PageRank, single column and batched.

Reference: the FP64 oracle (no PPR exists in the reference).  Each column is
compared with the oracle run for the same number of sweeps the GPU ran for
that column (columns retire independently).

Tolerances: sweep count within one of the FP64 oracle's own count (a column
whose L1 change lands within FP32 noise of epsilon may stop one sweep apart);
per column L1(gpu - fp64) <= 2e-6 and |gpu - fp64| <= 2e-5 |fp64| + 1e-9.
"""
import numpy as np
import pytest

import oracle
from gapbs_b200 import PageRankEngine
from gapbs_b200.graph import Graph, make_graph
from conftest import gpu_available
from helpers import in_weights, row_sums, seed_teleports

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    if not gpu_available():
        pytest.skip("no CUDA device")
    eng = PageRankEngine(0)
    yield eng
    eng.close()


def check_columns(g, T, res, in_w=None, rowsum=None, max_iters=20, eps=1e-4):
    n, k = T.shape
    for c in range(k):
        t = T[:, c].astype(np.float64)
        _, k_own, _ = oracle.ppr_f64(n, g.in_offsets, g.in_neighbors, g.out_offsets, t,
                                     in_w=in_w, rowsum=rowsum, max_iters=max_iters, epsilon=eps)
        kg = int(res.sweeps[c])
        assert abs(kg - k_own) <= 1, (c, kg, k_own)
        s64, _, tr = oracle.ppr_f64(n, g.in_offsets, g.in_neighbors, g.out_offsets, t,
                                    in_w=in_w, rowsum=rowsum, max_iters=kg, epsilon=0.0)
        got = res.scores[:, c] if res.scores.ndim == 2 else res.scores
        l1 = float(np.abs(got - s64).sum())
        assert l1 <= 2e-6, (c, l1)
        assert np.all(np.abs(got - s64) <= 2e-5 * np.abs(s64) + 1e-9), c
        np.testing.assert_allclose(res.err_trace[:kg, c], tr, rtol=1e-3, atol=1e-6)


def test_single_column_ppr(engine):
    g = make_graph("-g 12")
    engine.upload(g)
    T = seed_teleports(g, 1, np.random.default_rng(1))
    res = engine.run(20, 1e-4, teleport=T[:, 0])
    check_columns(g, T, res)


@pytest.mark.parametrize("k", [2, 7, 64, 70])
def test_batched_ppr(engine, k):
    g = make_graph("-g 13")
    engine.upload(g)
    T = seed_teleports(g, k, np.random.default_rng(k))
    res = engine.run(20, 1e-4, teleport=T)
    assert res.scores.shape == (g.num_nodes, k)
    check_columns(g, T, res)


def test_batched_columns_retire_independently(engine):
    g = make_graph("-g 12")
    engine.upload(g)
    rng = np.random.default_rng(3)
    T = seed_teleports(g, 16, rng)
    T[:, 0] = np.float32(1.0 / g.num_nodes)     # uniform column converges fastest
    res = engine.run(30, 1e-4, teleport=T)
    assert len(set(res.sweeps.tolist())) > 1
    for c in range(16):
        kc = int(res.sweeps[c])
        assert np.all(res.err_trace[kc:, c] == 0.0)
    check_columns(g, T, res, max_iters=30)


def test_batched_uniform_columns_match_plain(engine):
    g = make_graph("-u 12")
    engine.upload(g)
    n = g.num_nodes
    T = np.full((n, 3), np.float32(1.0 / n))
    res = engine.run(20, 1e-4, teleport=T)
    plain = engine.run(20, 1e-4)
    for c in range(3):
        assert int(res.sweeps[c]) == int(plain.sweeps[0])
        assert np.abs(res.scores[:, c] - plain.scores).max() <= 1e-6 * plain.scores.max()


def test_weighted_ppr(engine):
    g = make_graph("-g 11")
    rng = np.random.default_rng(9)
    ew = rng.uniform(0.5, 1.5, g.num_edges_directed).astype(np.float32)
    engine.upload(g, edge_w=ew)
    T = seed_teleports(g, 5, rng)
    res = engine.run(20, 1e-4, teleport=T)
    check_columns(g, T, res, in_w=in_weights(g, ew), rowsum=row_sums(g, ew))
    res1 = engine.run(20, 1e-4, teleport=T[:, 2])
    check_columns(g, T[:, 2:3], res1, in_w=in_weights(g, ew), rowsum=row_sums(g, ew))


def test_directed_ppr(engine):
    rng = np.random.default_rng(4)
    g = Graph.from_edges(rng.integers(0, 2000, 15000), rng.integers(0, 2000, 15000))
    engine.upload(g)
    T = seed_teleports(g, 4, rng)
    res = engine.run(20, 1e-4, teleport=T)
    check_columns(g, T, res)


def test_batched_schedules(engine):
    """Every work schedule gives the oracle's columns (the schedule only moves
    rows between the lane-group and warp-per-row paths and hub rows in or
    out of L1); the autotuner's choice is one of the allowed values; bad
    settings are refused with PR_GPU_EINVAL."""
    from gapbs_b200.pagerank import PageRankError
    g = make_graph("-g 14")
    engine.upload(g)
    T = seed_teleports(g, 16, np.random.default_rng(6))
    for short_len, l1_kb in [(8, 16), (128, 224), (32, 64)]:
        engine.set_batch_schedule(short_len, l1_kb)
        engine.set_batch_tile(16)
        res = engine.run(20, 1e-4, teleport=T)
        sch = engine.batch_schedule()
        assert sch == {"tile_width": 16, "short_len": short_len, "l1_kb": l1_kb}
        check_columns(g, T, res)
    engine.set_batch_schedule(0, 0)
    engine.set_batch_tile(0)
    res = engine.run(20, 1e-4, teleport=T)
    sch = engine.batch_schedule()
    assert sch["tile_width"] in (8, 16)
    assert sch["short_len"] in (8, 16, 32, 64, 128) and 16 <= sch["l1_kb"] <= 224
    check_columns(g, T, res)
    for bad in [(12, 0), (0, 8), (0, 300)]:
        with pytest.raises(PageRankError) as ei:
            engine.set_batch_schedule(*bad)
        assert ei.value.code == -1
