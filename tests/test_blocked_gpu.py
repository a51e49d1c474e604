"""The slice-blocked sweep (pr_gpu_set_sweep_layout): its layout and its
results, through the C ABI.

  * the layout itself: the number of (row, slice) pairs the device built
    equals a CPU count over the degree-renumbered in-CSR (rows and slices as
    the engine defines them: vertices in descending in-degree order, ties by
    id; slice = new id // slice_verts; a pair longer than 2048 ids stored as
    pieces of 2048);
  * results against the oracle, with the plain parity tolerances (sweep count
    of the reference, per vertex 2e-5 relative + 1e-10 of FP64, L1 at most
    4x the reference's own FP32 L1 + 1e-7), on graphs shaped to stress the
    layout: one hub row holding a third of all edges (a pair spanning many
    32-lane windows and CTA units), isolated vertices, a directed graph with
    sinks and sources, slices and bins as small as the engine accepts;
  * single-column personalized PageRank on the blocked path against the
    FP64 oracle (the PPR tolerances of test_ppr_gpu.py);
  * the gather and blocked sweeps give the same sweep count and agree per
    vertex within 2e-5 relative; each is bit-reproducible;
  * argument checks: bad layout settings and a weighted graph under
    PR_GPU_SWEEP_BLOCKED return PR_GPU_EINVAL.
"""
import numpy as np
import pytest

import oracle
from gapbs_b200 import PageRankEngine
from gapbs_b200.graph import Graph, make_graph
from gapbs_b200.pagerank import PageRankError
from conftest import gpu_available
from helpers import seed_teleports

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    if not gpu_available():
        pytest.skip("no CUDA device")
    eng = PageRankEngine(0)
    yield eng
    eng.close()


MAX_PAIR_IDS = 2048  # longer (row, slice) pairs are stored as pieces of this many ids


def cpu_pair_count(g, slice_verts):
    """(row, slice) pairs of the degree-renumbered in-CSR, a pair of L ids
    counting as ceil(L / 2048) pieces."""
    n = g.num_nodes
    deg = np.diff(g.in_offsets)
    order = np.argsort(-deg, kind="stable")          # new -> old
    inv = np.empty(n, np.int64)
    inv[order] = np.arange(n)
    rows = inv[np.repeat(np.arange(n), deg)]
    slices = inv[g.in_neighbors] // slice_verts
    _, counts = np.unique(rows * (n // slice_verts + 2) + slices, return_counts=True)
    return int(((counts + MAX_PAIR_IDS - 1) // MAX_PAIR_IDS).sum())


def check_plain(engine, g, max_iters=20, epsilon=1e-4):
    res = engine.run(max_iters, epsilon)
    s32, k32, _ = oracle.pr_pull_f32(g, max_iters, epsilon)
    s64, _, _ = oracle.pr_pull_f64(g, max_iters, epsilon)
    assert int(res.sweeps[0]) == k32
    gpu = res.scores
    assert np.all(np.abs(gpu - s64) <= 2e-5 * np.abs(s64) + 1e-10)
    ref_l1 = float(np.abs(s32.astype(np.float64) - s64).sum())
    gpu_l1 = float(np.abs(gpu.astype(np.float64) - s64).sum())
    assert gpu_l1 <= 4 * ref_l1 + 1e-7, (gpu_l1, ref_l1)
    return res


def skewed_graph(seed=7, n=6000, m=60000):
    rng = np.random.default_rng(seed)
    u = rng.integers(0, n, m)
    v = rng.integers(0, n, m)
    u[: m // 3] = 5                       # one row with a third of the edges
    u[m // 3: m // 3 + 200] = n + 100     # and some isolated ids below n + 100
    return Graph.from_edges(u, v, symmetrize=True)


CASES = {
    "g14": lambda: make_graph("-g 14"),
    "u13": lambda: make_graph("-u 13"),
    "skewed": skewed_graph,
    "directed": lambda: Graph.from_edges(*np.random.default_rng(9).integers(0, 4000, (2, 30000))),
}


@pytest.mark.parametrize("slice_verts,bin_words", [(64, 1024), (128, 4096), (0, 0)])
@pytest.mark.parametrize("case", sorted(CASES))
def test_blocked_layout_and_results(engine, case, slice_verts, bin_words):
    g = CASES[case]()
    engine.set_sweep_layout("blocked", slice_verts, bin_words)
    engine.upload(g)
    info = engine.sweep_layout_info()
    assert info["blocked"]
    sv = slice_verts or 49152
    assert info["pairs"] == cpu_pair_count(g, sv)
    res = check_plain(engine, g)
    assert engine.sweep_layout_info()["last_run_blocked"]
    again = engine.run(20, 1e-4)
    assert np.array_equal(res.scores.view(np.uint32), again.scores.view(np.uint32))
    assert np.array_equal(res.err_trace, again.err_trace)
    engine.set_sweep_layout("gather")
    gat = engine.run(20, 1e-4)
    assert not engine.sweep_layout_info()["last_run_blocked"]
    assert int(gat.sweeps[0]) == int(res.sweeps[0])
    assert np.all(np.abs(gat.scores - res.scores) <= 2e-5 * np.abs(gat.scores) + 1e-10)
    engine.set_sweep_layout("auto")


def test_blocked_single_column_ppr(engine):
    g = make_graph("-g 13")
    engine.set_sweep_layout("blocked", 64, 2048)
    engine.upload(g)
    T = seed_teleports(g, 3, np.random.default_rng(4))
    n = g.num_nodes
    for c in range(3):
        res = engine.run(20, 1e-4, teleport=np.ascontiguousarray(T[:, c]))
        assert engine.sweep_layout_info()["last_run_blocked"]
        t = T[:, c].astype(np.float64)
        _, k_own, _ = oracle.ppr_f64(n, g.in_offsets, g.in_neighbors, g.out_offsets, t,
                                     max_iters=20, epsilon=1e-4)
        kg = int(res.sweeps[0])
        assert abs(kg - k_own) <= 1
        s64, _, _ = oracle.ppr_f64(n, g.in_offsets, g.in_neighbors, g.out_offsets, t,
                                   max_iters=kg, epsilon=0.0)
        assert float(np.abs(res.scores - s64).sum()) <= 2e-6
        assert np.all(np.abs(res.scores - s64) <= 2e-5 * np.abs(s64) + 1e-9)
    engine.set_sweep_layout("auto")


def test_blocked_zero_iterations_and_epsilon_zero(engine):
    g = make_graph("-g 11")
    engine.set_sweep_layout("blocked", 64, 1024)
    engine.upload(g)
    res = engine.run(0, 1e-4)
    assert int(res.sweeps[0]) == 0
    assert np.all(res.scores == np.float32(1.0) / np.float32(g.num_nodes))
    res = check_plain(engine, g, max_iters=15, epsilon=0.0)
    assert int(res.sweeps[0]) == 15
    engine.set_sweep_layout("auto")


def test_layout_argument_checks(engine):
    with pytest.raises(PageRankError) as ei:
        engine.set_sweep_layout("blocked", 100, 0)     # not a multiple of 64
    assert ei.value.code == -1
    with pytest.raises(PageRankError) as ei:
        engine.set_sweep_layout("blocked", 0, 512)     # bins too small
    assert ei.value.code == -1
    g = make_graph("-g 10")
    ew = np.random.default_rng(2).uniform(0.5, 1.5, g.num_edges_directed).astype(np.float32)
    engine.set_sweep_layout("blocked")
    engine.upload(g, edge_w=ew)
    with pytest.raises(PageRankError) as ei:
        engine.run(20, 1e-4)                          # weighted: gather only
    assert ei.value.code == -1
    engine.set_sweep_layout("auto")
    engine.run(20, 1e-4)                              # auto falls back to gather
    assert not engine.sweep_layout_info()["last_run_blocked"]


def test_sweep_kernel_times(engine):
    """pr_gpu_sweep_kernel_times: three kernels per slice-blocked sweep, one
    per gather sweep, each with a positive time, the same sweep count as a
    regular solve, and the regular solve's bits unchanged after it."""
    g = make_graph("-g 14")
    engine.set_sweep_layout("blocked", 128, 4096)
    engine.upload(g)
    before = engine.run(20, 1e-4)
    ms, sweeps = engine.sweep_kernel_times(20, 1e-4)
    assert len(ms) == 3 and all(t > 0 for t in ms)
    assert sweeps == int(before.sweeps[0])
    after = engine.run(20, 1e-4)
    assert np.array_equal(before.scores.view(np.uint32), after.scores.view(np.uint32))
    engine.set_sweep_layout("gather")
    ms, sweeps = engine.sweep_kernel_times(20, 1e-4)
    assert len(ms) == 1 and ms[0] > 0 and sweeps == int(before.sweeps[0])
    with pytest.raises(PageRankError) as ei:
        engine.sweep_kernel_times(-1, 1e-4)
    assert ei.value.code == -1
    engine.set_sweep_layout("auto")


def test_auto_rule(engine):
    """PR_GPU_SWEEP_AUTO keeps the gather sweep on graphs below 48 Mi edges
    and where nearly every in-edge is a (row, slice) pair of its own (a
    uniform graph cut into 64-vertex slices), where PR_GPU_SWEEP_BLOCKED
    still builds the layout and matches the oracle; it takes the layout on
    a Kronecker graph of 64 M edges."""
    g = make_graph("-u 14")
    engine.set_sweep_layout("auto", 64, 2048)
    engine.upload(g)
    assert not engine.sweep_layout_info()["blocked"]
    check_plain(engine, g)
    assert not engine.sweep_layout_info()["last_run_blocked"]
    engine.set_sweep_layout("blocked", 64, 2048)
    info = engine.sweep_layout_info()
    assert info["blocked"] and info["pairs"] > g.num_edges_directed // 2
    assert info["pairs"] == cpu_pair_count(g, 64)
    check_plain(engine, g)
    assert engine.sweep_layout_info()["last_run_blocked"]
    engine.set_sweep_layout("auto")
    engine.upload(make_graph("-g 14"))              # small: gather
    assert not engine.sweep_layout_info()["blocked"]
    n, m = engine.generate("-g 21")                 # 64 M edges, skewed: the layout
    info = engine.sweep_layout_info()
    assert m >= 48 << 20 and info["blocked"] and info["pairs"] <= m // 2
    res = engine.run(20, 1e-4)
    assert engine.sweep_layout_info()["last_run_blocked"] and int(res.sweeps[0]) > 0
