"""GPU parity of the plain PageRankPull path (through the C ABI).

Checked against the oracle (the FP32 mirror reproduces the reference bit for
bit; the FP64 restatement is the accuracy yardstick) on the reference's own
graphs and on hand-made corner cases.

Every test runs under three sweep layouts: the per-edge gather sweep, the
slice-blocked sweep with its default slices and bins, and the slice-blocked
sweep with 64-vertex slices and 2048-word bins, which cuts even these small
graphs into many slices, bins and CTA units.

Tolerances (FP32 scores summed in a different order than the reference):
  * sweep count identical to the reference's;
  * L1(gpu - fp64) <= 4 * L1(reference_fp32 - fp64) + 1e-7;
  * |gpu - fp64| <= 2e-5 * |fp64| + 1e-10 per vertex;
  * PRVerifier total error < epsilon (the reference's pass criterion);
  * per-sweep L1 changes within 1e-5 relative + 5 (R_k + R_(k-1)) of the
    reference's, where R_k is the reference's own rounding after sweep k
    (L1 distance of its FP32 scores from FP64 Jacobi run alongside,
    oracle.pr_rounding_f32).  The L1 change of sweep k is sum |new - old|,
    so two runs whose scores differ by e_k after sweep k differ in it by at
    most L1(e_k) + L1(e_(k-1)) (triangle inequality), and L1(e_k) <= G_k +
    R_k <= 5 R_k with the engine's own rounding G_k <= 4 R_k (the bound the
    final scores are held to).  In late sweeps the change per vertex is
    ~1e-4 of the score, so the last bits of the scores, where any other
    summation order differs, are ~1e-3 of the change: the rounding term, not
    the relative one, bounds those sweeps;
  * the reported L1 change of every sweep equals, to 1e-12 relative, the FP64
    sum of |new - old| over the engine's own float scores before and after
    that sweep (each float difference added in double, as
    src/pr_spmv.cc:42,53 does).
"""
import numpy as np
import pytest

import oracle
from gapbs_b200 import PageRankEngine, PageRankPull
from gapbs_b200.graph import Graph, make_graph
from conftest import golden_args, gpu_available, fmt_step

pytestmark = pytest.mark.gpu

CASES = ["g10", "u10", "g12", "u12", "g10k4", "g16", "u16", "g18", "el4", "el4s", "mtx4"]


# "blocked": the slice-blocked sweep forced (every graph here fits it);
# "blocked-small": the same with small slices and bins (many slices and
# bins per graph; every graph here fits them too)
LAYOUTS = {"gather": ("gather", 0, 0), "blocked": ("blocked", 0, 0),
           "blocked-small": ("blocked", 256, 4096)}


@pytest.fixture(scope="module", params=sorted(LAYOUTS))
def engine(request):
    if not gpu_available():
        pytest.skip("no CUDA device")
    eng = PageRankEngine(0)
    eng.set_sweep_layout(*LAYOUTS[request.param])
    eng.layout_name = request.param
    yield eng
    eng.close()


def check_parity(engine, g, max_iters=20, epsilon=1e-4, expect_sweeps=None):
    engine.upload(g)
    res = engine.run(max_iters, epsilon)
    s32, k32, tr32 = oracle.pr_pull_f32(g, max_iters, epsilon)
    s64, _, _ = oracle.pr_pull_f64(g, max_iters, epsilon)
    gpu = res.scores
    assert gpu.dtype == np.float32 and gpu.shape == (g.num_nodes,)
    assert int(res.sweeps[0]) == k32
    if expect_sweeps is not None:
        assert k32 == expect_sweeps
    ref_l1 = float(np.abs(s32.astype(np.float64) - s64).sum())
    gpu_l1 = float(np.abs(gpu.astype(np.float64) - s64).sum())
    assert gpu_l1 <= 4 * ref_l1 + 1e-7, (gpu_l1, ref_l1)
    assert np.all(np.abs(gpu - s64) <= 2e-5 * np.abs(s64) + 1e-10)
    if epsilon > 0 and k32 < max_iters:
        assert oracle.pr_verify_f32(g, gpu) < epsilon
    R = oracle.pr_rounding_f32(g, k32)
    bound = 1e-5 * tr32 + 5 * (R + np.concatenate([[0.0], R[:-1]]))
    dev = np.abs(res.err_trace[:k32, 0] - tr32)
    assert np.all(dev <= bound), (dev / np.maximum(tr32, 1e-300), bound / np.maximum(tr32, 1e-300))
    layout = getattr(engine, "layout_name", "gather")
    info = engine.sweep_layout_info()
    if layout.startswith("blocked") and g.num_edges_directed > 0:
        assert info["last_run_blocked"]
    if layout == "gather":
        assert not info["last_run_blocked"]
    return res


@pytest.mark.parametrize("case", CASES)
def test_parity_reference_graphs(engine, golden, case):
    e = golden["cases"][case]
    g = make_graph(golden_args(e))
    check_parity(engine, g, expect_sweeps=e["sweeps"])


def test_parity_adversarial(engine, adversarial):
    names = sorted({k.rsplit("_", 1)[0] for k in adversarial if k.endswith("_scores")})
    for name in names:
        g = Graph.from_edges(adversarial[f"{name}_u"], adversarial[f"{name}_v"],
                             symmetrize=bool(adversarial[f"{name}_sym"]))
        check_parity(engine, g, expect_sweeps=int(adversarial[f"{name}_sweeps"]))


def test_multi_segment_hubs(engine):
    """Rows longer than one hub segment (8192 entries) in several sizes."""
    rng = np.random.default_rng(11)
    us, vs = [], []
    for hub, deg in ((0, 30000), (1, 8192), (2, 8193), (3, 16385)):
        us.append(np.full(deg, hub))
        vs.append(rng.integers(10, 40000, deg))
    us.append(rng.integers(10, 40000, 60000))
    vs.append(rng.integers(10, 40000, 60000))
    g = Graph.from_edges(np.concatenate(us), np.concatenate(vs), symmetrize=True)
    check_parity(engine, g)


def test_directed_with_sinks_and_sources(engine):
    rng = np.random.default_rng(5)
    u = rng.integers(0, 3000, 20000)
    v = rng.integers(0, 3000, 20000)
    v[:500] = 7          # a hub sink
    u[500:1500] = 9      # a hub source
    g = Graph.from_edges(u, v, symmetrize=False)
    assert g.directed
    check_parity(engine, g)


def test_zero_iterations_returns_init(engine):
    g = make_graph("-g 10")
    engine.upload(g)
    res = engine.run(0, 1e-4)
    assert int(res.sweeps[0]) == 0
    assert np.all(res.scores == np.float32(1.0) / np.float32(g.num_nodes))


def test_epsilon_zero_runs_all_iterations(engine):
    g = make_graph("-u 10")
    res = check_parity(engine, g, max_iters=20, epsilon=0.0)
    assert int(res.sweeps[0]) == 20


def test_deterministic(engine):
    g = make_graph("-g 14")
    engine.upload(g)
    a = engine.run(20, 1e-4)
    b = engine.run(20, 1e-4)
    assert np.array_equal(a.scores.view(np.uint32), b.scores.view(np.uint32))
    assert np.array_equal(a.err_trace, b.err_trace)


@pytest.mark.parametrize("args", ["-g 12", "-u 11", "multi-hub"])
def test_l1_trace_is_fp64_sum_of_own_changes(engine, args):
    """Sweep k's reported L1 change is the FP64 sum of |s_k - s_(k-1)| over
    the engine's own float scores (runs of exactly k sweeps, epsilon 0)."""
    if args == "multi-hub":
        rng = np.random.default_rng(12)
        u = np.concatenate([np.zeros(20000, int), rng.integers(0, 9000, 30000)])
        g = Graph.from_edges(u, rng.integers(1, 9000, 50000), symmetrize=True)
    else:
        g = make_graph(args)
    engine.upload(g)
    full = engine.run(12, 0.0)
    prev = np.full(g.num_nodes, np.float32(1.0) / np.float32(g.num_nodes), np.float32)
    for k in range(1, 13):
        cur = engine.run(k, 0.0).scores
        l1 = float(np.abs(cur - prev).astype(np.float64).sum())
        np.testing.assert_allclose(full.err_trace[k - 1, 0], l1, rtol=1e-12)
        prev = cur


def test_pagerankpull_logging(engine, golden, capfd):
    e = golden["cases"]["g12"]
    g = make_graph(golden_args(e))
    s = PageRankPull(g, 20, 1e-4, logging_enabled=True)
    out = [ln for ln in capfd.readouterr().out.splitlines() if ln.strip()]
    assert len(out) == e["sweeps"]
    # same step numbers; values agree to the printed precision or one unit
    for got, want in zip(out, e["log_lines"]):
        assert got[:5] == want[:5]
        assert abs(float(got[5:]) - float(want[5:])) <= 1.01e-5
    assert s.dtype == np.float32


def test_invalid_csr_rejected(engine):
    from gapbs_b200.pagerank import PageRankError
    with pytest.raises(PageRankError) as ei:
        engine.upload_csr(3, [0, 1, 2, 3], [1, 2, 5])   # id 5 out of range
    assert ei.value.code == -5
    with pytest.raises(PageRankError) as ei:
        engine.upload_csr(3, [0, 2, 1, 3], [1, 2, 0])   # offsets not monotone
    assert ei.value.code == -5


def test_run_without_graph_fails_cleanly():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from gapbs_b200.pagerank import PageRankError
    eng = PageRankEngine(0)
    with pytest.raises(PageRankError) as ei:
        eng.run(20, 1e-4)
    assert ei.value.code == -4
    eng.close()


def test_bins_cover_all_rows(engine):
    g = make_graph("-g 16")
    engine.upload(g)
    info = engine.graph_info()
    assert sum(info["bin_rows"]) == g.num_nodes
    assert info["max_degree"] == int(np.diff(g.in_offsets).max())


def test_gather_roofline_probes(engine):
    # the ceilings bench.py divides by: positive and of the right order
    from gapbs_b200.pagerank import measure_gather_rate, measure_row_gather_rate
    g4 = measure_gather_rate(64 << 20, 0)
    assert 1e10 < g4 < 1e13  # 4-byte loads per second
    rows = [measure_row_gather_rate(64 << 20, rb, 0) for rb in (16, 256)]
    assert all(1e11 < r < 1e14 for r in rows)  # bytes per second
    assert rows[1] > rows[0]  # whole rows move more bytes per request
