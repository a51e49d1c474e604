"""GPU adjoint (K4/K5) against the FP64 oracle's adjoint, and through
torch.autograd.

The oracle's adjoint formulas are pinned to central finite differences in
tests/test_adjoint_oracle.py; here the GPU gradients (FP32) must match the
oracle's FP64 gradients computed at the GPU's own forward solution:
  relative L2 error <= 1e-4 for d/dteleport and <= 1e-3 for d/dweights.
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


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("kind", ["undirected_weighted", "undirected_unit", "directed_weighted"])
def test_adjoint_matches_oracle(engine, kind):
    rng = np.random.default_rng(21)
    if kind.startswith("directed"):
        g = Graph.from_edges(rng.integers(0, 3000, 30000), rng.integers(0, 3000, 30000))
    else:
        g = make_graph("-g 12")
    n, m = g.num_nodes, g.num_edges_directed
    ew = rng.uniform(0.5, 1.5, m).astype(np.float32) if kind.endswith("weighted") else None
    engine.upload(g, edge_w=ew)
    t = seed_teleports(g, 1, rng, max_seeds=200)[:, 0]
    fwd = engine.run(100, 1e-7, teleport=t)
    lw = rng.normal(size=n).astype(np.float32)
    gt, ge, sweeps = engine.adjoint(lw, fwd.scores, max_iters=400, epsilon=1e-7)
    assert 0 < sweeps <= 400
    w64 = None if ew is None else ew.astype(np.float64)
    lam, gt64, gw64, _ = oracle.ppr_adjoint_f64(n, g.out_offsets, g.out_neighbors, lw,
                                                fwd.scores.astype(np.float64), out_w=w64,
                                                max_iters=4000, epsilon=1e-13)
    assert rel_l2(gt, gt64) <= 1e-4
    assert rel_l2(ge, gw64) <= 1e-3


def test_autograd_function(engine):
    torch = pytest.importorskip("torch")
    from gapbs_b200.autograd import PageRankContext, personalized_pagerank
    rng = np.random.default_rng(5)
    g = make_graph("-g 11")
    n, m = g.num_nodes, g.num_edges_directed
    pctx = PageRankContext(g, max_iters=100, epsilon=1e-7, adjoint_max_iters=400,
                           adjoint_epsilon=1e-7)
    t_np = seed_teleports(g, 1, rng)[:, 0]
    t = torch.tensor(t_np, device="cuda", requires_grad=True)
    w = torch.tensor(rng.uniform(0.5, 1.5, m).astype(np.float32), device="cuda", requires_grad=True)
    lw = torch.tensor(rng.normal(size=n).astype(np.float32), device="cuda")
    s = personalized_pagerank(t, w, pctx)
    loss = (lw * s).sum()
    loss.backward()
    assert t.grad.shape == (n,) and w.grad.shape == (m,)
    # FP64 oracle at the same weights
    ew = w.detach().cpu().numpy().astype(np.float64)
    s64, _, _ = oracle.ppr_f64(n, g.in_offsets, g.in_neighbors, g.out_offsets,
                               t_np.astype(np.float64), in_w=in_weights(g, ew),
                               rowsum=row_sums(g, ew), max_iters=2000, epsilon=1e-14)
    assert np.abs(s.detach().cpu().numpy() - s64).sum() <= 1e-5
    _, gt64, gw64, _ = oracle.ppr_adjoint_f64(n, g.out_offsets, g.out_neighbors,
                                              lw.cpu().numpy().astype(np.float64), s64,
                                              out_w=ew, max_iters=4000, epsilon=1e-13)
    assert rel_l2(t.grad.cpu().numpy(), gt64) <= 1e-4
    assert rel_l2(w.grad.cpu().numpy(), gw64) <= 1e-3


def test_set_edge_weights_device(engine):
    """pr_gpu_set_edge_weights_device gives bit for bit what a fresh upload
    of the same weights gives (forward and adjoint); invalid weights are
    refused with PR_GPU_EGRAPH and leave the previous ones; a graph without
    weights refuses the call with PR_GPU_EINVAL."""
    torch = pytest.importorskip("torch")
    from gapbs_b200.pagerank import PageRankError
    rng = np.random.default_rng(8)
    for g in (make_graph("-g 12"),
              Graph.from_edges(rng.integers(0, 3000, 30000), rng.integers(0, 3000, 30000))):
        n, m = g.num_nodes, g.num_edges_directed
        w1 = rng.uniform(0.5, 1.5, m).astype(np.float32)
        w2 = rng.uniform(0.5, 1.5, m).astype(np.float32)
        t = seed_teleports(g, 1, rng)[:, 0]
        lw = rng.normal(size=n).astype(np.float32)
        engine.upload(g, edge_w=w2)
        want = engine.run(100, 1e-7, teleport=t)
        want_gt, want_ge, _ = engine.adjoint(lw, want.scores, max_iters=300, epsilon=1e-7)
        engine.upload(g, edge_w=w1)
        d_w2 = torch.from_numpy(w2).cuda()
        torch.cuda.synchronize()
        engine.set_edge_weights_device(d_w2.data_ptr())
        got = engine.run(100, 1e-7, teleport=t)
        assert np.array_equal(got.scores.view(np.uint32), want.scores.view(np.uint32))
        gt, ge, _ = engine.adjoint(lw, got.scores, max_iters=300, epsilon=1e-7)
        assert np.array_equal(gt, want_gt) and np.array_equal(ge, want_ge)
        bad = d_w2.clone()
        bad[m // 2] = -1.0
        with pytest.raises(PageRankError) as ei:
            engine.set_edge_weights_device(bad.data_ptr())
        assert ei.value.code == -5   # PR_GPU_EGRAPH
        again = engine.run(100, 1e-7, teleport=t)
        assert np.array_equal(again.scores.view(np.uint32), want.scores.view(np.uint32))
    engine.upload(make_graph("-g 10"))
    with pytest.raises(PageRankError) as ei:
        engine.set_edge_weights_device(d_w2.data_ptr())
    assert ei.value.code == -1       # PR_GPU_EINVAL


def test_autograd_training_loop_updates_weights_on_device(engine):
    """Ten SGD steps on the edge weights through torch.autograd: one graph
    upload, then device weight updates only; the final scores match the FP64
    oracle at the final weights."""
    torch = pytest.importorskip("torch")
    from gapbs_b200.autograd import PageRankContext, personalized_pagerank
    rng = np.random.default_rng(13)
    g = make_graph("-g 12")
    n, m = g.num_nodes, g.num_edges_directed
    pctx = PageRankContext(g, max_iters=100, epsilon=1e-7, adjoint_max_iters=300,
                           adjoint_epsilon=1e-7)
    t_np = seed_teleports(g, 1, rng)[:, 0]
    t = torch.tensor(t_np, device="cuda")
    w = torch.tensor(rng.uniform(0.5, 1.5, m).astype(np.float32), device="cuda",
                     requires_grad=True)
    lw = torch.tensor(rng.normal(size=n).astype(np.float32), device="cuda")
    for _ in range(10):
        s = personalized_pagerank(t, w, pctx)
        loss = (lw * s).sum()
        w.grad = None
        loss.backward()
        with torch.no_grad():
            w -= 1e3 * w.grad
            w.clamp_(min=0.05)
    assert pctx.uploads == 1 and pctx.weight_updates == 9
    s = personalized_pagerank(t, w, pctx)
    assert pctx.weight_updates == 10
    ew = w.detach().cpu().numpy().astype(np.float64)
    s64, _, _ = oracle.ppr_f64(n, g.in_offsets, g.in_neighbors, g.out_offsets,
                               t_np.astype(np.float64), in_w=in_weights(g, ew),
                               rowsum=row_sums(g, ew), max_iters=2000, epsilon=1e-14)
    assert np.abs(s.detach().cpu().numpy() - s64).sum() <= 1e-5
    pctx.engine.close()
