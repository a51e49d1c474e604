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
