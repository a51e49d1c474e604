"""The oracle's adjoint gradients agree with central finite differences (CPU).

L(t, w) = sum_v loss_w[v] * s[v] at the FP64 PPR fixed point; FD with
h = 1e-6 in FP64 on sampled teleport and edge-weight coordinates, each
perturbed problem converged from the unperturbed solution.  This pins the
gradient formulas the GPU adjoint implements.
"""
import numpy as np
import pytest

import oracle
from gapbs_b200.graph import Graph, make_graph
from helpers import in_weights, row_sums

TIGHT = dict(max_iters=2000, epsilon=1e-15)


def solve(g, t, ew, s0=None):
    n = g.num_nodes
    s, k, _ = oracle.ppr_f64(n, g.in_offsets, g.in_neighbors, g.out_offsets, t,
                             in_w=in_weights(g, ew), rowsum=row_sums(g, ew), s_init=s0, **TIGHT)
    return s


@pytest.mark.parametrize("args,directed", [("-g 9", False), (None, True)])
def test_adjoint_matches_finite_differences(args, directed):
    rng = np.random.default_rng(17)
    if directed:
        g = Graph.from_edges(rng.integers(0, 300, 2500), rng.integers(0, 300, 2500))
    else:
        g = make_graph(args)
    n, m = g.num_nodes, g.num_edges_directed
    ew = rng.uniform(0.5, 1.5, m)
    t = np.zeros(n)
    seeds = rng.choice(np.nonzero(np.diff(g.out_offsets) > 0)[0], 5, replace=False)
    t[seeds] = 0.2
    lw = rng.normal(size=n)
    s = solve(g, t, ew)
    lam, gt, gw, k = oracle.ppr_adjoint_f64(n, g.out_offsets, g.out_neighbors, lw, s, out_w=ew,
                                            max_iters=4000, epsilon=1e-15)
    h = 1e-6
    L = lambda s_: float(lw @ s_)
    for i in rng.choice(n, 12, replace=False):
        tp, tm = t.copy(), t.copy()
        tp[i] += h
        tm[i] -= h
        fd = (L(solve(g, tp, ew, s)) - L(solve(g, tm, ew, s))) / (2 * h)
        assert abs(fd - gt[i]) <= 1e-5 * max(1.0, abs(gt[i])), (i, fd, gt[i])
    for e in rng.choice(m, 12, replace=False):
        wp, wm = ew.copy(), ew.copy()
        wp[e] += h
        wm[e] -= h
        fd = (L(solve(g, t, wp, s)) - L(solve(g, t, wm, s))) / (2 * h)
        assert abs(fd - gw[e]) <= 1e-6 + 1e-4 * abs(gw[e]), (e, fd, gw[e])
