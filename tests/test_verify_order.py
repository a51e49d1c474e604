"""The ordering argument behind the device PRVerifier (pr_gpu_verify), on CPU.

The reference's PRVerifier (src/pr_spmv.cc:78-94) pushes contributions along
out-edges in ascending source order; the device kernels instead add each
in-row sequentially, in row order.  On the reference builder's graphs every
row is sorted, so both orders are the same sequence of float additions and
give the same error to the last bit.  This restates the device computation
in numpy (sequential float32 adds per in-row, float32 residual, double sum in
vertex order) and checks it against the oracle's push-order restatement
(oracle.pr_verify_f32) with ==, on the golden graphs, for random and
converged scores.
"""
import numpy as np
import pytest

import oracle
from gapbs_b200.graph import make_graph
from conftest import golden_args

D = np.float32(0.85)


def row_order_error(g, s):
    n = g.num_nodes
    deg = np.diff(np.asarray(g.out_offsets, np.int64)).astype(np.float32)
    with np.errstate(divide="ignore", invalid="ignore"):
        contrib = (s / deg).astype(np.float32)  # float division, as the reference
    base = np.float32((np.float32(1) - D) / np.float32(n))
    off = np.asarray(g.in_offsets, np.int64)
    nbr = np.asarray(g.in_neighbors, np.int64)
    error = 0.0
    for v in range(n):
        lo, hi = off[v], off[v + 1]
        incoming = (np.add.accumulate(contrib[nbr[lo:hi]], dtype=np.float32)[-1]
                    if hi > lo else np.float32(0))
        r = np.float32(np.float32(base + np.float32(D * incoming)) - s[v])
        error += float(abs(r))
    return error


@pytest.mark.parametrize("case", ["g10", "u10", "g12", "el4", "el4s", "gr4", "mtx4"])
def test_row_order_equals_push_order(golden, case):
    g = make_graph(golden_args(golden["cases"][case]))
    rng = np.random.default_rng(21)
    n = g.num_nodes
    converged, _, _ = oracle.pr_pull_f32(g, 20, 1e-4)
    for s in (rng.random(n, dtype=np.float32) / np.float32(n),
              np.asarray(converged, np.float32)):
        assert row_order_error(g, s) == oracle.pr_verify_f32(g, s)


def test_reversed_rows_change_the_error():
    """The check has teeth: with every in-row reversed (descending source
    order) the same computation no longer gives the push-order error."""
    g = make_graph("-g 10")

    class Reversed:
        pass
    r = Reversed()
    r.num_nodes, r.out_offsets = g.num_nodes, g.out_offsets
    r.in_offsets = np.asarray(g.in_offsets, np.int64)
    nbr = np.asarray(g.in_neighbors, np.int64).copy()
    for v in range(g.num_nodes):
        nbr[r.in_offsets[v]:r.in_offsets[v + 1]] = nbr[r.in_offsets[v]:r.in_offsets[v + 1]][::-1]
    r.in_neighbors = nbr
    s = np.random.default_rng(21).random(g.num_nodes, dtype=np.float32) / np.float32(g.num_nodes)
    assert row_order_error(g, s) == oracle.pr_verify_f32(g, s)
    assert row_order_error(r, s) != oracle.pr_verify_f32(g, s)
