"""Parity at the benchmark sizes, through size-independent properties.

The small-graph tests compare whole score vectors with the oracle; at the
benchmark sizes (-u 24 -k 16, -g 25 -k 16, 64 PPR columns on -g 22, the
adjoint on -g 20) the checks are the ones that do not need a full FP64 solve:

  * graph identity: the host builder's CSR hashes to the reference's;
  * the reference's own outputs, recorded by tests/golden/make_golden.py
    --fullsize: sweep count, per-sweep L1 change (-l lines, 5 decimals),
    float32 scores at 4096 fixed sample vertices, top-5, sum of scores;
  * PRVerifier, restated in the oracle (serial push, float sums, double L1):
    total error < 1e-4, the reference's pass criterion;
  * PPR: per column, the FP64 residual of the returned scores is at most
    the column's last L1 change (one Jacobi sweep contracts the residual by
    d), and batched columns agree with single-column solves;
  * adjoint: the GPU gradients against the FP64 oracle's adjoint at the GPU's
    own forward solution (relative L2 <= 1e-4 teleport, <= 1e-3 weights).
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from gapbs_b200 import PageRankEngine
from gapbs_b200.graph import make_graph
from conftest import GOLDEN, gpu_available
from helpers import seed_teleports

pytestmark = [pytest.mark.gpu, pytest.mark.fullsize]

with open(os.path.join(GOLDEN, "pr_fullsize.json")) as fh:
    FULL = json.load(fh)["cases"]


@pytest.fixture(scope="module")
def engine():
    if not gpu_available():
        pytest.skip("no CUDA device")
    eng = PageRankEngine(0)
    yield eng
    eng.close()


def csr_sha(g) -> str:
    h = hashlib.sha256()
    for a, dt in ((g.out_offsets, np.int64), (g.out_neighbors, np.int32),
                  (g.in_offsets, np.int64), (g.in_neighbors, np.int32)):
        h.update(np.ascontiguousarray(a, dt).tobytes())
    return h.hexdigest()


def load(case):
    e = FULL[case]
    g = make_graph(e["args"])
    assert (g.num_nodes, g.num_edges_directed) == (e["num_nodes"], e["num_edges_directed"])
    assert csr_sha(g) == e["csr_sha256"], "host builder differs from the reference's graph"
    return g, e


@pytest.mark.parametrize("layout", ["auto", "blocked", "gather"])
@pytest.mark.parametrize("case", ["u24", "g25"])
def test_pagerankpull_fullsize(engine, case, layout):
    g, e = load(case)
    engine.set_sweep_layout(layout)
    engine.upload(g)
    res = engine.run(20, 1e-4, 0.85)
    # auto takes the slice-blocked sweep on the Kronecker graph and keeps the
    # gather sweep on the uniform one (almost one (row, slice) pair per edge)
    blocked = layout == "blocked" or (layout == "auto" and case == "g25")
    assert engine.sweep_layout_info()["last_run_blocked"] == blocked
    engine.set_sweep_layout("auto")
    s = res.scores
    # the reference's sweep count and its printed per-sweep L1 change
    assert int(res.sweeps[0]) == e["sweeps"]
    ref_trace = [float(ln.split()[1]) for ln in e["log_lines"]]
    for it, r in enumerate(ref_trace):
        assert abs(res.err_trace[it, 0] - r) <= 0.5e-5 + 1e-3 * r, (it, res.err_trace[it, 0], r)
    # the reference's float32 scores at the sample vertices
    ids = np.asarray(e["sample_ids"], np.int64)
    ref = np.asarray(e["sample_scores"], np.float32)
    err = np.abs(s[ids].astype(np.float64) - ref)
    assert np.all(err <= 4e-5 * np.abs(ref) + 1e-10), float(err.max())
    # top-5 and the sum of scores
    top = [i for i, _ in e["top5"]]
    order = np.lexsort((np.arange(s.size), -s.astype(np.float64)))[:5]
    assert [int(i) for i in order] == top
    assert abs(float(s.astype(np.float64).sum()) - e["scores_sum"]) <= 1e-5 * e["scores_sum"]
    # the reference's verifier; the device verifier gives its error bit for bit
    e_or = oracle.pr_verify_f32(g, s)
    assert e_or < 1e-4
    assert engine.verify(s) == e_or


@pytest.mark.parametrize("case", ["u24", "g25"])
def test_device_generated_fullsize_graph(engine, case):
    e = FULL[case]
    n, m = engine.generate(e["args"])
    assert (n, m) == (e["num_nodes"], e["num_edges_directed"])
    res = engine.run(20, 1e-4, 0.85)
    assert int(res.sweeps[0]) == e["sweeps"]
    g = engine.download_graph()
    assert csr_sha(g) == e["csr_sha256"]


def test_batched_ppr_fullsize(engine):
    g, _ = load("g22")
    engine.upload(g)
    rng = np.random.default_rng(27491095 + 1)
    T = seed_teleports(g, 64, rng, max_seeds=4096)
    res = engine.run(20, 1e-4, 0.85, teleport=T)
    S, sweeps, trace = res.scores, res.sweeps, res.err_trace
    assert S.shape == (g.num_nodes, 64)
    for c in range(64):
        k = int(sweeps[c])
        assert 1 <= k <= 20
        last = float(trace[k - 1, c])
        if k < 20:
            assert last < 1e-4
        r = oracle.ppr_residual_f64(g, T[:, c], S[:, c])
        assert r <= last + 1e-6, (c, r, last)
    # batched columns against single-column solves of the same teleports
    for c in (0, 9, 31, 63):
        one = engine.run(20, 1e-4, 0.85, teleport=np.ascontiguousarray(T[:, c]))
        assert abs(int(one.sweeps[0]) - int(sweeps[c])) <= 1
        assert float(np.abs(one.scores.astype(np.float64) - S[:, c]).sum()) <= 2e-4


def test_adjoint_fullsize(engine):
    g, _ = load("g20")
    n, m = g.num_nodes, g.num_edges_directed
    rng = np.random.default_rng(20)
    ew = rng.uniform(0.5, 1.5, m).astype(np.float32)
    engine.upload(g, edge_w=ew)
    t = seed_teleports(g, 1, rng, max_seeds=4096)[:, 0]
    fwd = engine.run(200, 1e-7, teleport=t)
    lw = rng.normal(size=n).astype(np.float32)
    gt, ge, sweeps = engine.adjoint(lw, fwd.scores, max_iters=400, epsilon=1e-7)
    assert 0 < sweeps <= 400
    _, gt64, gw64, _ = oracle.ppr_adjoint_f64(n, g.out_offsets, g.out_neighbors, lw,
                                              fwd.scores.astype(np.float64),
                                              out_w=ew.astype(np.float64),
                                              max_iters=2000, epsilon=1e-10)

    def rel_l2(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))

    assert rel_l2(gt, gt64) <= 1e-4
    assert rel_l2(ge, gw64) <= 1e-3


def test_cc_and_bfs_fullsize(engine):
    """Connected components and BFS on the -g 25 graph: CC labels equal the
    reference's Afforest on the same CSR; a BFS tree passes the reference's
    verifier and its depths are the oracle's."""
    from helpers import depths_from_parents
    e = FULL["g25"]
    engine.generate(e["args"])
    g = engine.download_graph()
    assert csr_sha(g) == e["csr_sha256"]
    comp = engine.connected_components()
    ref_comp, _ = oracle.ref_cc_afforest_csr(g, trials=1)
    assert np.array_equal(comp, ref_comp)
    src = int(np.nonzero(np.diff(g.out_offsets) > 0)[0][12345])
    parent = engine.bfs(src)
    assert oracle.bfs_verify(g, src, parent)
    assert np.array_equal(depths_from_parents(parent, src), oracle.bfs_depths(g, src))
