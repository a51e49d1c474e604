"""Pins the oracle (CPU restatement) against the reference's own outputs.

The golden fixtures were produced by the reference compiled from its sources
(tests/golden/make_golden.py).  The FP32 oracle must reproduce the reference's
scores bit for bit, its sweep count, its -l lines and its PRVerifier result.
"""
import hashlib
import os

import numpy as np
import pytest

import oracle
from gapbs_b200.graph import Graph, make_graph
from conftest import GOLDEN, fmt_step, golden_args

FULL_SCORE_CASES = ["g10", "u10", "g12", "g10k4", "el4", "el4s"]
HASH_CASES = ["u12", "g16", "u16", "g18", "wel4", "gr4", "graph4", "mtx4", "graph4w", "mtx4w"]


def _sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("case", FULL_SCORE_CASES)
def test_oracle_f32_bitexact_scores(golden, case):
    e = golden["cases"][case]
    g = make_graph(golden_args(e))
    s, k, tr = oracle.pr_pull_f32(g)
    ref = np.load(os.path.join(GOLDEN, f"scores_{case}.npy"))
    assert np.array_equal(s.view(np.uint32), ref.view(np.uint32))
    assert k == e["sweeps"]
    assert [fmt_step(i, v) for i, v in enumerate(tr)] == e["log_lines"]


@pytest.mark.parametrize("case", HASH_CASES)
def test_oracle_f32_matches_reference_hash(golden, case):
    e = golden["cases"][case]
    g = make_graph(golden_args(e))
    s, k, tr = oracle.pr_pull_f32(g)
    assert _sha(s) == e["scores_sha256"]
    assert k == e["sweeps"]
    assert [fmt_step(i, v) for i, v in enumerate(tr)] == e["log_lines"]


@pytest.mark.parametrize("case", FULL_SCORE_CASES + HASH_CASES)
def test_oracle_verifier_matches_reference(golden, case):
    e = golden["cases"][case]
    g = make_graph(golden_args(e))
    s, _, _ = oracle.pr_pull_f32(g)
    err = oracle.pr_verify_f32(g, s)
    # the reference printed "Total Error:" with %3.5lf and passed
    assert e["verify_line"] == f"{'Total Error:':<21s}{err:3.5f}"
    assert (err < 1e-4) == e["verify_pass"]


def test_oracle_f64_close_to_f32(golden):
    g = make_graph("-g 12")
    s32, k32, _ = oracle.pr_pull_f32(g)
    s64, k64, _ = oracle.pr_pull_f64(g)
    assert k32 == k64
    assert np.abs(s32 - s64).sum() < 1e-6


def test_oracle_adversarial_matches_reference(adversarial):
    names = sorted({k.rsplit("_", 1)[0] for k in adversarial if k.endswith("_scores")})
    assert names
    for name in names:
        g = Graph.from_edges(adversarial[f"{name}_u"], adversarial[f"{name}_v"],
                             symmetrize=bool(adversarial[f"{name}_sym"]))
        s, k, _ = oracle.pr_pull_f32(g)
        assert np.array_equal(s.view(np.uint32), adversarial[f"{name}_scores"].view(np.uint32)), name
        assert k == int(adversarial[f"{name}_sweeps"]), name


def test_oracle_residual_property():
    g = make_graph("-u 12")
    s, _, _ = oracle.pr_pull_f32(g)
    r = oracle.pr_residual_f64(g, s)
    v = oracle.pr_verify_f32(g, s)
    assert r < 1e-4 and abs(r - v) < 1e-6


def test_oracle_ppr_uniform_equals_plain():
    g = make_graph("-g 10")
    n = g.num_nodes
    t = np.full(n, 1.0 / n)
    s_ppr, k, _ = oracle.ppr_f64(n, g.in_offsets, g.in_neighbors, g.out_offsets, t)
    s_pl, k2, _ = oracle.pr_pull_f64(g)
    assert k == k2
    assert np.allclose(s_ppr, s_pl, rtol=1e-12, atol=1e-15)
