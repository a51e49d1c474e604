"""The device PRVerifier (pr_gpu_verify) against the reference's own
PRVerifier (src/pr_spmv.cc:78-94, compiled into oracle/_ref from the
reference's sources) and the oracle's restatement (oracle.pr_verify_f32).

On every graph of the golden set (the reference's builder sorts and
deduplicates each row, so every in-row lists its sources in ascending
order) and on Kronecker scale 20, the device error must be the SAME double
as the oracle's and the reference's, bit for bit, for converged scores,
scores two sweeps in (errors far above the tolerance), random scores and
the reference's own scores where the golden set keeps them.  The
reference's error is read through its pass/fail answer: error < t is false
at t = e and true at the next double above e only when its error is
exactly e.

With rows in another order only the rounding of each incoming sum changes:
on Kronecker scale 12 with every row reversed the difference stays within
the first-order bound of two float sums of k terms (2 (k - 1) u times the
sum, u = 2^-24) plus the three roundings of each residual in both, taken
at the size of the residual's largest term.
"""
import os
from ctypes import byref, c_double

import numpy as np
import pytest

import oracle
from gapbs_b200 import PageRankEngine, PageRankPull, PRVerifier
from gapbs_b200._pr_abi import PR_GPU_EINVAL, PR_GPU_ENOGRAPH
from gapbs_b200.graph import make_graph
from conftest import GOLDEN, golden_args, gpu_available

pytestmark = pytest.mark.gpu

D = np.float32(0.85)


@pytest.fixture(scope="module")
def engine():
    if not gpu_available():
        pytest.skip("no CUDA device")
    eng = PageRankEngine(0)
    yield eng
    eng.close()


def ref_error_is(g, scores, e):
    """True when the reference's PRVerifier error on (g, scores) is exactly e."""
    if not oracle.ref_available():
        return True
    rg = oracle.RefGraph.from_csr(g)
    return (not rg.verify(scores, e)) and rg.verify(scores, float(np.nextafter(e, np.inf)))


def score_sets(eng, g, rng, name=None):
    sets = {"converged": eng.run(20, 1e-4).scores.copy(),
            "two sweeps": eng.run(2, 0.0).scores.copy(),
            "random": rng.random(g.num_nodes, dtype=np.float32) / np.float32(g.num_nodes)}
    path = os.path.join(GOLDEN, f"scores_{name}.npy")
    if name and os.path.exists(path):
        sets["reference"] = np.load(path).astype(np.float32)
    return sets


def check_graph(eng, g, rng, name=None):
    eng.upload(g)
    for label, s in score_sets(eng, g, rng, name).items():
        e_dev = eng.verify(s)
        e_or = oracle.pr_verify_f32(g, s)
        assert e_dev == e_or, (label, e_dev, e_or)
        assert ref_error_is(g, s, e_dev), label


GOLDEN_CASES = ["g10", "u10", "g12", "u12", "g10k4", "g16", "u16", "g18", "el4", "el4s",
                "wel4", "gr4", "graph4", "mtx4", "graph4w", "mtx4w"]


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_error_equals_reference(engine, golden, case):
    g = make_graph(golden_args(golden["cases"][case]))
    check_graph(engine, g, np.random.default_rng(11), case)


def test_error_equals_reference_g20(engine):
    check_graph(engine, make_graph("-g 20"), np.random.default_rng(12))


def test_python_prverifier(engine, capsys):
    g = make_graph("-g 12")
    scores = PageRankPull(g, 20, 1e-4)
    e_or = oracle.pr_verify_f32(g, scores)
    assert PRVerifier(g, scores, 1e-4) == (e_or < 1e-4)
    assert PRVerifier(g, scores, e_or) is False
    out = capsys.readouterr().out.splitlines()
    assert out[0] == f"{'Total Error:':<21}{e_or:3.5f}"


def test_reversed_rows_differ_by_rounding_only(engine):
    g = make_graph("-g 12")
    n = g.num_nodes
    off = g.out_offsets.astype(np.int64)
    nbr = g.out_neighbors.astype(np.int32).copy()
    for u in range(n):
        nbr[off[u]:off[u + 1]] = nbr[off[u]:off[u + 1]][::-1]
    engine.upload_csr(n, off.astype(np.int32), nbr)
    rng = np.random.default_rng(13)
    s = rng.random(n, dtype=np.float32) / np.float32(n)
    e_dev = engine.verify(s)
    e_or = oracle.pr_verify_f32(g, s)
    # first-order bound on |e_dev - e_or|
    u = 2.0 ** -24
    deg = np.diff(off)
    contrib = s.astype(np.float64) / np.maximum(deg, 1)
    incoming = np.zeros(n)
    np.add.at(incoming, nbr, np.repeat(contrib, deg))
    base = float((np.float32(1) - D) / np.float32(n))
    k = np.maximum(deg - 1, 0)  # undirected: in-degree = out-degree
    bound = float(np.sum(float(D) * 2.02 * k * u * incoming
                         + 6 * u * (base + float(D) * incoming + s)))
    bound += n * 2.0 ** -52 * e_or
    assert abs(e_dev - e_or) <= bound, (e_dev, e_or, bound)


def test_errors(engine):
    e = c_double()
    s = np.zeros(4, np.float32)
    fresh = PageRankEngine(0)
    try:
        rc = fresh._lib.pr_gpu_verify(fresh._h, s.ctypes.data, 0.85, byref(e))
        assert rc == PR_GPU_ENOGRAPH
    finally:
        fresh.close()
    g = make_graph("-g 10")
    engine.upload(g)
    assert engine._lib.pr_gpu_verify(engine._h, None, 0.85, byref(e)) == PR_GPU_EINVAL
    assert engine._lib.pr_gpu_verify(engine._h, s.ctypes.data, 0.85, None) == PR_GPU_EINVAL
    with pytest.raises(ValueError):
        engine.verify(np.zeros(g.num_nodes + 1, np.float32))
