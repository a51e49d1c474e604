"""pr_gpu_upload_sg: serialized graphs streamed from the file to the device.

A graph written with Graph.write_sg (the reference's .sg layout) and uploaded
straight from the file must solve exactly as the same graph uploaded from
host arrays, and both must match the oracle with the plain parity
tolerances (the reference's sweep count, per vertex 2e-5 relative + 1e-10 of
FP64, L1 at most 4x the reference's own FP32 L1 + 1e-7, PRVerifier below
epsilon); truncated files and missing files are rejected cleanly.
"""
import os

import numpy as np
import pytest

import oracle
from gapbs_b200 import PageRankEngine
from gapbs_b200.graph import Graph, make_graph
from gapbs_b200.pagerank import PageRankError
from conftest import gpu_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    if not gpu_available():
        pytest.skip("no CUDA device")
    eng = PageRankEngine(0)
    yield eng
    eng.close()


def directed_graph():
    rng = np.random.default_rng(3)
    return Graph.from_edges(rng.integers(0, 5000, 60000), rng.integers(0, 5000, 60000))


@pytest.mark.parametrize("kind", ["g16", "u14", "directed"])
def test_sg_upload_matches_host_upload(engine, kind, tmp_path):
    g = directed_graph() if kind == "directed" else make_graph(f"-{kind[0]} {kind[1:]}")
    path = str(tmp_path / "graph.sg")
    g.write_sg(path)
    n, m = engine.upload_sg(path)
    assert (n, m) == (g.num_nodes, g.num_edges_directed)
    assert engine.directed == g.directed
    from_file = engine.run(20, 1e-4)
    engine.upload(g)
    from_host = engine.run(20, 1e-4)
    assert np.array_equal(from_file.scores, from_host.scores)
    assert np.array_equal(from_file.sweeps, from_host.sweeps)
    s32, k32, _ = oracle.pr_pull_f32(g, 20, 1e-4)
    s64, _, _ = oracle.pr_pull_f64(g, 20, 1e-4)
    assert int(from_file.sweeps[0]) == k32
    gpu = from_file.scores
    assert np.all(np.abs(gpu - s64) <= 2e-5 * np.abs(s64) + 1e-10)
    ref_l1 = float(np.abs(s32.astype(np.float64) - s64).sum())
    assert float(np.abs(gpu.astype(np.float64) - s64).sum()) <= 4 * ref_l1 + 1e-7
    if k32 < 20:
        assert oracle.pr_verify_f32(g, gpu) < 1e-4


def test_sg_upload_rejects_bad_files(engine, tmp_path):
    g = make_graph("-g 12")
    path = str(tmp_path / "graph.sg")
    g.write_sg(path)
    size = os.path.getsize(path)
    with open(path, "rb") as fh:
        data = fh.read()
    cut = str(tmp_path / "cut.sg")
    with open(cut, "wb") as fh:
        fh.write(data[: size - 100])
    with pytest.raises(PageRankError) as ei:
        engine.upload_sg(cut)
    assert ei.value.code == -5  # PR_GPU_EGRAPH
    with pytest.raises(PageRankError):
        engine.upload_sg(str(tmp_path / "missing.sg"))
    # the engine stays usable
    engine.upload_sg(path)
    assert engine.run(20, 1e-4).sweeps[0] > 0
