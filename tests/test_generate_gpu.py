"""pr_gpu_generate: the reference's -g / -u graphs built on the device.

The device-built CSR must equal the host builder's (itself pinned to the
reference's CSR hashes in test_graph_builder.py) array for array, and a
solve on it must give the same result as on the uploaded host graph.
"""
import json
import os

import numpy as np
import pytest

from gapbs_b200 import PageRankEngine
from gapbs_b200.graph import make_graph
from conftest import GOLDEN, gpu_available

pytestmark = pytest.mark.gpu

with open(os.path.join(GOLDEN, "pr_golden.json")) as fh:
    GOLD = json.load(fh)["cases"]


@pytest.fixture(scope="module")
def engine():
    if not gpu_available():
        pytest.skip("no CUDA device")
    eng = PageRankEngine(0)
    yield eng
    eng.close()


@pytest.mark.parametrize("args", ["-g 10", "-u 10", "-g 10 -k 4", "-g 12 -k 1", "-u 12 -k 3",
                                  "-g 16", "-u 16", "-g 18 -k 8", "-g 20"])
def test_device_graph_equals_host_graph(engine, args):
    n, m = engine.generate(args)
    gd = engine.download_graph()
    gh = make_graph(args)
    assert (n, m) == (gh.num_nodes, gh.num_edges_directed)
    assert not gd.directed and gd.num_edges == gh.num_edges
    assert np.array_equal(gd.out_offsets, gh.out_offsets)
    assert np.array_equal(gd.out_neighbors, gh.out_neighbors)


@pytest.mark.parametrize("case", ["g10", "u10", "g16", "u16", "g18"])
def test_device_graph_matches_reference_hash(engine, case):
    import hashlib
    e = GOLD[case]
    engine.generate(e["args"])
    g = engine.download_graph()
    h = hashlib.sha256()
    for a, dt in ((g.out_offsets, np.int64), (g.out_neighbors, np.int32),
                  (g.in_offsets, np.int64), (g.in_neighbors, np.int32)):
        h.update(np.ascontiguousarray(a, dt).tobytes())
    assert h.hexdigest() == e["csr_sha256"]


def test_solve_on_generated_graph(engine):
    engine.generate("-g 14")
    on_device = engine.run(20, 1e-4)
    g = engine.download_graph()
    after_download = engine.run(20, 1e-4)  # the device graph stays
    engine.upload(make_graph("-g 14"))
    uploaded = engine.run(20, 1e-4)
    assert np.array_equal(on_device.scores, uploaded.scores)
    assert np.array_equal(after_download.scores, uploaded.scores)
    assert g.num_nodes == on_device.scores.size


def test_generate_rejects_bad_arguments(engine):
    from gapbs_b200.pagerank import PageRankError
    with pytest.raises(ValueError):
        engine.generate("-f graph.el")
    with pytest.raises(PageRankError):
        engine.generate("-g 24 -k 128")  # beyond int32 offsets
    with pytest.raises(PageRankError):
        engine.download_graph()  # nothing generated since the last download
