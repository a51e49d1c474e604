"""Connected components on the GPU (pr_gpu_connected_components) against the
oracle's restatement of the reference's Afforest and the reference's own
labels (tests/golden/cc_golden.json): identical int32 labels, original ids.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from gapbs_b200 import PageRankEngine
from gapbs_b200.graph import Graph, make_graph
from gapbs_b200.pagerank import PageRankError
from conftest import GOLDEN, gpu_available

pytestmark = pytest.mark.gpu

with open(os.path.join(GOLDEN, "cc_golden.json")) as fh:
    CASES = json.load(fh)["cases"]


@pytest.fixture(scope="module")
def engine():
    if not gpu_available():
        pytest.skip("no CUDA device")
    eng = PageRankEngine(0)
    yield eng
    eng.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_matches_reference_labels(engine, name):
    e = CASES[name]
    g = make_graph(e["args"].format(graphs=os.path.join(GOLDEN, "graphs")))
    engine.upload(g)
    comp = engine.connected_components()
    assert hashlib.sha256(comp.tobytes()).hexdigest() == e["labels_sha256"]


@pytest.mark.parametrize("args", ["-g 20", "-u 20 -k 1", "-g 20 -k 1", "-u 16 -k 2"])
def test_gpu_matches_oracle(engine, args):
    g = make_graph(args)
    engine.upload(g)
    assert np.array_equal(engine.connected_components(), oracle.cc_afforest(g))


def test_directed_and_adversarial(engine):
    rng = np.random.default_rng(4)
    d = Graph.from_edges(rng.integers(0, 20000, 15000), rng.integers(0, 20000, 15000))
    engine.upload(d)
    assert np.array_equal(engine.connected_components(), oracle.cc_afforest(d))
    adv = np.load(os.path.join(GOLDEN, "adversarial.npz"))
    for name in ("isolated", "star", "chain", "directed_sinks", "selfdup", "hub5000"):
        g = Graph.from_edges(adv[f"{name}_u"], adv[f"{name}_v"], symmetrize=bool(adv[f"{name}_sym"]))
        engine.upload(g)
        assert np.array_equal(engine.connected_components(), oracle.cc_afforest(g)), name


def test_generated_graph_and_determinism(engine):
    engine.generate("-g 18 -k 4")
    a = engine.connected_components()
    b = engine.connected_components()
    assert np.array_equal(a, b)
    e = CASES["g18k4"]
    assert hashlib.sha256(a.tobytes()).hexdigest() == e["labels_sha256"]


def test_requires_graph():
    if not gpu_available():
        pytest.skip("no CUDA device")
    eng = PageRankEngine(0)
    with pytest.raises(PageRankError):
        eng.connected_components()
    eng.close()
