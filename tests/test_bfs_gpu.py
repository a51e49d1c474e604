"""Direction-optimizing BFS on the GPU (pr_gpu_bfs) against the reference.

Parents may differ from the reference's (which same-depth candidate claims a
vertex is a race there too), so the checks are the reference's own verifier
(restated in the oracle) and what any BFS tree from the source determines:
the depths along the parent pointers, the reached set and the tree's edge
count, against the reference's DOBFS results in tests/golden/bfs_golden.json
and the oracle's search.
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
from helpers import depths_from_parents

pytestmark = pytest.mark.gpu

with open(os.path.join(GOLDEN, "bfs_golden.json")) as fh:
    CASES = json.load(fh)["cases"]


@pytest.fixture(scope="module")
def engine():
    if not gpu_available():
        pytest.skip("no CUDA device")
    eng = PageRankEngine(0)
    yield eng
    eng.close()


def check(g, src, parent):
    assert oracle.bfs_verify(g, src, parent)
    assert np.array_equal(depths_from_parents(parent, src), oracle.bfs_depths(g, src))


@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_matches_reference(engine, name):
    e = CASES[name]
    g = make_graph(e["args"].format(graphs=os.path.join(GOLDEN, "graphs")))
    engine.upload(g)
    odeg = np.diff(g.out_offsets)
    for run in e["runs"]:
        parent = engine.bfs(run["source"])
        assert oracle.bfs_verify(g, run["source"], parent)
        d = depths_from_parents(parent, run["source"])
        assert hashlib.sha256(d.tobytes()).hexdigest() == run["depth_sha256"]
        assert int((parent >= 0).sum()) == run["reached"]
        assert int(odeg[parent >= 0].sum()) == run["tree_edges"]


@pytest.mark.parametrize("args", ["-g 20", "-u 20", "-g 18 -k 2", "-u 16 -k 1"])
def test_gpu_bfs_larger_graphs(engine, args):
    g = make_graph(args)
    engine.upload(g)
    rng = np.random.default_rng(1)
    cand = np.nonzero(np.diff(g.out_offsets) > 0)[0]
    for src in rng.choice(cand, 3, replace=False):
        parent, steps = engine.bfs(int(src), with_steps=True)
        check(g, int(src), parent)
        assert steps[0][0] == "i"
        assert {k for k, _, _ in steps} <= {"i", "td", "e", "bu", "c"}


def test_directed_and_adversarial(engine):
    rng = np.random.default_rng(6)
    d = Graph.from_edges(rng.integers(0, 20000, 80000), rng.integers(0, 20000, 80000))
    engine.upload(d)
    for src in (0, 17, 4242):
        check(d, src, engine.bfs(src))
    adv = np.load(os.path.join(GOLDEN, "adversarial.npz"))
    for name in ("isolated", "star", "chain", "directed_sinks", "selfdup", "hub5000"):
        g = Graph.from_edges(adv[f"{name}_u"], adv[f"{name}_v"], symmetrize=bool(adv[f"{name}_sym"]))
        engine.upload(g)
        for src in {0, g.num_nodes - 1, g.num_nodes // 2}:
            check(g, src, engine.bfs(src))


def test_generated_graph_and_errors(engine):
    engine.generate("-g 16")
    e = CASES["g16"]
    src = e["runs"][0]["source"]
    parent = engine.bfs(src)
    d = depths_from_parents(parent, src)
    assert hashlib.sha256(d.tobytes()).hexdigest() == e["runs"][0]["depth_sha256"]
    with pytest.raises(PageRankError):
        engine.bfs(-1)
    with pytest.raises(PageRankError):
        engine.bfs(engine.n)


def layered(widths, rng, extra=1):
    """Source 0, then layers of the given widths; every vertex of a layer has
    one edge from a random vertex of the layer before, plus `extra` more."""
    us, vs = [], []
    prev = np.array([0])
    nxt = 1
    for w in widths:
        layer = np.arange(nxt, nxt + w)
        nxt += w
        for _ in range(1 + extra):
            us.append(rng.choice(prev, w))
            vs.append(layer)
        prev = layer
    return np.concatenate(us), np.concatenate(vs)


@pytest.mark.parametrize("widths", [(1023, 2000, 7), (1024, 1025, 3), (1025, 5000, 40, 1),
                                    (3000, 1024, 1023, 2)])
def test_frontier_sizes_around_block_scan(engine, widths):
    # top-down frontiers of up to 1,024 vertices are scanned inside each block,
    # larger ones by a device-wide scan: both sides of the boundary
    rng = np.random.default_rng(sum(widths))
    u, v = layered(widths, rng)
    for sym in (True, False):
        g = Graph.from_edges(u, v, symmetrize=sym)
        engine.upload(g)
        check(g, 0, engine.bfs(0))


def test_directed_source_without_in_edges(engine):
    # the source has out-edges only (it sorts after every row with in-edges)
    # and a large degree, so the search goes bottom-up from the first step and
    # stays there for several steps
    rng = np.random.default_rng(11)
    u, v = layered((20000, 30000, 30000, 500, 20), rng, extra=2)
    g = Graph.from_edges(u, v, symmetrize=False)
    engine.upload(g)
    parent, steps = engine.bfs(0, with_steps=True)
    check(g, 0, parent)
    kinds = [k for k, _, _ in steps]
    assert kinds[1] == "e" and kinds.count("bu") >= 3


def test_host_stepped_mode_matches(tmp_path):
    # GAPBS_PR_PLAIN_LAUNCH=1 runs the same step kernels launched one by one
    # from the host (the mode profilers use); same trees, same step sequence
    if not gpu_available():
        pytest.skip("no CUDA device")
    import subprocess
    import sys
    script = tmp_path / "plain_bfs.py"
    script.write_text(
        "import json, sys\n"
        "import numpy as np\n"
        "sys.path[:0] = [%r, %r]\n"
        "import oracle\n"
        "from gapbs_b200 import PageRankEngine\n"
        "from gapbs_b200.graph import make_graph\n"
        "from helpers import depths_from_parents\n"
        "eng = PageRankEngine(0)\n"
        "out = []\n"
        "for args in ('-g 14', '-u 12', '-g 12 -k 2'):\n"
        "    g = make_graph(args)\n"
        "    eng.upload(g)\n"
        "    cand = np.nonzero(np.diff(g.out_offsets) > 0)[0]\n"
        "    for src in (int(cand[0]), int(cand[-1])):\n"
        "        parent, steps = eng.bfs(src, with_steps=True)\n"
        "        ok = oracle.bfs_verify(g, src, parent) and np.array_equal(\n"
        "            depths_from_parents(parent, src), oracle.bfs_depths(g, src))\n"
        "        out.append([args, src, bool(ok), [k for k, _, _ in steps]])\n"
        "print(json.dumps(out))\n" % (os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                      os.path.dirname(os.path.abspath(__file__))))
    res = {}
    for mode in ("0", "1"):
        env = dict(os.environ, GAPBS_PR_PLAIN_LAUNCH=mode)
        r = subprocess.run([sys.executable, str(script)], env=env, capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        res[mode] = json.loads(r.stdout.strip().splitlines()[-1])
    assert all(ok for _, _, ok, _ in res["0"]) and all(ok for _, _, ok, _ in res["1"])
    assert [k for *_, k in res["0"]] == [k for *_, k in res["1"]]


def test_step_log_truncated_to_caller_buffer(engine):
    # pr_gpu_bfs fills at most max_steps records and reports the full count
    import ctypes
    g = make_graph("-g 14")
    engine.upload(g)
    src = int(np.argmax(np.diff(g.out_offsets)))
    full_parent, full = engine.bfs(src, with_steps=True)
    lib = engine._lib
    parent = np.empty(g.num_nodes, np.int32)
    rec = np.zeros(2, dtype=np.dtype([("kind", "S4"), ("count", "<i8"), ("seconds", "<f8")],
                                      align=True))
    nsteps = ctypes.c_int()
    rc = lib.pr_gpu_bfs(engine._h, src, parent.ctypes.data, rec.ctypes.data, 2,
                        ctypes.byref(nsteps))
    assert rc == 0
    assert nsteps.value == len(full) > 2
    assert [r["kind"].decode() for r in rec] == [k for k, _, _ in full[:2]]
    assert oracle.bfs_verify(g, src, parent)
    # no step buffer at all: still the count
    rc = lib.pr_gpu_bfs(engine._h, src, parent.ctypes.data, None, 0, ctypes.byref(nsteps))
    assert rc == 0 and nsteps.value == len(full)
