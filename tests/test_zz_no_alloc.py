"""pr_gpu_run_noalloc: PageRank for callers that cannot allocate GPU memory.

Some callers cannot call cudaMalloc (their GPU memory is reserved up front by
their own pool allocator, or they must not take the device-wide
synchronisation an allocation can cause while serving).  For them the engine
offers one entry point whose working memory is a fixed scratch area compiled
into the library.  This test calls it through the C ABI on buffers the test
itself owns, twice in a row, and checks each result against the regular
entry point (pr_gpu_upload + pr_gpu_run) with the tolerance of the other
parity tests: same sweep count, |a - b| <= 2e-5 |b| + 1e-10 per vertex and
per-sweep L1 errors within 1e-3 relative + 1e-6.

The file is named to be collected last, and it passes alone in a fresh
process as well as after the other tests.
"""
import ctypes

import numpy as np
import pytest

from gapbs_b200 import PageRankEngine
from gapbs_b200._native import pr_lib
from gapbs_b200.graph import Graph, make_graph
from conftest import gpu_available

pytestmark = pytest.mark.gpu


def run_noalloc(g, max_iters=20, epsilon=1e-4, damping=0.85):
    import torch
    dev = torch.device("cuda:0")
    n, m = g.num_nodes, g.num_edges_directed
    in_off = torch.tensor(np.asarray(g.in_offsets, np.int32), device=dev)
    in_nbr = torch.tensor(np.asarray(g.in_neighbors, np.int32), device=dev)
    out_deg = (torch.tensor(np.diff(g.out_offsets).astype(np.int32), device=dev)
               if g.directed else None)
    scores = torch.full((n,), float("nan"), dtype=torch.float32, device=dev)
    sweeps = np.zeros(1, np.int32)
    trace = np.zeros(max(max_iters, 1), np.float64)
    msg = ctypes.create_string_buffer(256)
    torch.cuda.synchronize()
    rc = pr_lib().pr_gpu_run_noalloc(
        0, n, m, in_off.data_ptr(), in_nbr.data_ptr(),
        None if out_deg is None else out_deg.data_ptr(), max_iters, epsilon, damping,
        scores.data_ptr(), sweeps.ctypes.data, trace.ctypes.data, None, msg, 256)
    return rc, msg.value.decode(), scores.cpu().numpy(), int(sweeps[0]), trace[:max_iters]


def regular(g, max_iters=20, epsilon=1e-4):
    eng = PageRankEngine(0)
    eng.upload(g)
    res = eng.run(max_iters, epsilon)
    eng.close()
    return res.scores, int(res.sweeps[0]), res.err_trace[:, 0]


def assert_same(a, b):
    scores, sweeps, trace = a
    ref_scores, ref_sweeps, ref_trace = b
    assert sweeps == ref_sweeps
    assert np.all(np.abs(scores - ref_scores) <= 2e-5 * np.abs(ref_scores) + 1e-10)
    np.testing.assert_allclose(trace[:sweeps], ref_trace[:sweeps], rtol=1e-3, atol=1e-6)


@pytest.fixture(scope="module")
def cuda():
    if not gpu_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("args", ["-g 16", "-u 14", "directed"])
def test_noalloc_matches_regular_entry_point_twice(cuda, args):
    if args == "directed":
        rng = np.random.default_rng(3)
        g = Graph.from_edges(rng.integers(0, 5000, 40000), rng.integers(0, 5000, 40000))
    else:
        g = make_graph(args)
    ref = regular(g)
    for _ in range(2):   # the shared scratch keeps the previous call's contents
        rc, msg, scores, sweeps, trace = run_noalloc(g)
        assert rc == 0, msg
        assert_same((scores, sweeps, trace), ref)


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    lib = pr_lib()
    msg = ctypes.create_string_buffer(256)
    too_many = (1 << 20) + 1
    rc = lib.pr_gpu_run_noalloc(0, too_many, 0, None, None, None, 20, 1e-4, 0.85, None, None,
                                None, None, msg, 256)
    assert rc == -6 and b"PR_GPU_NOALLOC_MAX_VERTICES" in msg.value
    rc = lib.pr_gpu_run_noalloc(0, 10, 0, None, None, None, 5000, 1e-4, 0.85, None, None, None,
                                None, msg, 256)
    assert rc == -6 and b"PR_GPU_NOALLOC_MAX_ITERS" in msg.value
