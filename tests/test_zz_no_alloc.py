"""pr_gpu_run_noalloc: PageRank for callers that cannot allocate GPU memory.

Some callers cannot call cudaMalloc (their GPU memory is reserved up front by
their own pool allocator, or they must not take the device-wide
synchronisation an allocation can cause while serving).  For them the engine
offers one entry point whose working memory is a fixed scratch area compiled
into the library.  This test calls it through the C ABI on buffers the test
itself owns, twice in a row, and checks each result

  * against the regular entry point (pr_gpu_upload + pr_gpu_run): same sweep
    count, |a - b| <= 2e-5 |b| + 1e-10 per vertex, per-sweep L1 changes
    within 1e-5 relative + 8 (R_k + R_(k-1)), R_k the reference's own
    rounding after sweep k (the bound the plain parity tests derive: score
    vectors that differ by e change the sum of |new - old| by at most
    L1(e_k) + L1(e_(k-1)), and each engine's rounding is at most 4 R_k);
  * against the oracle, with the tolerances of the plain parity tests: the
    reference's sweep count (FP32 mirror), |gpu - fp64| <= 2e-5 |fp64| + 1e-10
    per vertex, L1(gpu - fp64) <= 4 L1(reference - fp64) + 1e-7;

and that a second call leaves the device's free memory and torch's allocated
bytes unchanged.  Edge cases: the largest graph the scratch holds
(PR_GPU_NOALLOC_MAX_VERTICES vertices), max_iters = 0, epsilon = 0, invalid
CSRs (PR_GPU_EGRAPH) and sizes beyond the scratch (PR_GPU_ERANGE).

The file is named to be collected last, and it passes alone in a fresh
process as well as after the other tests.
"""
import ctypes

import numpy as np
import pytest

import oracle
from gapbs_b200 import PageRankEngine
from gapbs_b200._native import pr_lib
from gapbs_b200.graph import Graph, make_graph
from conftest import gpu_available

pytestmark = pytest.mark.gpu

MAX_VERTICES = 1 << 20


class NoAllocCall:
    """Device buffers owned by the caller (the test), reused across calls."""

    def __init__(self, g=None, n=None, in_off=None, in_nbr=None, out_deg=None):
        import torch
        dev = torch.device("cuda:0")
        if g is not None:
            n = g.num_nodes
            in_off = np.asarray(g.in_offsets, np.int32)
            in_nbr = np.asarray(g.in_neighbors, np.int32)
            out_deg = np.diff(g.out_offsets).astype(np.int32) if g.directed else None
        self.n, self.m = int(n), int(in_nbr.size)
        self.in_off = torch.tensor(in_off, device=dev)
        self.in_nbr = torch.tensor(in_nbr if in_nbr.size else np.zeros(1, np.int32), device=dev)
        self.out_deg = None if out_deg is None else torch.tensor(out_deg, device=dev)
        self.scores = torch.full((self.n,), float("nan"), dtype=torch.float32, device=dev)
        torch.cuda.synchronize()

    def __call__(self, max_iters=20, epsilon=1e-4, damping=0.85):
        sweeps = np.zeros(1, np.int32)
        trace = np.zeros(max(max_iters, 1), np.float64)
        msg = ctypes.create_string_buffer(256)
        rc = pr_lib().pr_gpu_run_noalloc(
            0, self.n, self.m, self.in_off.data_ptr(), self.in_nbr.data_ptr(),
            None if self.out_deg is None else self.out_deg.data_ptr(), max_iters, epsilon,
            damping, self.scores.data_ptr(), sweeps.ctypes.data, trace.ctypes.data, None, msg,
            256)
        return rc, msg.value.decode(), int(sweeps[0]), trace[:max_iters]

    def scores_host(self):
        return self.scores.cpu().numpy()


def regular(g, max_iters=20, epsilon=1e-4):
    eng = PageRankEngine(0)
    eng.upload(g)
    res = eng.run(max_iters, epsilon)
    eng.close()
    return res.scores, int(res.sweeps[0]), res.err_trace[:, 0]


def assert_matches_regular(g, scores, sweeps, trace, ref, max_iters=20, epsilon=1e-4):
    ref_scores, ref_sweeps, ref_trace = ref
    assert sweeps == ref_sweeps
    assert np.all(np.abs(scores - ref_scores) <= 2e-5 * np.abs(ref_scores) + 1e-10)
    R = oracle.pr_rounding_f32(g, sweeps)
    bound = 1e-5 * ref_trace[:sweeps] + 8 * (R + np.concatenate([[0.0], R[:-1]]))
    assert np.all(np.abs(trace[:sweeps] - ref_trace[:sweeps]) <= bound)


def assert_matches_oracle(g, scores, sweeps, max_iters=20, epsilon=1e-4):
    s32, k32, _ = oracle.pr_pull_f32(g, max_iters, epsilon)
    s64, _, _ = oracle.pr_pull_f64(g, max_iters, epsilon)
    assert sweeps == k32
    assert np.all(np.abs(scores - s64) <= 2e-5 * np.abs(s64) + 1e-10)
    ref_l1 = float(np.abs(s32.astype(np.float64) - s64).sum())
    gpu_l1 = float(np.abs(scores.astype(np.float64) - s64).sum())
    assert gpu_l1 <= 4 * ref_l1 + 1e-7, (gpu_l1, ref_l1)


@pytest.fixture(scope="module")
def cuda():
    if not gpu_available():
        pytest.skip("no CUDA device")


def _graph(args):
    if args == "directed":
        rng = np.random.default_rng(3)
        return Graph.from_edges(rng.integers(0, 5000, 40000), rng.integers(0, 5000, 40000))
    return make_graph(args)


@pytest.mark.parametrize("args", ["-g 16", "-u 14", "directed"])
def test_noalloc_matches_regular_entry_point_twice(cuda, args):
    import torch
    g = _graph(args)
    ref = regular(g)
    call = NoAllocCall(g)
    free_before = None
    for k in range(2):   # the shared scratch keeps the previous call's contents
        rc, msg, sweeps, trace = call()
        assert rc == 0, msg
        torch.cuda.synchronize()
        if k == 0:
            free_before = torch.cuda.mem_get_info()[0]
            alloc_before = torch.cuda.memory_allocated()
        else:
            # the call allocates nothing: the device's free memory and torch's
            # allocated bytes are the same after the second call
            assert torch.cuda.mem_get_info()[0] == free_before
            assert torch.cuda.memory_allocated() == alloc_before
        scores = call.scores_host()
        assert_matches_regular(g, scores, sweeps, trace, ref)
        assert_matches_oracle(g, scores, sweeps)


def test_noalloc_largest_graph_its_scratch_holds(cuda):
    """Exactly PR_GPU_NOALLOC_MAX_VERTICES vertices (a uniform -u 20 graph)."""
    g = make_graph("-u 20 -k 4")
    assert g.num_nodes == MAX_VERTICES
    ref = regular(g)
    call = NoAllocCall(g)
    for _ in range(2):
        rc, msg, sweeps, trace = call()
        assert rc == 0, msg
        scores = call.scores_host()
        assert_matches_regular(g, scores, sweeps, trace, ref)
        assert_matches_oracle(g, scores, sweeps)


def test_noalloc_zero_iterations_and_zero_epsilon(cuda):
    g = make_graph("-g 10")
    call = NoAllocCall(g)
    rc, msg, sweeps, _ = call(max_iters=0)
    assert rc == 0, msg
    assert sweeps == 0
    assert np.all(call.scores_host() == np.float32(1.0) / np.float32(g.num_nodes))
    # epsilon 0 never converges: every one of max_iters sweeps runs
    rc, msg, sweeps, trace = call(max_iters=7, epsilon=0.0)
    assert rc == 0, msg
    assert sweeps == 7
    assert_matches_oracle(g, call.scores_host(), sweeps, max_iters=7, epsilon=0.0)


def test_noalloc_rejects_invalid_csr(cuda):
    off = np.array([0, 2, 3, 4], np.int32)
    nbr = np.array([1, 2, 0, 0], np.int32)
    bad_id = nbr.copy()
    bad_id[1] = 3                       # id >= n
    rc, msg, _, _ = NoAllocCall(n=3, in_off=off, in_nbr=bad_id)()
    assert rc == -5 and "invalid CSR" in msg
    bad_end = off.copy()
    bad_end[3] = 3                      # in_off[n] != m
    rc, msg, _, _ = NoAllocCall(n=3, in_off=bad_end, in_nbr=nbr)()
    assert rc == -5 and "invalid CSR" in msg
    rc, msg, sweeps, _ = NoAllocCall(n=3, in_off=off, in_nbr=nbr)()
    assert rc == 0 and sweeps >= 1, msg


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    lib = pr_lib()
    msg = ctypes.create_string_buffer(256)
    too_many = MAX_VERTICES + 1
    rc = lib.pr_gpu_run_noalloc(0, too_many, 0, None, None, None, 20, 1e-4, 0.85, None, None,
                                None, None, msg, 256)
    assert rc == -6 and b"PR_GPU_NOALLOC_MAX_VERTICES" in msg.value
    rc = lib.pr_gpu_run_noalloc(0, 10, 0, None, None, None, 5000, 1e-4, 0.85, None, None, None,
                                None, msg, 256)
    assert rc == -6 and b"PR_GPU_NOALLOC_MAX_ITERS" in msg.value
