"""TEST INFRASTRUCTURE ONLY -- the checker, never the product.

ctypes wrappers over
  * ``liboracle.so``: the CPU restatement of the reference's PageRankPull /
    PRVerifier (src/pr_spmv.cc:35-61,78-94) plus FP64 PPR and adjoint;
  * ``_ref/libgapbs_ref.so``: the reference's own code compiled from its
    sources (built only where the reference tree exists; the built file then
    travels with the repository snapshot).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this package.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_lib = None
_ref = None

P = c_void_p


def _ptr(a):
    return None if a is None else a.ctypes.data


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing; run `make -C oracle`")
        L = ctypes.CDLL(path)
        L.oracle_pr_pull_f32.argtypes = [c_int64, P, P, P, c_int, c_double, c_float, P, P]
        L.oracle_pr_pull_f32.restype = c_int
        L.oracle_pr_pull_f64.argtypes = [c_int64, P, P, P, c_int, c_double, c_double, P, P]
        L.oracle_pr_pull_f64.restype = c_int
        L.oracle_pr_verify_f32.argtypes = [c_int64, P, P, c_float, P]
        L.oracle_pr_verify_f32.restype = c_double
        L.oracle_pr_residual_f64.argtypes = [c_int64, P, P, P, c_float, P]
        L.oracle_pr_residual_f64.restype = c_double
        L.oracle_bfs_depths.argtypes = [c_int64, P, P, c_int, P]
        L.oracle_bfs_depths.restype = None
        L.oracle_bfs_verify.argtypes = [c_int64, P, P, P, P, c_int, P]
        L.oracle_bfs_verify.restype = c_int
        L.oracle_cc_afforest.argtypes = [c_int64, P, P, P, P, c_int, P]
        L.oracle_cc_afforest.restype = None
        L.oracle_ppr_residual_f64.argtypes = [c_int64, P, P, P, c_float, P, P]
        L.oracle_ppr_residual_f64.restype = c_double
        L.oracle_ppr_f64.argtypes = [c_int64, P, P, P, P, P, c_double, P, c_int, c_double, P, P]
        L.oracle_ppr_f64.restype = c_int
        L.oracle_ppr_f64_from.argtypes = [c_int64, P, P, P, P, P, c_double, P, P, c_int, c_double, P, P]
        L.oracle_ppr_f64_from.restype = c_int
        L.oracle_pr_rounding_f32.argtypes = [c_int64, P, P, P, c_int, c_float, P]
        L.oracle_pr_rounding_f32.restype = None
        L.oracle_ppr_adjoint_f64.argtypes = [c_int64, P, P, P, c_double, P, P, c_int, c_double, P, P, P]
        L.oracle_ppr_adjoint_f64.restype = c_int
        _lib = L
    return _lib


def _csr(g):
    """(n, in_off, in_nbr, out_off, out_nbr) as contiguous int64/int32 arrays."""
    n = g.num_nodes
    return (n,
            np.ascontiguousarray(g.in_offsets, np.int64),
            np.ascontiguousarray(g.in_neighbors, np.int32),
            np.ascontiguousarray(g.out_offsets, np.int64),
            np.ascontiguousarray(g.out_neighbors, np.int32))


def pr_pull_f32(g, max_iters=20, epsilon=1e-4, damping=0.85):
    """FP32 mirror of PageRankPull -> (scores float32, sweeps, err_trace)."""
    n, io, inb, oo, _ = _csr(g)
    s = np.empty(n, np.float32)
    tr = np.zeros(max(max_iters, 1), np.float64)
    k = lib().oracle_pr_pull_f32(n, _ptr(io), _ptr(inb), _ptr(oo), max_iters, epsilon,
                                 damping, _ptr(s), _ptr(tr))
    return s, k, tr[:k].copy()


def pr_pull_f64(g, max_iters=20, epsilon=1e-4, damping=0.85):
    n, io, inb, oo, _ = _csr(g)
    s = np.empty(n, np.float64)
    tr = np.zeros(max(max_iters, 1), np.float64)
    k = lib().oracle_pr_pull_f64(n, _ptr(io), _ptr(inb), _ptr(oo), max_iters, epsilon,
                                 damping, _ptr(s), _ptr(tr))
    return s, k, tr[:k].copy()


def pr_rounding_f32(g, nsweeps, damping=0.85):
    """Per sweep, L1 distance of the reference's FP32 scores from FP64 Jacobi
    run side by side from the same start (the reference's own rounding)."""
    n, io, inb, oo, _ = _csr(g)
    l1 = np.zeros(max(nsweeps, 1), np.float64)
    lib().oracle_pr_rounding_f32(n, _ptr(io), _ptr(inb), _ptr(oo), int(nsweeps), damping,
                                 _ptr(l1))
    return l1[:nsweeps].copy()


def pr_verify_f32(g, scores, damping=0.85) -> float:
    """PRVerifier's total error (pass when < tolerance)."""
    n, _, _, oo, onb = _csr(g)
    s = np.ascontiguousarray(scores, np.float32)
    return float(lib().oracle_pr_verify_f32(n, _ptr(oo), _ptr(onb), damping, _ptr(s)))


def pr_residual_f64(g, scores, damping=0.85) -> float:
    n, io, inb, oo, _ = _csr(g)
    s = np.ascontiguousarray(scores, np.float32)
    return float(lib().oracle_pr_residual_f64(n, _ptr(io), _ptr(inb), _ptr(oo), damping, _ptr(s)))


def cc_afforest(g) -> np.ndarray:
    """Component labels by the serial restatement of the reference's Afforest."""
    n = g.num_nodes
    oo = np.ascontiguousarray(g.out_offsets, np.int64)
    on = np.ascontiguousarray(g.out_neighbors, np.int32)
    io = np.ascontiguousarray(g.in_offsets, np.int64)
    inb = np.ascontiguousarray(g.in_neighbors, np.int32)
    comp = np.empty(n, np.int32)
    lib().oracle_cc_afforest(n, _ptr(oo), _ptr(on), _ptr(io), _ptr(inb), int(g.directed),
                             _ptr(comp))
    return comp


def bfs_depths(g, source: int) -> np.ndarray:
    """BFS depths from source (-1 unreachable), the reference verifier's search."""
    oo = np.ascontiguousarray(g.out_offsets, np.int64)
    on = np.ascontiguousarray(g.out_neighbors, np.int32)
    depth = np.empty(g.num_nodes, np.int32)
    lib().oracle_bfs_depths(g.num_nodes, _ptr(oo), _ptr(on), int(source), _ptr(depth))
    return depth


def bfs_verify(g, source: int, parent) -> bool:
    """The reference's BFSVerifier restated."""
    oo = np.ascontiguousarray(g.out_offsets, np.int64)
    on = np.ascontiguousarray(g.out_neighbors, np.int32)
    io = np.ascontiguousarray(g.in_offsets, np.int64)
    inb = np.ascontiguousarray(g.in_neighbors, np.int32)
    p = np.ascontiguousarray(parent, np.int32)
    return bool(lib().oracle_bfs_verify(g.num_nodes, _ptr(oo), _ptr(on), _ptr(io), _ptr(inb),
                                        int(source), _ptr(p)))


def ref_bfs(args: str, k: int = 1, source: int = -1, run: bool = True):
    """The reference's SourcePicker and DOBFS on the graph its builder makes
    for args.  Returns (first k picked sources, parents from `source` or the
    first pick, kernel seconds); parents is None when run is False."""
    path = os.path.join(REF_DIR, "libgapbs_ref_bfs.so")
    if not os.path.exists(path):
        raise RuntimeError(f"{path} missing (built by `make -C oracle` where the reference "
                           "tree exists)")
    R = ctypes.CDLL(path)
    R.ref_bfs.argtypes = [c_int, POINTER(c_char_p), c_int, P, c_int64, P, c_int64,
                          POINTER(c_double)]
    R.ref_bfs.restype = c_int64
    toks = ["bfs"] + args.split()
    argv = (c_char_p * len(toks))(*[t.encode() for t in toks])
    srcs = np.empty(max(k, 1), np.int32)
    sec = c_double()
    n = R.ref_bfs(len(toks), argv, k, _ptr(srcs), -1, None, 0, ctypes.byref(sec))
    if n < 0:
        raise RuntimeError(f"reference rejected {args!r}")
    parent = None
    if run:
        parent = np.empty(n, np.int32)
        R.ref_bfs(len(toks), argv, k, _ptr(srcs), int(source), _ptr(parent), n,
                  ctypes.byref(sec))
    return srcs[:k], parent, float(sec.value)


def ref_bfs_csr(g, sources):
    """The reference's DOBFS on graph g's CSR from each source in turn.
    Returns (last search's parents, total kernel seconds)."""
    path = os.path.join(REF_DIR, "libgapbs_ref_bfs.so")
    if not os.path.exists(path):
        raise RuntimeError(f"{path} missing (built by `make -C oracle` where the reference "
                           "tree exists)")
    R = ctypes.CDLL(path)
    R.ref_bfs_csr.argtypes = [c_int64, c_int, P, P, P, P, c_int, P, P]
    R.ref_bfs_csr.restype = c_double
    oo = np.ascontiguousarray(g.out_offsets, np.int64)
    on = np.ascontiguousarray(g.out_neighbors, np.int32)
    io = np.ascontiguousarray(g.in_offsets, np.int64)
    inb = np.ascontiguousarray(g.in_neighbors, np.int32)
    src = np.ascontiguousarray(sources, np.int32)
    parent = np.empty(g.num_nodes, np.int32)
    sec = R.ref_bfs_csr(g.num_nodes, int(g.directed), _ptr(oo), _ptr(on), _ptr(io), _ptr(inb),
                        int(src.size), _ptr(src), _ptr(parent))
    return parent, float(sec)


def ref_cc_afforest(args: str):
    """The reference's own Afforest on the graph its builder makes for args
    (pr_spmv-style options).  Returns (labels, kernel seconds)."""
    path = os.path.join(REF_DIR, "libgapbs_ref_cc.so")
    if not os.path.exists(path):
        raise RuntimeError(f"{path} missing (built by `make -C oracle` where the reference "
                           "tree exists)")
    R = ctypes.CDLL(path)
    R.ref_cc_afforest.argtypes = [c_int, POINTER(c_char_p), P, c_int64, POINTER(c_double)]
    R.ref_cc_afforest.restype = c_int64
    toks = ["cc"] + args.split()
    argv = (c_char_p * len(toks))(*[t.encode() for t in toks])
    sec = c_double()
    n = R.ref_cc_afforest(len(toks), argv, None, 0, ctypes.byref(sec))
    if n < 0:
        raise RuntimeError(f"reference rejected {args!r}")
    comp = np.empty(n, np.int32)
    R.ref_cc_afforest(len(toks), argv, _ptr(comp), n, ctypes.byref(sec))
    return comp, float(sec.value)


def ref_cc_afforest_csr(g, trials: int = 1):
    """The reference's Afforest on graph g's CSR.  Returns (labels, fastest
    kernel seconds over `trials` runs)."""
    path = os.path.join(REF_DIR, "libgapbs_ref_cc.so")
    if not os.path.exists(path):
        raise RuntimeError(f"{path} missing (built by `make -C oracle` where the reference "
                           "tree exists)")
    R = ctypes.CDLL(path)
    R.ref_cc_afforest_csr.argtypes = [c_int64, c_int, P, P, P, P, c_int, P]
    R.ref_cc_afforest_csr.restype = c_double
    oo = np.ascontiguousarray(g.out_offsets, np.int64)
    on = np.ascontiguousarray(g.out_neighbors, np.int32)
    io = np.ascontiguousarray(g.in_offsets, np.int64)
    inb = np.ascontiguousarray(g.in_neighbors, np.int32)
    comp = np.empty(g.num_nodes, np.int32)
    sec = R.ref_cc_afforest_csr(g.num_nodes, int(g.directed), _ptr(oo), _ptr(on), _ptr(io),
                                _ptr(inb), int(trials), _ptr(comp))
    return comp, float(sec)


def ppr_residual_f64(g, t, s, damping=0.85) -> float:
    """L1 residual of one PPR score column (unit weights); see pr_oracle.h."""
    n, io, inb, oo, _ = _csr(g)
    t = np.ascontiguousarray(t, np.float32)
    s = np.ascontiguousarray(s, np.float32)
    return float(lib().oracle_ppr_residual_f64(n, _ptr(io), _ptr(inb), _ptr(oo), damping,
                                               _ptr(t), _ptr(s)))


def ppr_f64(n, in_off, in_nbr, out_off, t, in_w=None, rowsum=None, damping=0.85,
            max_iters=20, epsilon=1e-4, s_init=None):
    t = np.ascontiguousarray(t, np.float64)
    s = np.empty(n, np.float64)
    tr = np.zeros(max(max_iters, 1), np.float64)
    in_off = np.ascontiguousarray(in_off, np.int64)
    in_nbr = np.ascontiguousarray(in_nbr, np.int32)
    out_off = np.ascontiguousarray(out_off, np.int64)
    in_w = None if in_w is None else np.ascontiguousarray(in_w, np.float64)
    rowsum = None if rowsum is None else np.ascontiguousarray(rowsum, np.float64)
    if s_init is None:
        k = lib().oracle_ppr_f64(n, _ptr(in_off), _ptr(in_nbr), _ptr(in_w), _ptr(rowsum),
                                 _ptr(out_off), damping, _ptr(t), max_iters, epsilon,
                                 _ptr(s), _ptr(tr))
    else:
        s0 = np.ascontiguousarray(s_init, np.float64)
        k = lib().oracle_ppr_f64_from(n, _ptr(in_off), _ptr(in_nbr), _ptr(in_w), _ptr(rowsum),
                                      _ptr(out_off), damping, _ptr(t), _ptr(s0), max_iters,
                                      epsilon, _ptr(s), _ptr(tr))
    return s, k, tr[:k].copy()


def ppr_adjoint_f64(n, out_off, out_nbr, loss_w, s, out_w=None, damping=0.85,
                    max_iters=200, epsilon=1e-4):
    out_off = np.ascontiguousarray(out_off, np.int64)
    out_nbr = np.ascontiguousarray(out_nbr, np.int32)
    out_w = None if out_w is None else np.ascontiguousarray(out_w, np.float64)
    loss_w = np.ascontiguousarray(loss_w, np.float64)
    s = np.ascontiguousarray(s, np.float64)
    lam = np.empty(n, np.float64)
    gt = np.empty(n, np.float64)
    gw = np.empty(out_nbr.size, np.float64)
    k = lib().oracle_ppr_adjoint_f64(n, _ptr(out_off), _ptr(out_nbr), _ptr(out_w), damping,
                                     _ptr(loss_w), _ptr(s), max_iters, epsilon, _ptr(lam),
                                     _ptr(gt), _ptr(gw))
    return lam, gt, gw, k


# ---------------------------------------------------------------------------
# The reference itself (oracle/_ref), compiled from its sources.

def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libgapbs_ref.so"))


def ref() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        path = os.path.join(REF_DIR, "libgapbs_ref.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing (built by `make -C oracle` where the "
                               "reference tree exists)")
        R = ctypes.CDLL(path)
        R.ref_make_graph.argtypes = [c_int, POINTER(c_char_p)]
        R.ref_make_graph.restype = P
        R.ref_graph_from_csr.argtypes = [c_int64, c_int, P, P, P, P]
        R.ref_graph_from_csr.restype = P
        R.ref_free_graph.argtypes = [P]
        R.ref_free_graph.restype = None
        for fn in ("ref_num_nodes", "ref_num_edges", "ref_num_edges_directed"):
            getattr(R, fn).argtypes = [P]
            getattr(R, fn).restype = c_int64
        R.ref_directed.argtypes = [P]
        R.ref_directed.restype = c_int
        R.ref_export_csr.argtypes = [P, P, P, P, P]
        R.ref_export_csr.restype = None
        R.ref_pagerank_pull.argtypes = [P, c_int, c_double, c_int, P]
        R.ref_pagerank_pull.restype = None
        R.ref_time_pagerank_pull.argtypes = [P, c_int, c_double, c_int, P]
        R.ref_time_pagerank_pull.restype = c_double
        R.ref_pagerank_gs.argtypes = [P, c_int, c_double, c_int, P]
        R.ref_pagerank_gs.restype = None
        R.ref_time_pagerank_gs.argtypes = [P, c_int, c_double, c_int, P]
        R.ref_time_pagerank_gs.restype = c_double
        R.ref_pr_verifier.argtypes = [P, P, c_double]
        R.ref_pr_verifier.restype = c_int
        _ref = R
    return _ref


class RefGraph:
    """A graph held by the reference's own CSRGraph."""

    def __init__(self, handle):
        self.h = handle
        R = ref()
        self.num_nodes = int(R.ref_num_nodes(handle))
        self.num_edges = int(R.ref_num_edges(handle))
        self.num_edges_directed = int(R.ref_num_edges_directed(handle))
        self.directed = bool(R.ref_directed(handle))

    @staticmethod
    def build(args: str) -> "RefGraph":
        toks = ["pr_spmv"] + args.split()
        argv = (c_char_p * len(toks))(*[t.encode() for t in toks])
        h = ref().ref_make_graph(len(toks), argv)
        if not h:
            raise RuntimeError(f"reference builder rejected {args!r}")
        return RefGraph(h)

    @staticmethod
    def from_csr(g) -> "RefGraph":
        oo = np.ascontiguousarray(g.out_offsets, np.int64)
        onb = np.ascontiguousarray(g.out_neighbors, np.int32)
        io = np.ascontiguousarray(g.in_offsets, np.int64)
        inb = np.ascontiguousarray(g.in_neighbors, np.int32)
        h = ref().ref_graph_from_csr(g.num_nodes, int(g.directed), _ptr(oo), _ptr(onb),
                                     _ptr(io), _ptr(inb))
        return RefGraph(h)

    def csr(self):
        n = self.num_nodes
        R = ref()
        oo = np.empty(n + 1, np.int64)
        m = self.num_edges_directed
        onb = np.empty(max(m, 1), np.int32)
        if self.directed:
            io = np.empty(n + 1, np.int64)
            inb = np.empty(max(m, 1), np.int32)
            R.ref_export_csr(self.h, _ptr(oo), _ptr(onb), _ptr(io), _ptr(inb))
            return oo, onb[:m], io, inb[:m]
        R.ref_export_csr(self.h, _ptr(oo), _ptr(onb), None, None)
        return oo, onb[:m], oo, onb[:m]

    def pagerank_pull(self, max_iters=20, epsilon=1e-4, logging=False):
        s = np.empty(self.num_nodes, np.float32)
        ref().ref_pagerank_pull(self.h, max_iters, epsilon, int(logging), _ptr(s))
        return s

    def time_pagerank_pull(self, trials=1, max_iters=20, epsilon=1e-4):
        per = np.zeros(trials, np.float64)
        tot = ref().ref_time_pagerank_pull(self.h, max_iters, epsilon, trials, _ptr(per))
        return tot, per

    def pagerank_gs(self, max_iters=20, epsilon=1e-4, logging=False):
        """The reference's Gauss-Seidel PageRankPullGS (src/pr.cc:34-61)."""
        s = np.empty(self.num_nodes, np.float32)
        ref().ref_pagerank_gs(self.h, max_iters, epsilon, int(logging), _ptr(s))
        return s

    def time_pagerank_gs(self, trials=1, max_iters=20, epsilon=1e-4):
        per = np.zeros(trials, np.float64)
        tot = ref().ref_time_pagerank_gs(self.h, max_iters, epsilon, trials, _ptr(per))
        return tot, per

    def verify(self, scores, tolerance=1e-4) -> bool:
        s = np.ascontiguousarray(scores, np.float32)
        return bool(ref().ref_pr_verifier(self.h, _ptr(s), tolerance))

    def __del__(self):
        if getattr(self, "h", None):
            ref().ref_free_graph(self.h)
            self.h = None
