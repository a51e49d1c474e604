"""PageRank on the B200 engine (``libgapbs_pr.so``) -- the Python host mirror.

``PageRankPull(g, max_iters, epsilon, logging_enabled)`` keeps the reference's
signature and result (src/pr_spmv.cc:35-61): float32 scores, the same sweep
count, and with ``logging_enabled`` the same per-sweep lines
(src/util.h:37-46).  The graph is uploaded to the GPU once and cached on the
``Graph`` object, so repeated trials do not re-upload (the reference's graph
likewise stays resident between trials, src/benchmark.h:100-123).

``PageRankEngine`` is the handle-level API over include/pr_gpu.h: upload,
single and batched (personalized) solves from host or device buffers, the
adjoint, timing and graph facts.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import byref, c_double, c_int, c_int32, c_int64, c_void_p
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _pr_abi
from ._native import graph_lib, pr_lib
from .graph import Graph

K_DAMP = np.float32(0.85)   # kDamp, src/pr_spmv.cc:33
NUM_BINS = 8


class PageRankError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (pr_gpu code {code})")
        self.code = code


def _ptr(a) -> Optional[int]:
    return None if a is None else a.ctypes.data


@dataclass
class PageRankResult:
    scores: np.ndarray          # float32, (n,) or (n, ncols)
    sweeps: np.ndarray          # int32 per column
    err_trace: np.ndarray       # float64, (max_iters, ncols)

    @property
    def num_sweeps(self) -> int:
        return int(self.sweeps.max()) if self.sweeps.size else 0


class PageRankEngine:
    """One engine handle on one CUDA device, holding at most one graph."""

    def __init__(self, device: int = 0):
        self._lib = pr_lib()
        self._h = ctypes.c_void_p()
        rc = self._lib.pr_gpu_create(byref(self._h), int(device))
        if rc != 0:
            raise PageRankError(rc, "pr_gpu_create failed (is a CUDA device visible?)")
        self.device = device
        self.n = 0
        self.m = 0
        self.directed = False
        self.weighted = False

    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = self._lib.pr_gpu_last_error(self._h)
            raise PageRankError(rc, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.pr_gpu_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- upload ---------------------------------------------------------------
    def upload_csr(self, n: int, out_off, out_nbr, in_off=None, in_nbr=None, edge_w=None):
        """CSR with int32 offsets/ids (converted if needed); in_* None => undirected."""
        oo = np.ascontiguousarray(out_off, dtype=np.int32)
        on = np.ascontiguousarray(out_nbr, dtype=np.int32)
        m = int(on.size)
        io = inb = None
        if in_off is not None:
            io = np.ascontiguousarray(in_off, dtype=np.int32)
            inb = np.ascontiguousarray(in_nbr, dtype=np.int32)
        w = None if edge_w is None else np.ascontiguousarray(edge_w, dtype=np.float32)
        if w is not None and w.size != m:
            raise ValueError("edge_w must hold one weight per out-CSR entry")
        rc = self._lib.pr_gpu_upload(self._h, int(n), m, _ptr(oo), _ptr(on), _ptr(io), _ptr(inb),
                                     _ptr(w))
        self._check(rc, "pr_gpu_upload")
        self.n, self.m = int(n), m
        self.directed = io is not None
        self.weighted = w is not None

    def set_edge_weights_device(self, w_ptr: int):
        """New edge weights for the weighted graph on the device, from a
        device pointer to m float32 weights in the uploaded out-CSR order
        (pr_gpu_set_edge_weights_device): no host copy, no re-upload."""
        self._check(self._lib.pr_gpu_set_edge_weights_device(self._h, c_void_p(int(w_ptr))),
                    "pr_gpu_set_edge_weights_device")

    def upload(self, g: Graph, edge_w=None):
        if g.num_edges_directed > 0x7FFFFFFF - 8:
            raise PageRankError(_pr_abi.PR_GPU_ERANGE, "graph exceeds int32 offsets")
        if g.directed:
            self.upload_csr(g.num_nodes, g.out_offsets, g.out_neighbors, g.in_offsets,
                            g.in_neighbors, edge_w)
        else:
            self.upload_csr(g.num_nodes, g.out_offsets, g.out_neighbors, None, None, edge_w)

    def bfs(self, source: int, with_steps: bool = False):
        """Direction-optimizing BFS from `source`: parent of every vertex
        (the source for itself, -1 when unreachable).  with_steps: also the
        step log [(kind, count, seconds)] as the reference prints it with -l."""
        parent = np.empty(self.n, np.int32)
        steps = np.zeros(256, dtype=np.dtype([("kind", "S4"), ("count", "<i8"), ("seconds", "<f8")],
                                             align=True))  # pr_gpu_bfs_step_t, 24 bytes
        nsteps = ctypes.c_int()
        self._check(self._lib.pr_gpu_bfs(self._h, int(source), _ptr(parent), _ptr(steps),
                                         steps.size, byref(nsteps)), "pr_gpu_bfs")
        if not with_steps:
            return parent
        k = min(nsteps.value, steps.size)
        return parent, [(s["kind"].decode(), int(s["count"]), float(s["seconds"]))
                        for s in steps[:k]]

    def bfs_device(self, source: int, parent_ptr: int) -> int:
        """BFS parents into a device buffer of n int32; returns the step count."""
        nsteps = ctypes.c_int()
        self._check(self._lib.pr_gpu_bfs_device(self._h, int(source), parent_ptr, None, 0,
                                                byref(nsteps)), "pr_gpu_bfs_device")
        return nsteps.value

    def connected_components(self) -> np.ndarray:
        """Component label of every vertex of the uploaded graph: the smallest
        vertex id of its component (the reference's Afforest labelling)."""
        comp = np.empty(self.n, np.int32)
        self._check(self._lib.pr_gpu_connected_components(self._h, _ptr(comp)),
                    "pr_gpu_connected_components")
        return comp

    def connected_components_device(self, comp_ptr: int):
        """Component labels into a device buffer of n int32 (on the handle's GPU)."""
        self._check(self._lib.pr_gpu_connected_components_device(self._h, comp_ptr),
                    "pr_gpu_connected_components_device")

    def upload_sg(self, path: str):
        """Uploads a serialized (.sg) graph file straight to the device (no host
        CSR); returns (num_nodes, CSR entries)."""
        rc = self._lib.pr_gpu_upload_sg(self._h, os.fsencode(path))
        self._check(rc, "pr_gpu_upload_sg")
        with open(path, "rb") as fh:
            head = fh.read(17)  # bool directed, int64 entries, int64 n
        self.directed = head[0] != 0
        self.m = int.from_bytes(head[1:9], "little", signed=True)
        self.n = int.from_bytes(head[9:17], "little", signed=True)
        self.weighted = False
        return self.n, self.m

    def generate(self, args: str):
        """Builds pr_spmv's synthetic graph ("-g SCALE [-k DEGREE]" or
        "-u SCALE [-k DEGREE]") on the device, identical to the reference's,
        and uploads it.  Returns (num_nodes, CSR entries)."""
        toks = args.split()
        kind = scale = None
        degree = 16
        i = 0
        while i < len(toks):
            if toks[i] in ("-g", "-u") and i + 1 < len(toks):
                kind, scale = toks[i], int(toks[i + 1])
                i += 2
            elif toks[i] == "-k" and i + 1 < len(toks):
                degree = int(toks[i + 1])
                i += 2
            else:
                raise ValueError(f"generate takes -g/-u SCALE [-k DEGREE], got {args!r}")
        if kind is None:
            raise ValueError("generate needs -g SCALE or -u SCALE")
        perm = None
        if kind == "-g":
            perm = np.empty(1 << scale, np.int32)
            if graph_lib().gapbs_rmat_permutation(scale, _ptr(perm)) != 0:
                raise ValueError(f"invalid scale {scale}")
        n, m = ctypes.c_int64(), ctypes.c_int64()
        rc = self._lib.pr_gpu_generate(self._h, int(kind == "-u"), scale, degree, _ptr(perm),
                                       byref(n), byref(m))
        self._check(rc, "pr_gpu_generate")
        self.n, self.m = int(n.value), int(m.value)
        self.directed = False
        self.weighted = False
        return self.n, self.m

    def download_graph(self) -> Graph:
        """The last generated graph as a host Graph (frees its device copy)."""
        lib = graph_lib()
        h = ctypes.c_void_p()
        off = ctypes.POINTER(ctypes.c_int64)()
        nbr = ctypes.POINTER(ctypes.c_int32)()
        if lib.gapbs_graph_new_undirected(byref(h), self.n, self.m, byref(off), byref(nbr)) != 0:
            raise MemoryError("host graph allocation failed")
        rc = self._lib.pr_gpu_download_csr(self._h, ctypes.cast(off, ctypes.c_void_p),
                                           ctypes.cast(nbr, ctypes.c_void_p))
        if rc != 0:
            lib.gapbs_graph_free(h)
            self._check(rc, "pr_gpu_download_csr")
        return Graph(h)

    # -- solves ---------------------------------------------------------------
    def run(self, max_iters: int = 20, epsilon: float = 1e-4, damping: float = float(K_DAMP),
            teleport=None, out: Optional[np.ndarray] = None) -> PageRankResult:
        """Host buffers in and out.  teleport: None, (n,) or (n, ncols) float32.
        out: optional preallocated float32 buffer of n * ncols elements (for
        example pinned memory) that receives the scores."""
        ncols = 1
        tele = None
        if teleport is not None:
            tele = np.ascontiguousarray(teleport, dtype=np.float32)
            if tele.shape[0] != self.n:
                raise ValueError("teleport must have one row per vertex")
            ncols = 1 if tele.ndim == 1 else int(tele.shape[1])
        if out is None:
            out = np.empty((self.n, ncols), np.float32)
        else:
            if out.dtype != np.float32 or out.size != self.n * ncols or not out.flags.c_contiguous:
                raise ValueError("out must be a contiguous float32 buffer of n * ncols elements")
            out = out.reshape(self.n, ncols)
        sweeps = np.zeros(ncols, np.int32)
        trace = np.zeros((max(max_iters, 1), ncols), np.float64)
        rc = self._lib.pr_gpu_run(self._h, int(max_iters), float(epsilon), float(damping), ncols,
                                  _ptr(tele), _ptr(out), _ptr(sweeps), _ptr(trace))
        self._check(rc, "pr_gpu_run")
        if teleport is None or (tele is not None and tele.ndim == 1):
            out = out.reshape(self.n)
        return PageRankResult(out, sweeps, trace[:max_iters])

    def run_device(self, max_iters: int, epsilon: float, damping: float, ncols: int,
                   teleport_ptr: Optional[int], out_ptr: int):
        """Device pointers in and out; returns (sweeps, err_trace)."""
        sweeps = np.zeros(ncols, np.int32)
        trace = np.zeros((max(max_iters, 1), ncols), np.float64)
        rc = self._lib.pr_gpu_run_device(self._h, int(max_iters), float(epsilon), float(damping),
                                         int(ncols), teleport_ptr, out_ptr, _ptr(sweeps),
                                         _ptr(trace))
        self._check(rc, "pr_gpu_run_device")
        return sweeps, trace[:max_iters]

    def adjoint(self, loss_w, scores, max_iters: int = 200, epsilon: float = 1e-4,
                damping: float = float(K_DAMP), want_edge_grad: bool = True):
        """Host buffers: returns (grad_teleport (n,), grad_edge_w (m,) or None, sweeps)."""
        w = np.ascontiguousarray(loss_w, dtype=np.float32)
        s = np.ascontiguousarray(scores, dtype=np.float32)
        gt = np.empty(self.n, np.float32)
        ge = np.empty(self.m, np.float32) if want_edge_grad else None
        sw = np.zeros(1, np.int32)
        rc = self._lib.pr_gpu_adjoint(self._h, int(max_iters), float(epsilon), float(damping),
                                      _ptr(w), _ptr(s), _ptr(gt), _ptr(ge), _ptr(sw))
        self._check(rc, "pr_gpu_adjoint")
        return gt, ge, int(sw[0])

    def adjoint_device(self, max_iters: int, epsilon: float, damping: float, loss_w_ptr: int,
                       scores_ptr: int, grad_t_ptr: Optional[int], grad_ew_ptr: Optional[int]) -> int:
        sw = np.zeros(1, np.int32)
        rc = self._lib.pr_gpu_adjoint_device(self._h, int(max_iters), float(epsilon),
                                             float(damping), loss_w_ptr, scores_ptr, grad_t_ptr,
                                             grad_ew_ptr, _ptr(sw))
        self._check(rc, "pr_gpu_adjoint_device")
        return int(sw[0])

    def set_batch_tile(self, width: int):
        """Column tile width of batched solves (8/16/32/64), 0 = autotuned."""
        self._check(self._lib.pr_gpu_set_batch_tile(self._h, int(width)), "pr_gpu_set_batch_tile")

    def batch_tile(self) -> int:
        w = ctypes.c_int()
        self._check(self._lib.pr_gpu_get_batch_tile(self._h, byref(w)), "pr_gpu_get_batch_tile")
        return w.value

    def set_batch_schedule(self, short_len: int = 0, l1_kb: int = 0):
        """Work schedule of batched solves (pr_gpu_set_batch_schedule); 0
        leaves a field to the autotuner."""
        self._check(self._lib.pr_gpu_set_batch_schedule(self._h, int(short_len), int(l1_kb)),
                    "pr_gpu_set_batch_schedule")

    def batch_schedule(self) -> dict:
        """Tile width and schedule batched solves run with."""
        w, sl, kb = c_int(), c_int(), c_int()
        self._check(self._lib.pr_gpu_get_batch_schedule(self._h, byref(w), byref(sl), byref(kb)),
                    "pr_gpu_get_batch_schedule")
        return {"tile_width": w.value, "short_len": sl.value, "l1_kb": kb.value}

    def set_sweep_layout(self, layout: str = "auto", slice_verts: int = 0, bin_words: int = 0):
        """Sweep layout of single-column solves on unweighted graphs:
        "auto" (slice-blocked when the graph fits it), "gather" or "blocked";
        slice_verts / bin_words 0 keep the defaults (see pr_gpu_set_sweep_layout)."""
        code = {"auto": _pr_abi.PR_GPU_SWEEP_AUTO, "gather": _pr_abi.PR_GPU_SWEEP_GATHER,
                "blocked": _pr_abi.PR_GPU_SWEEP_BLOCKED}[layout]
        self._check(self._lib.pr_gpu_set_sweep_layout(self._h, code, int(slice_verts),
                                                      int(bin_words)), "pr_gpu_set_sweep_layout")

    def sweep_layout_info(self) -> dict:
        on, sl, bn, last = c_int(), c_int(), c_int(), c_int()
        pairs, ids, nbytes = c_int64(), c_int64(), c_int64()
        self._check(self._lib.pr_gpu_sweep_layout_info(self._h, byref(on), byref(sl), byref(bn),
                                                       byref(pairs), byref(ids), byref(nbytes),
                                                       byref(last)),
                    "pr_gpu_sweep_layout_info")
        return {"blocked": bool(on.value), "slices": sl.value, "bins": bn.value,
                "pairs": pairs.value, "ids": ids.value, "bytes": nbytes.value,
                "last_run_blocked": bool(last.value)}

    def verify(self, scores, damping: float = float(K_DAMP)) -> float:
        """The reference's PRVerifier error (src/pr_spmv.cc:78-94) of `scores`
        (n float32 in original ids) on the uploaded graph, computed on the
        device (pr_gpu_verify): bit-identical to the reference's when every
        in-row lists its sources in ascending order, as the builder's do."""
        s = np.ascontiguousarray(scores, dtype=np.float32)
        if s.ndim != 1 or s.shape[0] != self.n:
            raise ValueError("scores must hold one float per vertex")
        err = c_double()
        self._check(self._lib.pr_gpu_verify(self._h, _ptr(s), float(damping), byref(err)),
                    "pr_gpu_verify")
        return err.value

    def sweep_kernel_times(self, max_iters: int = 20, epsilon: float = 1e-4):
        """One plain solve with every sweep kernel timed on its own
        (pr_gpu_sweep_kernel_times): the average device ms per sweep of each
        kernel of the sweep body in launch order, and the sweep count."""
        ms = (c_double * 3)()
        nk, sw = c_int(), c_int32()
        self._check(self._lib.pr_gpu_sweep_kernel_times(self._h, int(max_iters), float(epsilon),
                                                        ms, 3, byref(nk), byref(sw)),
                    "pr_gpu_sweep_kernel_times")
        return [float(ms[k]) for k in range(nk.value)], int(sw.value)

    def set_stream(self, stream_handle: Optional[int]):
        """Issue work on a caller stream (raw cudaStream_t), None = own stream."""
        self._check(self._lib.pr_gpu_set_stream(self._h, stream_handle), "pr_gpu_set_stream")

    # -- introspection --------------------------------------------------------
    def last_timing(self):
        sweep_ms, total_ms, launches = c_double(), c_double(), c_int64()
        self._check(self._lib.pr_gpu_last_timing(self._h, byref(sweep_ms), byref(total_ms),
                                                 byref(launches)), "pr_gpu_last_timing")
        return sweep_ms.value, total_ms.value, launches.value

    def graph_info(self):
        n, m, md = c_int64(), c_int64(), c_int64()
        bins = (c_int64 * NUM_BINS)()
        self._check(self._lib.pr_gpu_graph_info(self._h, byref(n), byref(m), byref(md), bins,
                                                NUM_BINS), "pr_gpu_graph_info")
        return {"n": n.value, "m": m.value, "max_degree": md.value, "bin_rows": list(bins)}


# ---------------------------------------------------------------------------
# Reference-shaped entry points

def engine_for(g: Graph, device: int = 0) -> PageRankEngine:
    """The engine holding g (uploaded on first use, then cached on g)."""
    eng = getattr(g, "_pr_engine", None)
    if eng is None or eng.device != device:
        eng = PageRankEngine(device)
        eng.upload(g)
        g._pr_engine = eng
    return eng


def measure_gather_rate(array_bytes: int, device: int = 0) -> float:
    """Random 4-byte gathers per second that bypass L1, from an array of
    array_bytes (see pr_gpu_measure_gather_rate): the ceiling of the sweep
    kernels' gathers when the array fits in L2."""
    lib = pr_lib()
    out = c_double()
    rc = lib.pr_gpu_measure_gather_rate(int(device), int(array_bytes), byref(out))
    if rc != 0:
        raise PageRankError(rc, "pr_gpu_measure_gather_rate failed")
    return out.value


def measure_row_gather_rate(array_bytes: int, row_bytes: int, device: int = 0) -> float:
    """Bytes per second gathered as random rows of row_bytes with 16-byte
    loads (see pr_gpu_measure_row_gather_rate): the ceiling of a batched
    sweep's contrib-row gathers when the tile fits in L2."""
    lib = pr_lib()
    out = c_double()
    rc = lib.pr_gpu_measure_row_gather_rate(int(device), int(array_bytes), int(row_bytes),
                                            byref(out))
    if rc != 0:
        raise PageRankError(rc, "pr_gpu_measure_row_gather_rate failed")
    return out.value


def print_step(step: int, value: float) -> None:
    """The reference's -l line (src/util.h:37-46): '%5s%23.5lf'."""
    print(f"{step:>5d}{value:23.5f}")


def PageRankPull(g: Graph, max_iters: int, epsilon: float = 0.0,
                 logging_enabled: bool = False, device: int = 0) -> np.ndarray:
    """Drop-in for src/pr_spmv.cc:35-61 (returns float32 scores)."""
    res = engine_for(g, device).run(max_iters, epsilon, float(K_DAMP))
    if logging_enabled:
        for i in range(res.num_sweeps):
            print_step(i, float(res.err_trace[i, 0]))
    return res.scores


def PRVerifier(g: Graph, scores, target_error: float, device: int = 0) -> bool:
    """Drop-in for src/pr_spmv.cc:78-94: prints the reference's "Total Error"
    line (src/util.h PrintTime format) and returns error < target_error; the
    error is computed on the device (PageRankEngine.verify)."""
    error = engine_for(g, device).verify(scores, float(K_DAMP))
    print(f"{'Total Error:':<21}{error:3.5f}")
    return error < target_error


def PersonalizedPageRank(g: Graph, teleport, max_iters: int = 20, epsilon: float = 1e-4,
                         damping: float = float(K_DAMP), device: int = 0) -> PageRankResult:
    """Batched PPR: teleport (n,) or (n, k); columns retire independently."""
    return engine_for(g, device).run(max_iters, epsilon, damping, teleport=teleport)


def top_scores(scores: np.ndarray, k: int = 5):
    """(id, score) pairs of the k largest scores with the reference's order and
    tie rule (PrintTopScores / TopK, src/pr_spmv.cc:64-73,
    src/benchmark.h:72-88), computed by the native host library."""
    from ._native import graph_lib
    s = np.ascontiguousarray(scores, dtype=np.float32)
    ids = np.zeros(k, np.int32)
    vals = np.zeros(k, np.float32)
    cnt = graph_lib().gapbs_top_scores(s.ctypes.data, s.size, k, ids.ctypes.data, vals.ctypes.data)
    return [(int(ids[i]), float(vals[i])) for i in range(cnt)]


__all__ = ["PageRankEngine", "PageRankResult", "PageRankError", "PageRankPull",
           "PersonalizedPageRank", "engine_for", "top_scores", "K_DAMP"]
