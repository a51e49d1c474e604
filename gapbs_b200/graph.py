"""Host CSR graphs, built by the native builder (``libgapbs_graph.so``).

``Graph`` mirrors the parts of the reference's ``CSRGraph<int32_t>``
(src/graph.h:98-273) that PageRank touches: node and edge counts with the
reference's conventions, out/in degrees and neighbour ranges.  ``Builder``
mirrors ``BuilderBase::MakeGraph`` (src/builder.h:343-364) over the same
command-line options; the graph it returns is identical to the reference's.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from ._native import graph_lib


class GraphBuildError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (code {code})")
        self.code = code


class Graph:
    """CSR graph; owns the native handle, exposes zero-copy numpy views."""

    def __init__(self, handle: ctypes.c_void_p):
        self._h = handle
        lib = graph_lib()
        self._lib = lib
        self.num_nodes = int(lib.gapbs_graph_num_nodes(handle))
        self.num_edges = int(lib.gapbs_graph_num_edges(handle))
        self.num_edges_directed = int(lib.gapbs_graph_num_edges_directed(handle))
        self.directed = bool(lib.gapbs_graph_directed(handle))
        n = self.num_nodes
        out_entries = int(lib.gapbs_graph_out_offsets(handle)[n]) if n else 0
        in_entries = int(lib.gapbs_graph_in_offsets(handle)[n]) if n else 0
        self.out_offsets = np.ctypeslib.as_array(lib.gapbs_graph_out_offsets(handle), shape=(n + 1,))
        self.in_offsets = np.ctypeslib.as_array(lib.gapbs_graph_in_offsets(handle), shape=(n + 1,))
        self.out_neighbors = (np.ctypeslib.as_array(lib.gapbs_graph_out_neighbors(handle), shape=(out_entries,))
                              if out_entries else np.zeros(0, np.int32))
        self.in_neighbors = (np.ctypeslib.as_array(lib.gapbs_graph_in_neighbors(handle), shape=(in_entries,))
                             if in_entries else np.zeros(0, np.int32))
        for a in (self.out_offsets, self.in_offsets, self.out_neighbors, self.in_neighbors):
            a.flags.writeable = False

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.gapbs_graph_free(h)
            self._h = None

    # --- CSRGraph-style accessors -------------------------------------------------
    def out_degree(self, v=None):
        d = np.diff(self.out_offsets)
        return d if v is None else int(d[v])

    def in_degree(self, v=None):
        d = np.diff(self.in_offsets)
        return d if v is None else int(d[v])

    def out_neigh(self, v: int) -> np.ndarray:
        return self.out_neighbors[self.out_offsets[v]:self.out_offsets[v + 1]]

    def in_neigh(self, v: int) -> np.ndarray:
        return self.in_neighbors[self.in_offsets[v]:self.in_offsets[v + 1]]

    def stats_line(self) -> str:
        """The reference's PrintStats line (src/graph.h:223-230)."""
        kind = "directed" if self.directed else "undirected"
        deg = self.num_edges // self.num_nodes if self.num_nodes else 0
        return (f"Graph has {self.num_nodes} nodes and {self.num_edges} {kind} "
                f"edges for degree: {deg}")

    def write_sg(self, path: str) -> None:
        rc = self._lib.gapbs_graph_write_sg(self._h, path.encode())
        if rc != 0:
            raise GraphBuildError(rc, self._lib.gapbs_graph_last_error().decode())

    @staticmethod
    def from_edges(u, v, symmetrize: bool = False) -> "Graph":
        u = np.ascontiguousarray(u, dtype=np.int32)
        v = np.ascontiguousarray(v, dtype=np.int32)
        if u.shape != v.shape:
            raise ValueError("u and v must have the same length")
        lib = graph_lib()
        h = ctypes.c_void_p()
        rc = lib.gapbs_graph_from_edges(ctypes.byref(h), u.ctypes.data, v.ctypes.data,
                                        int(u.size), int(symmetrize))
        if rc != 0:
            raise GraphBuildError(rc, lib.gapbs_graph_last_error().decode())
        return Graph(h)


class Builder:
    """``Builder(args).MakeGraph()`` with pr_spmv options, e.g. ``"-g 16"``."""

    def __init__(self, args: str, verbose: bool = False):
        self.args = args
        self.verbose = verbose

    def MakeGraph(self) -> Graph:
        lib = graph_lib()
        h = ctypes.c_void_p()
        rc = lib.gapbs_graph_build(ctypes.byref(h), self.args.encode(), int(self.verbose))
        if rc != 0:
            raise GraphBuildError(rc, lib.gapbs_graph_last_error().decode())
        return Graph(h)


def make_graph(args: str, verbose: bool = False) -> Graph:
    return Builder(args, verbose).MakeGraph()


def generate(scale: int, degree: int = 16, uniform: bool = False) -> Graph:
    return make_graph(f"-{'u' if uniform else 'g'} {scale} -k {degree}")


__all__ = ["Graph", "Builder", "make_graph", "generate", "GraphBuildError"]
