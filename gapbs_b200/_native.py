"""Loading of the in-tree native libraries (ctypes).

``libgapbs_graph.so`` is the host graph builder, ``libgapbs_pr.so`` the
sm_100a PageRank engine.  Both are built in-tree (``make`` at the repository
root, or ``__graft_entry__.build()``).  A missing library is an error: there
is no Python fallback for either.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_void_p

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(_HERE, "lib")
BIN_DIR = os.path.join(_HERE, "bin")

_graph_lib = None
_pr_lib = None


class NativeLibraryMissing(RuntimeError):
    pass


def _load(name: str) -> ctypes.CDLL:
    path = os.path.join(LIB_DIR, name)
    if not os.path.exists(path):
        raise NativeLibraryMissing(
            f"{path} is not built; run `make` at the repository root "
            "(or __graft_entry__.build())")
    return ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)


def graph_lib() -> ctypes.CDLL:
    global _graph_lib
    if _graph_lib is None:
        lib = _load("libgapbs_graph.so")
        P = c_void_p
        lib.gapbs_graph_build.argtypes = [POINTER(P), c_char_p, c_int]
        lib.gapbs_graph_build.restype = c_int
        lib.gapbs_graph_from_edges.argtypes = [POINTER(P), P, P, c_int64, c_int]
        lib.gapbs_graph_from_edges.restype = c_int
        lib.gapbs_graph_new_undirected.argtypes = [POINTER(P), c_int64, c_int64,
                                                   POINTER(POINTER(c_int64)),
                                                   POINTER(POINTER(c_int32))]
        lib.gapbs_graph_new_undirected.restype = c_int
        lib.gapbs_rmat_permutation.argtypes = [c_int, P]
        lib.gapbs_rmat_permutation.restype = c_int
        lib.gapbs_graph_write_sg.argtypes = [P, c_char_p]
        lib.gapbs_graph_write_sg.restype = c_int
        lib.gapbs_graph_free.argtypes = [P]
        lib.gapbs_graph_free.restype = None
        for fn in ("num_nodes", "num_edges", "num_edges_directed"):
            f = getattr(lib, "gapbs_graph_" + fn)
            f.argtypes = [P]
            f.restype = c_int64
        lib.gapbs_graph_directed.argtypes = [P]
        lib.gapbs_graph_directed.restype = c_int
        for fn in ("out_offsets", "in_offsets"):
            f = getattr(lib, "gapbs_graph_" + fn)
            f.argtypes = [P]
            f.restype = POINTER(c_int64)
        for fn in ("out_neighbors", "in_neighbors"):
            f = getattr(lib, "gapbs_graph_" + fn)
            f.argtypes = [P]
            f.restype = POINTER(c_int32)
        lib.gapbs_graph_print_stats.argtypes = [P]
        lib.gapbs_graph_print_stats.restype = None
        lib.gapbs_top_scores.argtypes = [P, c_int64, c_int, P, P]
        lib.gapbs_top_scores.restype = c_int
        lib.gapbs_graph_last_error.argtypes = []
        lib.gapbs_graph_last_error.restype = c_char_p
        _graph_lib = lib
    return _graph_lib


def pr_lib() -> ctypes.CDLL:
    global _pr_lib
    if _pr_lib is None:
        lib = _load("libgapbs_pr.so")
        from . import _pr_abi
        _pr_abi.declare(lib)
        _pr_lib = lib
    return _pr_lib


__all__ = ["graph_lib", "pr_lib", "NativeLibraryMissing", "LIB_DIR", "BIN_DIR",
           "c_double", "c_float", "c_int"]
