"""The C-ABI libraries load and export every symbol include/*.h declares.

No compute calls: these run on machines without a GPU.
"""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADERS = {
    "gapbs_graph.h": os.path.join(ROOT, "gapbs_b200", "lib", "libgapbs_graph.so"),
    "pr_gpu.h": os.path.join(ROOT, "gapbs_b200", "lib", "libgapbs_pr.so"),
}


def declared_functions(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", text)
    return sorted({n for n in names if n.startswith(("pr_gpu_", "gapbs_"))})


@pytest.mark.parametrize("header", sorted(HEADERS))
def test_library_exports_declared_symbols(header):
    lib_path = HEADERS[header]
    if not os.path.exists(lib_path):
        pytest.fail(f"{lib_path} not built (run make)")
    lib = ctypes.CDLL(lib_path)
    names = declared_functions(header)
    assert names, header
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_declares_every_pr_symbol():
    from gapbs_b200 import _pr_abi
    assert sorted(_pr_abi.SYMBOLS) == declared_functions("pr_gpu.h")


def test_last_error_on_null_handle():
    lib = ctypes.CDLL(HEADERS["pr_gpu.h"])
    lib.pr_gpu_last_error.restype = ctypes.c_char_p
    lib.pr_gpu_last_error.argtypes = [ctypes.c_void_p]
    assert lib.pr_gpu_last_error(None) == b"invalid handle"


def test_engine_library_is_sm100a():
    """The engine is compiled for sm_100a only (no other targets)."""
    mk = open(os.path.join(ROOT, "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk


def test_gather_probes_reject_bad_arguments():
    """The roofline probes check their arguments before touching a device."""
    lib = ctypes.CDLL(HEADERS["pr_gpu.h"])
    out = ctypes.c_double()
    lib.pr_gpu_measure_gather_rate.argtypes = [ctypes.c_int, ctypes.c_int64,
                                               ctypes.POINTER(ctypes.c_double)]
    lib.pr_gpu_measure_row_gather_rate.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int,
                                                   ctypes.POINTER(ctypes.c_double)]
    assert lib.pr_gpu_measure_gather_rate(0, 1024, ctypes.byref(out)) == -1
    assert lib.pr_gpu_measure_gather_rate(0, 1 << 20, None) == -1
    for row_bytes in (0, 8, 24, 1024):
        assert lib.pr_gpu_measure_row_gather_rate(0, 1 << 20, row_bytes, ctypes.byref(out)) == -1
    assert lib.pr_gpu_measure_row_gather_rate(0, 1 << 20, 256, None) == -1
