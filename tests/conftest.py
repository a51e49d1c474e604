"""Shared pytest configuration.

Markers: ``gpu`` -- needs a CUDA device (the parity tests proper, run on a
B200); everything else runs on CPU.  The native libraries are built in-tree
by ``make`` if they are missing.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "fullsize: full benchmark-size graphs (slow)")


def _ensure_built():
    libs = [os.path.join(ROOT, "gapbs_b200", "lib", "libgapbs_graph.so"),
            os.path.join(ROOT, "oracle", "liboracle.so")]
    if not all(os.path.exists(p) for p in libs):
        subprocess.run(["make", "-C", ROOT, "graph"], check=True)
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)


_ensure_built()


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "pr_golden.json")) as fh:
        return json.load(fh)


@pytest.fixture(scope="session")
def adversarial():
    return dict(np.load(os.path.join(GOLDEN, "adversarial.npz")))


def golden_args(entry) -> str:
    return entry["args"].format(graphs=os.path.join(GOLDEN, "graphs"))


def fmt_step(i: int, v: float) -> str:
    """The reference's -l line format (src/util.h:37-46)."""
    return f"{i:>5d}{v:23.5f}"
