"""The pr_gpu / cc_gpu / bfs_gpu command lines against the reference's
pr_spmv / cc / bfs (no GPU needed).

Help text, and every invocation that the reference rejects before running a
kernel, must give the reference's exit code and stdout byte for byte
(recorded from the reference binary in tests/golden/cli_golden.json).
"""
import json
import os
import subprocess

import pytest

from conftest import GOLDEN, ROOT

BIN = os.path.join(ROOT, "gapbs_b200", "bin")
OURS = {"pr_spmv": "pr_gpu", "cc": "cc_gpu", "bfs": "bfs_gpu"}  # reference binary -> drop-in
with open(os.path.join(GOLDEN, "cli_golden.json")) as fh:
    CASES = json.load(fh)["cases"]


@pytest.fixture(scope="module")
def bins():
    if not all(os.path.exists(os.path.join(BIN, b)) for b in OURS.values()):
        subprocess.run(["make", "-C", ROOT, "cli"], check=True)
    return BIN


@pytest.mark.parametrize("case", CASES, ids=[f"{c['binary']} {c['args']}" for c in CASES])
def test_cli_matches_reference(bins, case, tmp_path):
    (tmp_path / "x.foo").write_text("")
    exe = os.path.join(bins, OURS[case["binary"]])
    args = case["args"].format(tmp=str(tmp_path)).split()
    p = subprocess.run([exe] + args, capture_output=True, text=True, timeout=60)
    assert p.returncode == case["returncode"]
    assert p.stdout.replace(str(tmp_path), "{tmp}") == case["stdout"]
