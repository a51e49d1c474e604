"""The pr_gpu command line against the reference pr_spmv (no GPU needed).

Help text, and every invocation that the reference rejects before running a
kernel, must give the reference's exit code and stdout byte for byte
(recorded from the reference binary in tests/golden/cli_golden.json).
"""
import json
import os
import subprocess

import pytest

from conftest import GOLDEN, ROOT

EXE = os.path.join(ROOT, "gapbs_b200", "bin", "pr_gpu")
with open(os.path.join(GOLDEN, "cli_golden.json")) as fh:
    CASES = json.load(fh)["cases"]


@pytest.fixture(scope="module")
def exe():
    if not os.path.exists(EXE):
        subprocess.run(["make", "-C", ROOT, "cli"], check=True)
    return EXE


@pytest.mark.parametrize("case", CASES, ids=[c["args"] for c in CASES])
def test_cli_matches_reference(exe, case, tmp_path):
    (tmp_path / "x.foo").write_text("")
    args = case["args"].format(tmp=str(tmp_path)).split()
    p = subprocess.run([exe] + args, capture_output=True, text=True, timeout=60)
    assert p.returncode == case["returncode"]
    assert p.stdout.replace(str(tmp_path), "{tmp}") == case["stdout"]
