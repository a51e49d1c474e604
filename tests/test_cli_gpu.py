"""pr_gpu and cc_gpu end to end on the GPU, the way the reference's
test/test.mk runs pr_spmv and cc: the verification line, the -l step lines,
the -a top scores of PageRank and the -a cluster lines of CC.
"""
import json
import os
import re
import subprocess

import pytest

from conftest import GOLDEN, ROOT, gpu_available

pytestmark = pytest.mark.gpu
EXE = os.path.join(ROOT, "gapbs_b200", "bin", "pr_gpu")
CC_EXE = os.path.join(ROOT, "gapbs_b200", "bin", "cc_gpu")
BFS_EXE = os.path.join(ROOT, "gapbs_b200", "bin", "bfs_gpu")
with open(os.path.join(GOLDEN, "cli_golden.json")) as fh:
    _CLI = json.load(fh)
CC_ANALYSIS = _CLI["cc_analysis"]
BFS_ANALYSIS = _CLI["bfs_analysis"]
with open(os.path.join(GOLDEN, "pr_golden.json")) as fh:
    GOLD = json.load(fh)["cases"]
STEP = re.compile(r"^ {4}\d+ +\d+\.\d{5}$")
TOP = re.compile(r"^(\d+):(\S+)$")


@pytest.fixture(scope="module")
def exe():
    if not gpu_available():
        pytest.skip("no CUDA device")
    if not os.path.exists(EXE):
        subprocess.run(["make", "-C", ROOT, "cli"], check=True)
    return EXE


def run(exe, args):
    p = subprocess.run([exe] + args, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    return p.stdout


@pytest.mark.parametrize("args,trials", [("-g 10 -n 1 -v", 1), ("-u 10 -n 2 -v", 2),
                                          ("-g 12 -n 1 -v -i 30 -t 1e-6", 1)])
def test_verification_passes(exe, args, trials):
    out = run(exe, args.split())
    assert out.count("Verification:           PASS") == trials
    assert "FAIL" not in out
    assert "Generate Time:" in out and "Build Time:" in out and "Average Time:" in out


def test_log_lines_and_top_scores(exe):
    e = GOLD["el4"]
    out = run(exe, ["-f", os.path.join(GOLDEN, "graphs", "4.el"), "-n", "1", "-v", "-a", "-l"])
    lines = out.splitlines()
    assert [ln for ln in lines if STEP.match(ln)] == e["log_lines"]
    assert "Verification:           PASS" in out
    assert "Upload Time:" in out
    top = [TOP.match(ln) for ln in lines if TOP.match(ln)]
    assert [int(t.group(1)) for t in top] == [v for v, _ in e["top5"]]
    for t, (_, sc) in zip(top, e["top5"]):
        assert abs(float(t.group(2)) - sc) <= 1e-5 * sc


@pytest.mark.parametrize("case", CC_ANALYSIS, ids=[c["args"] for c in CC_ANALYSIS])
def test_cc_analysis_and_verification(exe, case):
    args = case["args"].format(graphs=os.path.join(GOLDEN, "graphs")).split() + ["-v"]
    out = run(CC_EXE, args)
    lines = out.splitlines()
    i = next(k for k, ln in enumerate(lines) if ln.endswith("biggest clusters"))
    j = next(k for k, ln in enumerate(lines) if ln.startswith("There are "))
    assert lines[i - 1:j + 1] == case["lines"]
    assert "Verification:           PASS" in out


def test_cc_verification_on_larger_graphs(exe):
    for args in ("-g 16 -n 2 -v", "-u 16 -k 2 -n 1 -v"):
        out = run(CC_EXE, args.split())
        assert out.count("Verification:           PASS") == int(args.split()[args.split().index("-n") + 1])


@pytest.mark.parametrize("case", BFS_ANALYSIS, ids=[c["args"] for c in BFS_ANALYSIS])
def test_bfs_analysis_and_verification(exe, case):
    args = case["args"].format(graphs=os.path.join(GOLDEN, "graphs")).split() + ["-v"]
    out = run(BFS_EXE, args)
    assert case["line"] in out.splitlines()
    trials = int(args[args.index("-n") + 1])
    assert out.count("Verification:           PASS") == trials


def test_bfs_logging_lines(exe):
    out = run(BFS_EXE, ["-g", "14", "-n", "1", "-l"])
    lines = out.splitlines()
    assert any(ln.startswith("Source:") for ln in lines)
    kinds = [ln.split()[0] for ln in lines if ln.split() and ln.split()[0] in ("i", "td", "e", "bu", "c")]
    assert kinds and kinds[0] == "i"
