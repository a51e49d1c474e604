"""The drop-in boundary exercised from the reference's own code.

oracle/_ref/pr_spmv_b200 is the reference's src/pr_spmv.cc compiled from its
sources with PageRankPull replaced by the binding INTEGRATION.md section 1
gives (oracle/b200_pagerank_pull.inc: pr_gpu_create, pr_gpu_upload of the
reference's CSRGraph arrays, pr_gpu_run), and linked against
gapbs_b200/lib/libgapbs_pr.so.  Its main, Builder, BenchmarkKernel,
PrintTopScores and PRVerifier are the reference's.  Checked the way the
reference's test/test.mk:73-86 checks pr_spmv (-g10 -vn1 greps
"Verification:           PASS"), plus:
  * the -l lines against the reference binary's own (oracle/_ref/pr_spmv) on
    the same graph: same step numbers, values equal to the printed precision
    or one unit of its last digit;
  * the -a top scores on the reference's 4.el fixture against the reference
    binary's, and verification on a directed and a weighted-file graph.
"""
import os
import subprocess

import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
EXE = os.path.join(REF_DIR, "pr_spmv_b200")
REF_EXE = os.path.join(REF_DIR, "pr_spmv")
GRAPHS = os.path.join(ROOT, "tests", "golden", "graphs")


@pytest.fixture(scope="module")
def exe():
    if not gpu_available():
        pytest.skip("no CUDA device")
    if not (os.path.exists(EXE) and os.path.exists(REF_EXE)):
        pytest.skip("oracle/_ref/pr_spmv_b200 not built (make -C oracle REF=<reference tree>)")
    return EXE


def run(path, *args):
    p = subprocess.run([path, *args], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, (args, p.stdout[-2000:], p.stderr[-2000:])
    return p.stdout


def step_lines(out):
    return [ln for ln in out.splitlines()
            if ln.strip() and ln[:5].strip().isdigit() and len(ln.split()) == 2]


@pytest.mark.parametrize("args", [["-g", "10", "-vn1"], ["-u", "10", "-vn1"],
                                  ["-g", "14", "-vn3"], ["-g", "12", "-s", "-vn1"]])
def test_reference_main_verifies(exe, args):
    out = run(exe, *args)
    assert "Verification:           PASS" in out
    assert out.count("Trial Time:") == int(args[-1][-1])


@pytest.mark.parametrize("args", [["-g", "10"], ["-g", "16"], ["-u", "12"]])
def test_log_lines_equal_reference(exe, args):
    ours = step_lines(run(exe, *args, "-n", "1", "-l"))
    ref = step_lines(run(REF_EXE, *args, "-n", "1", "-l"))
    assert len(ours) == len(ref) > 0
    for got, want in zip(ours, ref):
        assert got.split()[0] == want.split()[0]
        assert abs(float(got.split()[1]) - float(want.split()[1])) <= 1.01e-5, (got, want)


def test_top_scores_and_file_graphs(exe):
    el = os.path.join(GRAPHS, "4.el")
    ours = run(exe, "-f", el, "-n", "1", "-v", "-a")
    ref = run(REF_EXE, "-f", el, "-n", "1", "-v", "-a")
    assert "Verification:           PASS" in ours

    def top(out):
        rows = [ln.split(":") for ln in out.splitlines()
                if ":" in ln and ln.split(":")[0].strip().isdigit()]
        return [(int(a), float(b)) for a, b in rows]
    t_ours, t_ref = top(ours), top(ref)
    assert len(t_ours) == len(t_ref) > 0
    for (vo, so), (vr, sr) in zip(t_ours, t_ref):
        assert vo == vr and abs(so - sr) <= 2e-5 * sr + 1e-7
    for f in ("4.gr", "4.mtx", "4.wel"):
        out = run(exe, "-f", os.path.join(GRAPHS, f), "-n", "1", "-v")
        assert "Verification:           PASS" in out, f
