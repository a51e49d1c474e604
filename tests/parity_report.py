"""Per-graph accuracy report of the GPU PageRankPull against the FP64 oracle.

For each graph: sweeps (GPU / reference FP32 restatement), L1 and max-abs
error of the GPU scores against the FP64 oracle, the same for the
reference's FP32 scores (the oracle's bit-exact restatement of
src/pr_spmv.cc:35-61), and the PRVerifier total error of the GPU scores,
once per sweep layout (slice-blocked and gather, each forced).
Prints a markdown table.  Needs a GPU; run as `python tests/parity_report.py`.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from gapbs_b200 import PageRankEngine  # noqa: E402
from gapbs_b200.graph import make_graph  # noqa: E402

GRAPHS = ["-g 10", "-u 10", "-g 12", "-u 12", "-g 16", "-u 16", "-g 18", "-u 18", "-g 20",
          "-u 20", "-g 22"]


def main():
    eng = PageRankEngine(0)
    print("| graph | N | M | sweeps GPU / ref | L1(GPU-fp64) | max abs(GPU-fp64) "
          "| L1(ref fp32-fp64) | max abs(ref-fp64) | PRVerifier error (GPU) | sweep |")
    print("|---|---:|---:|---|---:|---:|---:|---:|---:|---|")
    for args, layout in [(a, l) for a in GRAPHS for l in ("blocked", "gather")]:
        g = make_graph(args)
        eng.set_sweep_layout(layout)
        eng.upload(g)
        res = eng.run(20, 1e-4)
        s = res.scores.astype(np.float64)
        s64, _, _ = oracle.pr_pull_f64(g, 20, 1e-4)
        s32, k32, _ = oracle.pr_pull_f32(g, 20, 1e-4)
        r = s32.astype(np.float64)
        ver = oracle.pr_verify_f32(g, res.scores)
        print(f"| `{args}` | {g.num_nodes} | {g.num_edges_directed} | {int(res.sweeps[0])} / {k32} "
              f"| {np.abs(s - s64).sum():.3e} | {np.abs(s - s64).max():.3e} "
              f"| {np.abs(r - s64).sum():.3e} | {np.abs(r - s64).max():.3e} | {ver:.3e} "
              f"| {'slice-blocked' if eng.sweep_layout_info()['last_run_blocked'] else 'gather'} |",
              flush=True)
    eng.close()


if __name__ == "__main__":
    main()
