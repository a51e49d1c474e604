"""Regenerates the golden fixtures in this directory from the REFERENCE.

Runs only where the reference tree and oracle/_ref (the reference compiled
from its own sources by oracle/Makefile) exist.  Writes:

  graphs/4*.{el,wel,gr,graph,mtx}   the reference's tiny loader fixtures
                                     (test/graphs/), copied as test inputs
  pr_golden.json                     per case: graph identity (N, edge counts,
                                     sha256 of the CSR arrays), the reference
                                     PageRankPull's sweep count, its -l lines,
                                     sha256 of its float32 scores, top-5, and
                                     PRVerifier's total error
  scores_<case>.npy                  the reference's float32 scores (small
                                     graphs only)
  adversarial.npz                    small hand-made edge lists (isolated
                                     vertices, star hub, chain, directed sinks)
                                     with the reference's scores on each
  pr_fullsize.json                   (--fullsize) the benchmark-size graphs
                                     (-u 24 -k 16, -g 25 -k 16, and the graphs
                                     of the PPR and adjoint workloads): graph
                                     identity, the reference's sweep count and
                                     -l lines, top-5, PRVerifier line, and its
                                     float32 scores at 4096 fixed sample
                                     vertices

  cli_golden.json                    (--cli) the reference pr_spmv's exit code
                                     and stdout for -h and for rejected
                                     invocations (missing file, unknown
                                     suffix, missing or unknown option)

  cc_golden.json                     (--cc) the reference's Afforest connected
                                     components on small and mid-size graphs:
                                     component count, sha256 of the int32
                                     labels, the labels themselves for the
                                     smallest graphs

  bfs_golden.json                    (--bfs) the reference's SourcePicker
                                     sources and, per source, what its DOBFS
                                     tree gives: reached count, PrintBFSStats
                                     edge count, sha256 of the depths along
                                     its parent pointers (the depths themselves
                                     for the smallest graphs)

Usage:  GAPBS_REFERENCE_TREE=<reference source tree> \
            python tests/golden/make_golden.py [--fullsize | --cli | --cc | --bfs]
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
# the reference's source tree (its test/graphs and test/reference fixtures)
REF_TREE = os.environ.get("GAPBS_REFERENCE_TREE", "")
sys.path.insert(0, ROOT)

import oracle  # noqa: E402


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def capture_stdout(fn, *args, **kw):
    """Run fn with the process's fd 1 redirected to a temp file; return (ret, text)."""
    sys.stdout.flush()
    saved = os.dup(1)
    with tempfile.TemporaryFile(mode="w+b") as tmp:
        os.dup2(tmp.fileno(), 1)
        try:
            ret = fn(*args, **kw)
        finally:
            sys.stdout.flush()
            os.dup2(saved, 1)
            os.close(saved)
        tmp.seek(0)
        text = tmp.read().decode()
    return ret, text


GRAPH_FILES = ["4.el", "4.wel", "4.gr", "4.graph", "4.mtx", "4w.graph", "4w.mtx"]

# (case name, pr_spmv arguments, keep full score vector)
CASES = [
    ("g10", "-g 10", True),
    ("u10", "-u 10", True),
    ("g12", "-g 12", True),
    ("u12", "-u 12", False),
    ("g10k4", "-g 10 -k 4", True),
    ("g16", "-g 16", False),
    ("u16", "-u 16", False),
    ("g18", "-g 18", False),
    ("el4", "-f {graphs}/4.el", True),
    ("el4s", "-f {graphs}/4.el -s", True),
    ("wel4", "-f {graphs}/4.wel", False),
    ("gr4", "-f {graphs}/4.gr", False),
    ("graph4", "-f {graphs}/4.graph", False),
    ("mtx4", "-f {graphs}/4.mtx", False),
    ("graph4w", "-f {graphs}/4w.graph", False),
    ("mtx4w", "-f {graphs}/4w.mtx", False),
]


def adversarial_edge_lists():
    """Small graphs that exercise the corner cases of the sweep."""
    cases = {}
    # isolated vertices interleaved with a triangle and a pendant: ids 0..9
    cases["isolated"] = (np.array([1, 2, 3, 3, 9], np.int32), np.array([2, 3, 1, 7, 3], np.int32), True)
    # star: hub 0 with 300 leaves (hub degree above a warp and a block)
    leaves = np.arange(1, 301, dtype=np.int32)
    cases["star"] = (np.zeros_like(leaves), leaves, True)
    # chain of 50
    a = np.arange(0, 49, dtype=np.int32)
    cases["chain"] = (a, a + 1, True)
    # directed with sinks (vertices with no out-edges) and sources
    u = np.array([0, 0, 1, 2, 2, 3, 5, 5, 6, 7], np.int32)
    v = np.array([1, 2, 3, 3, 4, 4, 4, 6, 4, 0], np.int32)
    cases["directed_sinks"] = (u, v, False)
    # self loops and duplicates only (squish removes them)
    cases["selfdup"] = (np.array([0, 0, 1, 1, 2, 2, 2], np.int32), np.array([0, 1, 0, 1, 2, 0, 0], np.int32), True)
    # one big hub (degree 5000) plus a random sparse remainder
    rng = np.random.default_rng(7)
    hu = np.zeros(5000, np.int32)
    hv = rng.integers(1, 6000, 5000).astype(np.int32)
    ru = rng.integers(1, 6000, 20000).astype(np.int32)
    rv = rng.integers(1, 6000, 20000).astype(np.int32)
    cases["hub5000"] = (np.concatenate([hu, ru]), np.concatenate([hv, rv]), True)
    return cases


def main():
    if not REF_TREE or not os.path.isdir(REF_TREE) or not oracle.ref_available():
        sys.exit("needs GAPBS_REFERENCE_TREE (the reference source tree) and oracle/_ref "
                 "(make -C oracle REF=<tree>)")
    gdir = os.path.join(HERE, "graphs")
    os.makedirs(gdir, exist_ok=True)
    for f in GRAPH_FILES:
        shutil.copyfile(os.path.join(REF_TREE, "test", "graphs", f), os.path.join(gdir, f))
    expected = {}
    for f in os.listdir(os.path.join(REF_TREE, "test", "reference")):
        with open(os.path.join(REF_TREE, "test", "reference", f)) as fh:
            expected[f] = fh.read().strip()

    out = {"generator": "tests/golden/make_golden.py", "reference_outputs": expected, "cases": {}}
    for name, args, keep in CASES:
        a = args.format(graphs=gdir)
        g, _ = capture_stdout(oracle.RefGraph.build, a)
        oo, onb, io, inb = g.csr()
        scores, log = capture_stdout(g.pagerank_pull, 20, 1e-4, True)
        step_lines = [ln for ln in log.splitlines() if ln.strip()]
        ok, vlog = capture_stdout(g.verify, scores, 1e-4)
        order = np.lexsort((np.arange(scores.size), -scores.astype(np.float64)))[:5]
        entry = {
            "args": args,
            "num_nodes": g.num_nodes,
            "num_edges": g.num_edges,
            "num_edges_directed": g.num_edges_directed,
            "directed": g.directed,
            "csr_sha256": sha(oo, onb, io, inb),
            "sweeps": len(step_lines),
            "log_lines": step_lines,
            "scores_sha256": sha(scores),
            "scores_sum": float(scores.astype(np.float64).sum()),
            "top5": [[int(i), float(scores[i])] for i in order],
            "verify_pass": ok,
            "verify_line": vlog.strip(),
        }
        if keep:
            np.save(os.path.join(HERE, f"scores_{name}.npy"), scores)
        out["cases"][name] = entry
        print(name, g.num_nodes, g.num_edges, entry["sweeps"], ok)

    adv = {}
    for name, (u, v, sym) in adversarial_edge_lists().items():
        from gapbs_b200.graph import Graph
        hg = Graph.from_edges(u, v, symmetrize=sym)
        rg = oracle.RefGraph.from_csr(hg)
        scores, log = capture_stdout(rg.pagerank_pull, 20, 1e-4, True)
        adv[f"{name}_u"] = u
        adv[f"{name}_v"] = v
        adv[f"{name}_sym"] = np.array(sym)
        adv[f"{name}_scores"] = scores
        adv[f"{name}_sweeps"] = np.array(len([ln for ln in log.splitlines() if ln.strip()]))
        print("adversarial", name, hg.num_nodes, hg.num_edges_directed)
    np.savez_compressed(os.path.join(HERE, "adversarial.npz"), **adv)
    with open(os.path.join(HERE, "pr_golden.json"), "w") as fh:
        json.dump(out, fh, indent=1)


# (case name, pr_spmv arguments, run PageRankPull)
FULLSIZE_CASES = [
    ("u24", "-u 24 -k 16", True),
    ("g25", "-g 25 -k 16", True),
    ("g22", "-g 22", True),
    ("g20", "-g 20", False),
]
SAMPLE_SEED = 27491095 + 2
SAMPLE_COUNT = 4096


def sample_vertices(n: int) -> np.ndarray:
    """Fixed sample: the 64 lowest ids, then uniform ids, sorted, unique."""
    rng = np.random.default_rng(SAMPLE_SEED)
    ids = np.concatenate([np.arange(min(64, n)), rng.integers(0, n, SAMPLE_COUNT)])
    return np.unique(ids)[:SAMPLE_COUNT]


def main_fullsize():
    if not oracle.ref_available():
        sys.exit("needs oracle/_ref (make -C oracle where the reference tree exists)")
    out = {"generator": "tests/golden/make_golden.py --fullsize", "sample_seed": SAMPLE_SEED,
           "cases": {}}
    for name, args, run in FULLSIZE_CASES:
        g, _ = capture_stdout(oracle.RefGraph.build, args)
        oo, onb, io, inb = g.csr()
        entry = {
            "args": args,
            "num_nodes": g.num_nodes,
            "num_edges": g.num_edges,
            "num_edges_directed": g.num_edges_directed,
            "directed": g.directed,
            "csr_sha256": sha(oo, onb, io, inb),
        }
        del oo, onb, io, inb
        if run:
            scores, log = capture_stdout(g.pagerank_pull, 20, 1e-4, True)
            step_lines = [ln for ln in log.splitlines() if ln.strip()]
            ok, vlog = capture_stdout(g.verify, scores, 1e-4)
            order = np.lexsort((np.arange(scores.size), -scores.astype(np.float64)))[:5]
            ids = sample_vertices(g.num_nodes)
            entry.update({
                "sweeps": len(step_lines),
                "log_lines": step_lines,
                "scores_sum": float(scores.astype(np.float64).sum()),
                "top5": [[int(i), float(scores[i])] for i in order],
                "verify_pass": ok,
                "verify_line": vlog.strip(),
                "sample_ids": [int(i) for i in ids],
                "sample_scores": [float(scores[i]) for i in ids],
            })
        out["cases"][name] = entry
        print(name, g.num_nodes, g.num_edges_directed, entry.get("sweeps"), flush=True)
        del g
    with open(os.path.join(HERE, "pr_fullsize.json"), "w") as fh:
        json.dump(out, fh, indent=1)


# pr_spmv invocations that end before any kernel runs; {tmp} is a scratch
# directory holding an empty file x.foo
CLI_CASES = ["-h", "-f {tmp}/missing.el", "-f {tmp}/x.foo", "-g", "-z", "-n"]


# cc -a runs whose analysis lines (clusters, component count) are recorded
CC_ANALYSIS_CASES = ["-g 10 -n 1 -a", "-u 12 -k 1 -n 1 -a", "-f {graphs}/4.el -n 1 -a"]
# bfs -a runs whose "BFS Tree has ..." line (last trial's source) is recorded
BFS_ANALYSIS_CASES = ["-g 10 -n 3 -a", "-u 12 -k 1 -n 2 -a", "-f {graphs}/4.el -n 3 -a",
                      "-g 12 -r 5 -n 1 -a", "-f {graphs}/4.el -s -n 2 -a"]


def main_cli():
    import subprocess
    out = {"generator": "tests/golden/make_golden.py --cli", "cases": [], "cc_analysis": []}
    with tempfile.TemporaryDirectory() as tmp:
        open(os.path.join(tmp, "x.foo"), "w").close()
        for binary in ("pr_spmv", "cc", "bfs"):
            exe = os.path.join(ROOT, "oracle", "_ref", binary)
            if not os.path.exists(exe):
                sys.exit(f"needs oracle/_ref/{binary} (make -C oracle where the reference tree exists)")
            for args in CLI_CASES:
                p = subprocess.run([exe] + args.format(tmp=tmp).split(), capture_output=True,
                                   text=True)
                out["cases"].append({"binary": binary, "args": args, "returncode": p.returncode,
                                     "stdout": p.stdout.replace(tmp, "{tmp}")})
                print(binary, args, p.returncode)
    gdir = os.path.join(HERE, "graphs")
    exe = os.path.join(ROOT, "oracle", "_ref", "cc")
    for args in CC_ANALYSIS_CASES:
        p = subprocess.run([exe] + args.format(graphs=gdir).split(), capture_output=True, text=True)
        lines = p.stdout.splitlines()
        i = next(k for k, ln in enumerate(lines) if ln.endswith("biggest clusters"))
        j = next(k for k, ln in enumerate(lines) if ln.startswith("There are "))
        out["cc_analysis"].append({"args": args, "lines": lines[i - 1:j + 1]})
        print("cc", args, lines[j])
    out["bfs_analysis"] = []
    exe = os.path.join(ROOT, "oracle", "_ref", "bfs")
    for args in BFS_ANALYSIS_CASES:
        p = subprocess.run([exe] + args.format(graphs=gdir).split(), capture_output=True, text=True)
        line = next(ln for ln in p.stdout.splitlines() if ln.startswith("BFS Tree has "))
        out["bfs_analysis"].append({"args": args, "line": line})
        print("bfs", args, line)
    with open(os.path.join(HERE, "cli_golden.json"), "w") as fh:
        json.dump(out, fh, indent=1)


# (case name, options, keep the label array)
CC_CASES = [
    ("g10", "-g 10", True), ("u10", "-u 10", True), ("g12k2", "-g 12 -k 2", True),
    ("u12k1", "-u 12 -k 1", True), ("g14k2", "-g 14 -k 2", False), ("g16", "-g 16", False),
    ("g18k4", "-g 18 -k 4", False), ("u18k1", "-u 18 -k 1", False),
    ("el4", "-f {graphs}/4.el", True), ("el4s", "-f {graphs}/4.el -s", True),
    ("mtx4", "-f {graphs}/4.mtx", True), ("gr4", "-f {graphs}/4.gr", True),
]


def main_cc():
    gdir = os.path.join(HERE, "graphs")
    out = {"generator": "tests/golden/make_golden.py --cc", "cases": {}}
    for name, args, keep in CC_CASES:
        a = args.format(graphs=gdir)
        (comp, _), _ = capture_stdout(oracle.ref_cc_afforest, a)
        entry = {"args": args, "num_nodes": int(comp.size),
                 "components": int(np.unique(comp).size), "labels_sha256": sha(comp)}
        if keep:
            entry["labels"] = [int(x) for x in comp]
        out["cases"][name] = entry
        print(name, comp.size, entry["components"])
    with open(os.path.join(HERE, "cc_golden.json"), "w") as fh:
        json.dump(out, fh, separators=(",", ":"))


BFS_CASES = [
    ("g10", "-g 10", True), ("u10", "-u 10", True), ("g12k4", "-g 12 -k 4", True),
    ("u12k1", "-u 12 -k 1", True), ("g14", "-g 14", False), ("g16", "-g 16", False),
    ("el4", "-f {graphs}/4.el", True), ("el4s", "-f {graphs}/4.el -s", True),
    ("mtx4", "-f {graphs}/4.mtx", True),
]


def depths_from_parents(parent, src):
    """Depth of every vertex along the parent pointers (-1 unreached)."""
    n = parent.size
    d = np.full(n, -1, np.int32)
    d[src] = 0
    level = np.array([src])
    k = 0
    not_src = np.arange(n) != src
    while level.size:
        nxt = np.nonzero(np.isin(parent, level) & (d == -1) & not_src)[0]
        k += 1
        d[nxt] = k
        level = nxt
    return d


def main_bfs():
    from gapbs_b200.graph import make_graph
    gdir = os.path.join(HERE, "graphs")
    out = {"generator": "tests/golden/make_golden.py --bfs", "cases": {}}
    for name, args, keep in BFS_CASES:
        a = args.format(graphs=gdir)
        (srcs, _, _), _ = capture_stdout(oracle.ref_bfs, a, 3, -1, False)
        g = make_graph(a)
        odeg = np.diff(g.out_offsets)
        runs = []
        for src in srcs:
            (_, parent, _), _ = capture_stdout(oracle.ref_bfs, a, 3, int(src), True)
            d = depths_from_parents(parent, int(src))
            reached = parent >= 0
            run = {"source": int(src), "reached": int(reached.sum()),
                   "tree_edges": int(odeg[reached].sum()), "depth_sha256": sha(d),
                   "max_depth": int(d.max())}
            if keep:
                run["depths"] = [int(x) for x in d]
            runs.append(run)
        out["cases"][name] = {"args": args, "num_nodes": g.num_nodes, "runs": runs}
        print(name, [r["source"] for r in runs], [r["reached"] for r in runs])
    with open(os.path.join(HERE, "bfs_golden.json"), "w") as fh:
        json.dump(out, fh, separators=(",", ":"))


if __name__ == "__main__":
    if "--bfs" in sys.argv[1:]:
        main_bfs()
    elif "--fullsize" in sys.argv[1:]:
        main_fullsize()
    elif "--cli" in sys.argv[1:]:
        main_cli()
    elif "--cc" in sys.argv[1:]:
        main_cc()
    else:
        main()
        main_cli()
        main_cc()
        main_bfs()
