"""Replica plumbing of bench.py at world size 2 on CPU (gloo).

bench.py runs N independent PageRank solves, one per GPU: rank 0 builds the
graph once and the other ranks read it back from a .sg file; timings are
combined with one barrier and a max over ranks.  These tests run that
plumbing as two gloo ranks under torch.distributed.run on 127.0.0.1 and check
that both ranks hold the identical graph, that max/sum reduce across ranks,
and that the reference arm prints one line from rank 0 and nothing else.
"""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
import textwrap

import pytest

from conftest import ROOT

WORKER = textwrap.dedent("""
    import hashlib, json, os, sys
    sys.path.insert(0, {root!r})
    import bench
    d = bench.Dist(init=True)
    assert d.world == 2 and d.pg is not None
    g = bench.load_graph("-g 10", d)
    h = hashlib.sha256()
    for a in (g.out_offsets, g.out_neighbors, g.in_offsets, g.in_neighbors):
        h.update(a.tobytes())
    mx = d.max(float(d.rank + 1))
    sm = d.sum(float(10 * (d.rank + 1)))
    hashes = [None, None]
    d.pg.all_gather_object(hashes, h.hexdigest())
    leftover = os.path.exists(bench.shm_graph_path("-g 10"))
    d.barrier()
    with open(f"rank{{d.rank}}.json", "w") as f:
        json.dump({{"rank": d.rank, "max": mx, "sum": sm, "hashes": hashes,
                   "n": g.num_nodes, "m": g.num_edges_directed, "leftover": leftover}}, f)
    d.close()
""")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _torchrun(args, tmp_path, timeout=240):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port())] + args
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="2")
    return subprocess.run(cmd, cwd=str(tmp_path), env=env, capture_output=True, text=True,
                          timeout=timeout)


def test_replicas_share_identical_graph(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(root=ROOT))
    p = _torchrun([str(script)], tmp_path)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-4000:]
    rows = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in (0, 1)]
    assert sorted(r["rank"] for r in rows) == [0, 1]
    from gapbs_b200.graph import make_graph
    g = make_graph("-g 10")
    for r in rows:
        assert r["max"] == 2.0
        assert r["sum"] == 30.0
        assert r["hashes"][0] == r["hashes"][1]
        assert (r["n"], r["m"]) == (g.num_nodes, g.num_edges_directed)
        assert not r["leftover"]


def test_reference_arm_prints_once_under_torchrun(tmp_path):
    import oracle
    if not oracle.ref_available():
        pytest.skip("reference not compiled here")
    p = _torchrun([os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                   "--graph", "-g 10", "--steps", "2", "--warmup", "3"], tmp_path)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-4000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    res = json.loads(lines[0])
    assert res["impl"] == "reference"
    assert res["n_gpus"] == 2
    assert res["value"] > 0
    assert res["e2e"]["h2d_bytes_per_step"] == 0
    assert res["cpu_baseline"]["kind"] == "reference"
