"""bench.py's multi-rank host logic on CPU, two ranks (gloo).

bench.py --gpus N runs one rank per GPU: each rank solves its own replica,
the step times are the maximum over ranks (one all-reduce per timing, in the
same order on every rank), and rank 0 alone prints the JSON line. The
reference arm runs on rank 0 only; the other ranks exit at once. Both are
checked here on CPU, launched as bench.py is for N > 1 (torch.distributed.run).
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def torchrun(args, nproc=2, timeout=300):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", str(nproc),
           "--master-addr", "127.0.0.1", "--master-port", str(free_port())] + args
    env = dict(os.environ, OMP_NUM_THREADS="1")
    return subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=timeout, env=env)


def json_lines(text):
    return [json.loads(line) for line in text.splitlines() if line.startswith("{")]


def test_step_times_are_max_over_ranks(tmp_path):
    out = torchrun([os.path.join("tests", "multirank_worker.py"), str(tmp_path)])
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(2)]
    assert [d["rank"] for d in lines] == [0, 1]
    for d in lines:
        assert d["world"] == 2
        assert (d["total"], d["sweep"], d["e2e"]) == (110.0, 2.0, 100.0)
        # whole-job throughput: 2 replicas x 1e6 entries x 20 sweeps in 11 ms
        assert d["gteps"] == pytest.approx(2 * 1e6 * 20 / 11e-3 / 1e9)


def test_job_gteps_counts_every_replica():
    sys.path.insert(0, ROOT)
    import bench
    one = bench.job_gteps(1, 5e8, 20, 30.0)
    assert bench.job_gteps(4, 5e8, 20, 30.0) == pytest.approx(4 * one)
    assert one == pytest.approx(5e8 * 20 / 0.030 / 1e9)
    assert bench.max_over_ranks([1.0, 2.5]) == [1.0, 2.5]  # one process: no collective


def test_reference_arm_prints_once_under_torchrun():
    out = torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--scale", "10", "--steps", "1",
                    "--warmup", "1", "--cpu-sample-sweeps", "1"])
    assert out.returncode == 0, out.stderr[-2000:]
    lines = json_lines(out.stdout)
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] in ("reference", "port")


def test_hub_tier_counts_follow_the_relabelling():
    """bench.hub_tier_counts (the gather roofline's load count) against a
    brute-force count over the engine's relabelling: vertices by descending
    row length, stably."""
    import numpy as np
    import torch

    import bench
    from nwgraph_b200 import graphs as G
    g = G.rmat(11, 16, 7)
    lens = np.diff(g.row_ptr.astype(np.int64))
    order = np.argsort(-lens, kind="stable")
    newid = np.empty(g.n, np.int64)
    newid[order] = np.arange(g.n)
    ids = newid[g.col.astype(np.int64)]
    thresholds = [0, 100, 512, 2000, g.n]
    got = bench.hub_tier_counts(torch.from_numpy(g.row_ptr.view(np.int32)), torch.from_numpy(g.col.view(np.int32)),
                                thresholds)
    assert got == [int((ids >= t).sum()) for t in thresholds]
