"""The benchmark's multi-rank plumbing on CPU: two gloo ranks on 127.0.0.1
take the max of their step times, pass the barrier, and convert different
seeded clouds (replicas: no data-path collective); the reference arm runs
on rank 0 only."""

import os
import socket
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys
sys.path.insert(0, sys.argv[1])
import torch
import bench
dist = bench.dist_init("gloo")
rank = int(os.environ["RANK"])
dev = torch.device("cpu")
v = bench.max_over_ranks(dist, 10.0 + 5.0 * rank, dev)
bench.barrier(dist, dev)
print("RESULT", rank, v, bench.replica_seed(rank), flush=True)
dist.destroy_process_group()
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_max_barrier_and_seeds(tmp_path):
    port = _free_port()
    script = tmp_path / "worker.py"
    script.write_text(WORKER)
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), LOCAL_RANK=str(rank),
                   WORLD_SIZE="2", CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, str(script), REPO], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        out, _ = p.communicate(timeout=180)
        assert p.returncode == 0, out
        outs.append(out)
    results = {}
    for out in outs:
        for line in out.splitlines():
            if line.startswith("RESULT"):
                _, rank, v, seed = line.split()
                results[int(rank)] = (float(v), int(seed))
    assert set(results) == {0, 1}
    assert results[0][0] == results[1][0] == 15.0  # max over ranks
    assert results[0][1] != results[1][1]           # each rank its own cloud


def test_aggregate_is_total_points_over_max_time():
    sys.path.insert(0, REPO)
    import bench
    assert bench.aggregate_mpts(2, 50_000_000, 250.0) == pytest.approx(400.0)
    assert bench.aggregate_mpts(1, 50_000_000, 250.0) == pytest.approx(200.0)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
