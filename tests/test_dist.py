"""The multi-GPU path's host plumbing on CPU (gloo, world size 2): samples are independent
replicas, so the only cross-rank steps are bench.py's timing barrier and its reductions
(max of the ranks' times, sum of their work), and rank 0 alone prints the JSON line."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench

    dist = bench.Dist()
    try:
        dist.barrier()
        result = {"max": dist.reduce(10.0 * (rank + 1), "max"), "sum": dist.reduce(rank + 1.5, "sum"),
                  "world": dist.world, "rank": dist.rank}
    finally:
        dist.close()
    with open(out / f"rank{rank}.json", "w") as f:
        json.dump(result, f)


def test_barrier_and_reductions_over_two_ranks(tmp_path):
    port = free_port()
    mp.start_processes(_rank, args=(2, port, tmp_path), nprocs=2, join=True, start_method="spawn")
    for rank in range(2):
        r = json.loads((tmp_path / f"rank{rank}.json").read_text())
        assert r == {"max": 20.0, "sum": 4.0, "world": 2, "rank": rank}


def test_reference_arm_under_torchrun_prints_one_line():
    """bench.py --impl reference launched as the driver launches it for N=2: rank 0 times the
    oracle port (one whole FP64 step here) and prints one JSON line, the other rank exits 0
    without work."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(free_port()), str(ROOT / "bench.py"), "--impl", "reference", "--gpus",
           "2", "--steps", "1", "--warmup", "0"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    done = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert done.returncode == 0, done.stderr[-2000:]
    lines = [json.loads(l) for l in done.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["metric"] == "pair-evals/s"
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["ms_per_step"] == line["step_ms"]["p50"]  # measured, one step
    assert line["e2e"] == {"value": line["value"], "unit": "pair-evals/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def _served_split_rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    from zxtalori_b200 import serve

    dist = bench.Dist()
    try:
        reqs = serve.poisson_requests(2.0, 40.0, seed=5)
        mine = serve.shard_requests(reqs, dist.rank, dist.world)
        gathered = dist.gather([r.id for r in mine])
    finally:
        dist.close()
    with open(out / f"served{rank}.json", "w") as f:
        json.dump({"total": len(reqs), "parts": gathered}, f)


def test_served_stream_split_over_two_ranks(tmp_path):
    """bench.py --gpus N splits config 5's request stream over the ranks (request k to rank
    k mod N) and gathers every rank's results: each request is served by exactly one rank,
    and every rank sees the same gathered list."""
    port = free_port()
    mp.start_processes(_served_split_rank, args=(2, port, tmp_path), nprocs=2, join=True, start_method="spawn")
    seen = [json.loads((tmp_path / f"served{rank}.json").read_text()) for rank in range(2)]
    assert seen[0] == seen[1]
    parts = seen[0]["parts"]
    ids = sorted(i for part in parts for i in part)
    assert ids == list(range(seen[0]["total"]))
    assert all(i % 2 == rank for rank, part in enumerate(parts) for i in part)
