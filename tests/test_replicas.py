"""Replicas (one process per GPU, no data-path collective): the bench's
max-over-ranks time and summed work, and the reference arm under a
2-rank launch, on CPU with gloo."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, out):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2)
    out[rank] = bench.replica_totals(dist, "cpu", 1.5 + rank, 10 * (rank + 1))
    dist.destroy_process_group()


def test_replica_totals_take_the_slowest_rank_and_all_work():
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(_free_port(), out), nprocs=2, join=True)
    assert out[0] == out[1] == (2.5, 30.0)


def test_reference_arm_under_two_ranks():
    env = dict(os.environ, MASTER_ADDR="127.0.0.1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--bodies", "2000"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
