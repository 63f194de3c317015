"""The multi-rank plumbing of bench.py on CPU: two `gloo` ranks (world size 2,
rendezvous on 127.0.0.1) run its barrier and max-over-ranks helpers and the
whole-job throughput formula, as `bench.py --gpus 2` does over NCCL with one
replica of the contraction per GPU; and the reference arm, launched as rank 1
of 2, exits without work or output (rank 0 alone prints its line)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        barrier_sync, max_over_ranks = bench.rank_sync(torch, dist, None)
        barrier_sync()
        seconds = 1.0 + rank                  # the slower rank sets the job's time
        t = max_over_ranks(seconds)
        value = bench.aggregate_tflops(world, 1e12, 3, t)
        barrier_sync()
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"t": t, "value": value}, f)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(rank_main, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for rank in range(world):
        with open(tmp_path / f"rank{rank}.json") as f:
            r = json.load(f)
        assert r["t"] == 2.0
        # 2 replicas x 3 steps x 1 TFLOP in 2 s
        assert r["value"] == pytest.approx(3.0)


def test_single_process_needs_no_group():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    barrier_sync, max_over_ranks = bench.rank_sync(torch, None, None)
    barrier_sync()
    assert max_over_ranks(1.25) == 1.25


def test_reference_arm_on_a_nonzero_rank_is_silent():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--gpus", "2"], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""
