"""The replica path of `bench.py --gpus N` on CPU: two gloo ranks, no GPU.

Each GPU runs its own world; the only collectives are the measurement's (a barrier and the
reduction of work and device time), and the reference arm runs on rank 0 alone.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world_size, port, out_dir):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from solunar_b200.replicas import reduce_timing

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world_size)
    try:
        # rank r did 10 + r substeps in 5 (r + 1) ms
        work, slowest = reduce_timing(10 + rank, 5.0 * (rank + 1), world_size)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"work": work, "slowest": slowest}, f)
    finally:
        dist.destroy_process_group()


def test_two_ranks_sum_their_work_over_the_slowest_time(tmp_path):
    port = free_port()
    mp.start_processes(rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for rank in range(2):
        got = json.load(open(tmp_path / f"rank{rank}.json"))
        assert got == {"work": 21, "slowest": 10.0}


def test_one_rank_exchanges_nothing():
    sys.path.insert(0, ROOT)
    from solunar_b200.replicas import reduce_timing

    assert reduce_timing(7, 3.5, 1) == (7, 3.5)


def test_the_reference_arm_runs_on_rank_zero_alone():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
