"""The multi-GPU path of bench.py is N independent replicas (no data-path
collective): each rank times its own steps, and the job's figures are the
slowest rank's time and the edges of all ranks.  These tests run that
reduction with two gloo ranks on the CPU, and check that the reference arm
runs on rank 0 alone."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        ms = 10.0 + 5.0 * rank          # rank 1 is the slower replica
        edges = 1000.0 * (rank + 1)
        res = bench.replica_totals(ms, edges, world)
        bench.barrier(world)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(res, f)
    finally:
        dist.destroy_process_group()


def test_replica_totals_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for rank in range(world):
        ms_max, tot, value = json.load(open(tmp_path / f"rank{rank}.json"))
        assert ms_max == 15.0              # max over ranks, not the local time
        assert tot == 3000.0               # edges of both replicas
        assert value == pytest.approx(3000.0 / 0.015)


def test_replica_totals_single_rank_is_local():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.replica_totals(4.0, 200.0, 1) == (4.0, 200.0, 200.0 / 0.004)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0
    assert p.stdout.strip() == ""
