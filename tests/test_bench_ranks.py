"""The multi-GPU plumbing of bench.py on CPU: N replicas (one lattice per
GPU, no data-path collective) report the whole job's MLUPS over the slowest
replica's time, taken as the maximum over ranks; the reference arm runs on
rank 0 only.  Two `gloo` ranks on 127.0.0.1 stand in for two GPUs."""
import argparse
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    seconds = bench.max_over_ranks(dist, 0.5 + rank, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, seconds, bench.job_mlups(world, 1000, 10, seconds)))


def test_two_replicas_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [1.5, 1.5]
    assert all(abs(o[2] - 2 * 1000 * 10 / 1.5 / 1e6) < 1e-12 for o in out)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import bench
    args = argparse.Namespace(steps=1, warmup=1)
    assert bench.reference_arm(args, rank=1, world=2) == 0
    assert capsys.readouterr().out == ""
    assert bench.max_over_ranks(None, 3.25, "cpu") == 3.25
