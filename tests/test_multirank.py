"""The bench's multi-rank host logic on two gloo ranks (CPU): device times combine as the
maximum over ranks, the whole-job rate counts every rank's elements at that time, and the
reference arm runs on rank 0 alone."""
import json
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = [1.0 + rank, 10.0 - rank]  # rank 1 is slower on the first time, faster on the second
        got = bench.max_over_ranks(mine, dist, "cpu")
        dist.barrier()
        out.put((rank, got, bench.whole_job_rate(world, 1_000_000, got[0])))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rate_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, rate in res:
        assert got == [2.0, 10.0]  # element-wise maximum over the two ranks
        assert rate == pytest.approx(2 * 1_000_000 / 2e-3 / 1e6)  # both ranks' elements at the slowest time


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import argparse

    import bench

    args = argparse.Namespace(steps=1, warmup=1)
    bench.run_reference_arm(args, rank=1, world=2, workload="jacobian_60")
    assert capsys.readouterr().out == ""  # a non-zero rank does no work and prints nothing
