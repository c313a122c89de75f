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


def _partition_rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch

    from magpackage_b200 import synth
    from magpackage_b200.partition import partition_instances

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sizes = synth.frequency_sweep_sizes(64)
        mine = partition_instances(sizes, world)[rank]  # computed locally: no exchange
        # what the ranks would assemble, gathered only to check the split
        t = torch.zeros(64, dtype=torch.int64)
        t[mine] = rank + 1
        got = [torch.zeros(64, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(got, t)
        out.put((rank, mine, [g.tolist() for g in got]))
    finally:
        dist.destroy_process_group()


def test_frequency_sweep_meshes_split_across_two_gloo_ranks():
    """Config 3's 64 meshes are independent: each rank computes the same split from the
    meshes' sizes, with no exchange, and assembles its own part. Gathered here only to
    check it: every mesh on exactly one rank, loads within the largest mesh of each other."""
    from magpackage_b200 import synth

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_partition_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sizes = synth.frequency_sweep_sizes(64)
    owner = [0] * 64
    for rank, mine, gathered in res:
        assert gathered == res[0][2]  # both ranks see the same assignment
        for i in mine:
            assert owner[i] == 0
            owner[i] = rank + 1
    assert all(o in (1, 2) for o in owner)
    assert owner == [max(g[i] for g in res[0][2]) for i in range(64)]  # the gathered view agrees
    loads = [sum(s for s, o in zip(sizes, owner) if o == r + 1) for r in range(2)]
    assert abs(loads[0] - loads[1]) <= max(sizes)


def test_partition_instances_properties():
    import numpy as np

    from magpackage_b200.partition import partition_instances, rank_loads

    rng = np.random.default_rng(3)
    for world in (1, 2, 3, 4, 8, 70):
        sizes = [int(x) for x in rng.integers(0, 10_000, size=64)]
        parts = partition_instances(sizes, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))  # a partition of the instances
        assert all(p == sorted(p) for p in parts)
        loads = rank_loads(sizes, parts)
        assert max(loads) - min(loads) <= max(sizes)  # largest-first to the least loaded
        assert parts == partition_instances(sizes, world)  # deterministic
    assert partition_instances([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        partition_instances([1, 2], 0)
