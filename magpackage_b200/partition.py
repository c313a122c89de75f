"""Independent assembly instances split across ranks, one process per GPU.

The instances of a batched assembly (the meshes of a frequency sweep, the harmonics of
an HBFEM run, unrelated meshes; FrequencySolver.m:131 assembles each frequency's
K + j*omega*M on its own) share no data, so ranks need no exchange to assemble them:
each rank computes the same split from the instances' sizes and assembles its own part
in one batch. The only collective of a multi-rank run is the maximum of the device
times that the benchmark reports.
"""
from __future__ import annotations


def partition_instances(sizes, world: int) -> list[list[int]]:
    """One ascending list of instance indices per rank.

    Largest instance first, each to the rank with the least work so far (ties go to the
    lower rank; instances of equal size are taken in index order), so that the ranks'
    loads differ by at most the largest instance. The split depends only on `sizes` and
    `world`: every rank that calls it gets the same answer. A rank may get no instance
    when there are fewer instances than ranks.
    """
    world = int(world)
    if world < 1:
        raise ValueError("world must be at least 1")
    sizes = [int(s) for s in sizes]
    if any(s < 0 for s in sizes):
        raise ValueError("instance sizes must be non-negative")
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


def rank_loads(sizes, parts) -> list[int]:
    """Total size each rank assembles under `parts`."""
    return [sum(int(sizes[i]) for i in p) for p in parts]
