"""Batched worlds shard across ranks with no data-path collective (CPU, gloo, world size 2).

Rank r builds the worlds i with i % N == r; each world is the same whichever rank builds it,
every world lands on exactly one rank, and one all-reduce of the ranks' counts after the timed
region gives the whole batch's contact-solves (the bench's strong-scaling line)."""
from __future__ import annotations

import os
import socket

import numpy as np
import torch.multiprocessing as mp

COUNT = 48
MAX_BODIES = 96


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch
    import torch.distributed as dist

    from nepheline_b200 import scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    scs = scenes.batched_worlds(COUNT, seed=3, max_bodies=MAX_BODIES, shard=rank, shards=world)
    mine = [(i, len(sc.bodies), len(sc.contacts), len(sc.joints))
            for i, sc in zip(range(rank, COUNT, world), scs)]
    solves = torch.tensor([float(sum(2 * 4 * m for _, _, m, _ in mine)), float(len(mine))],
                          dtype=torch.float64)
    dist.all_reduce(solves)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    if rank == 0:
        out.put((solves.tolist(), gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_worlds_shard_over_two_ranks():
    from nepheline_b200 import scenes
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    solves, gathered = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    whole = scenes.batched_worlds(COUNT, seed=3, max_bodies=MAX_BODIES)
    expect = {i: (len(sc.bodies), len(sc.contacts), len(sc.joints)) for i, sc in enumerate(whole)}
    seen = {}
    for rank_worlds in gathered:
        for i, nb, m, nj in rank_worlds:
            assert i not in seen
            seen[i] = (nb, m, nj)
    assert seen == expect
    assert solves[1] == COUNT
    assert solves[0] == float(sum(2 * 4 * m for _, m, _ in expect.values()))
    # Each world is the same whichever rank builds it.
    again = scenes.batched_worlds(COUNT, seed=3, max_bodies=MAX_BODIES, shard=1, shards=2)
    assert np.array_equal(again[0].bodies, whole[1].bodies)
