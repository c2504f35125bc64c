"""Batched worlds shard across ranks with no data-path collective (CPU, gloo, world size 2).

Rank r builds the worlds i with i % N == r; each world is the same whichever rank builds it,
every world lands on exactly one rank, and one all-reduce of the ranks' counts after the timed
region gives the whole batch's contact-solves (the bench's strong-scaling line). Each rank steps
its shard (here with the CPU restatement of the solver stage, the device's checker) with no
collective between steps, and every world's result equals the world stepped in the unsharded
batch."""
from __future__ import annotations

import os
import socket

import numpy as np
import torch.multiprocessing as mp

COUNT = 48
MAX_BODIES = 96
STEPS = 3
DT = 1.0 / 60.0


def _digest(view) -> str:
    import hashlib
    h = hashlib.sha256()
    for a in (view.bodies, view.contacts, view.joints):
        h.update(a.tobytes())
    return h.hexdigest()


def _step_worlds(scs) -> list:
    """Each world coloured in insertion order and stepped STEPS times."""
    from nepheline_b200 import abi, scenes
    from oracle.refworld import port32
    params = abi.WorldParams.default()
    out = []
    for sc in scs:
        v = sc.to_view(*scenes.host_color(sc))
        for _ in range(STEPS):
            v = port32(v, params, DT)
        out.append(_digest(v))
    return out


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
    digests = _step_worlds(scs)  # the shard's steps: no collective until the counts below
    mine = [(i, len(sc.bodies), len(sc.contacts), len(sc.joints), dg)
            for i, sc, dg in zip(range(rank, COUNT, world), scs, digests)]
    solves = torch.tensor([float(STEPS * sum(2 * 4 * m for _, _, m, _, _ in mine)),
                           float(len(mine))],
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
    stepped = _step_worlds(whole)
    expect = {i: (len(sc.bodies), len(sc.contacts), len(sc.joints), stepped[i])
              for i, sc in enumerate(whole)}
    seen = {}
    for rank_worlds in gathered:
        for i, nb, m, nj, dg in rank_worlds:
            assert i not in seen
            seen[i] = (nb, m, nj, dg)
    assert seen == expect  # every world on one rank, its results those of the unsharded run
    assert solves[1] == COUNT
    assert solves[0] == float(STEPS * sum(2 * 4 * m for _, m, _, _ in expect.values()))
    # Each world is the same whichever rank builds it.
    again = scenes.batched_worlds(COUNT, seed=3, max_bodies=MAX_BODIES, shard=1, shards=2)
    assert np.array_equal(again[0].bodies, whole[1].bodies)
