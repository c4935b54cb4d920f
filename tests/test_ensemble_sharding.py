"""Sharding of the batched ensemble over ranks (schemi_b200.ensemble): every case on exactly one
rank, the same partition on every rank, balanced estimated work, and the two-rank aggregation the
benchmark performs (sum of cell updates, max of device time) over torch.distributed with gloo."""

import math
import os
import socket

import pytest


def _rm_work(n_cases):
    from schemi_b200 import cases, ensemble

    ws = 1.2 * math.sqrt(1.4)
    draws = [cases.richtmyer_meshkov_draws(i) for i in range(n_cases)]
    return [ensemble.case_work(n * n, tr / ws, 0.5 / (n * 2.5)) for n, _, _, tr in draws]


@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_partition_covers_every_case_once_and_balances(world):
    from schemi_b200 import ensemble

    work = _rm_work(512)
    shares = ensemble.partition(work, world)
    flat = sorted(i for s in shares for i in s)
    assert flat == list(range(512))
    assert ensemble.partition(work, world) == shares  # deterministic
    assert ensemble.imbalance(work, shares) < 1.01


def test_partition_edge_cases():
    from schemi_b200 import ensemble

    assert ensemble.partition([], 3) == [[], [], []]
    assert ensemble.partition([5.0], 2) == [[0], []]
    assert ensemble.partition([1.0, 1.0, 1.0], 3) == [[0], [1], [2]]
    with pytest.raises(ValueError):
        ensemble.partition([1.0], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    from schemi_b200 import ensemble

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        work = _rm_work(64)
        shares = ensemble.partition(work, world)
        mine = shares[rank]
        # what every rank reports: its cell updates and a device time; the job value uses the
        # sum of updates and the max of times
        tot = ensemble.combine_rank_totals(dist, "cpu", sums={"updates": sum(work[i] for i in mine)},
                                           maxes={"ms": 1.0 + rank})
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        out[rank] = (gathered, tot["updates"], tot["ms"])
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_with_gloo():
    import torch.multiprocessing as mp

    world, port = 2, _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    work = _rm_work(64)
    g0, u0, m0 = res[0]
    g1, u1, m1 = res[1]
    assert g0 == g1  # every rank sees the same shares
    assert sorted(g0[0] + g0[1]) == list(range(64)) and not set(g0[0]) & set(g0[1])
    assert u0 == u1 == pytest.approx(sum(work))
    assert m0 == m1 == 2.0
