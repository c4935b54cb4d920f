"""Sharding of a batched ensemble across GPUs.

The cases of an ensemble are independent, so an ensemble spread over N GPUs needs no per-step
exchange: each rank advances its own share with the persistent ensemble kernel and only the
totals are combined at the end.  Shares are balanced by estimated work (cells x steps) with the
greedy longest-processing-time rule: cases in decreasing order of work, each to the rank with
the least work so far (ties to the lower rank), which every rank computes identically.
"""

from __future__ import annotations

from typing import List, Sequence


def case_work(n_cells: int, t_end: float, dt_estimate: float) -> float:
    """Estimated work of a case: cells x steps to its end time."""
    return float(n_cells) * max(1.0, t_end / dt_estimate)


def partition(work: Sequence[float], world: int) -> List[List[int]]:
    """Case indices per rank (each list in increasing index order)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(work)), key=lambda i: (-work[i], i))
    load = [0.0] * world
    shares: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        shares[r].append(i)
        load[r] += work[i]
    return [sorted(s) for s in shares]


def imbalance(work: Sequence[float], shares: Sequence[Sequence[int]]) -> float:
    """Largest rank load over the mean rank load (1.0 is perfect balance)."""
    loads = [sum(work[i] for i in s) for s in shares]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


def combine_rank_totals(dist, device, sums: dict, maxes: dict) -> dict:
    """Job totals of per-rank figures: `sums` (cell updates, cells) summed and `maxes` (device
    times) maxed over the ranks of the process group `dist` (torch.distributed; None for one
    rank).  Every rank takes the same two collectives in the same order."""
    out = dict(sums)
    out.update(maxes)
    if dist is None:
        return out
    import torch

    ks, km = sorted(sums), sorted(maxes)
    if ks:
        t = torch.tensor([float(sums[k]) for k in ks], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        out.update({k: float(v) for k, v in zip(ks, t.tolist())})
    if km:
        m = torch.tensor([float(maxes[k]) for k in km], device=device, dtype=torch.float64)
        dist.all_reduce(m, op=dist.ReduceOp.MAX)
        out.update({k: float(v) for k, v in zip(km, m.tolist())})
    return out
