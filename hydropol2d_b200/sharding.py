"""Batched-ensemble members across GPUs, one process per GPU.

Members are independent (HydroPol2D_Main_While_Ensemble.m:46-139 runs them one after the
other; Probabilistic_dam_break_analysis.m:8-60 only combines their maps afterwards), so the
multi-GPU form needs no collective on the data path: every rank builds its own share of
the members and advances them as one ``Ensemble`` on its own GPU.  The host-side
collectives are the maximum over ranks of the device time and one gather of the
per-member results to rank 0, both over ``torch.distributed`` (NCCL between GPUs, gloo on
CPU).

The share is a longest-processing-time-first partition of the members' a priori costs,
computed identically on every rank, so no rank has to tell another what to run.
"""
from __future__ import annotations

from typing import Callable, Sequence


def shard(costs: Sequence[float], world: int) -> list[list[int]]:
    """Members (by index) per rank: members in decreasing cost (ties by lower index) go
    one by one to the rank with the least total cost so far (ties to the lower rank).
    Every member lands on exactly one rank; each rank's list is in increasing index."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def rank_world(group=None) -> tuple[int, int]:
    """This process's rank and the world size (0, 1 without an initialised process group)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def max_over_ranks(value: float, group=None, device=None) -> float:
    """The largest ``value`` over the ranks of ``group`` (the value itself on one rank)."""
    import torch
    import torch.distributed as dist
    _, world = rank_world(group)
    if world == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_results(local: list[dict], group=None) -> list[dict] | None:
    """Rank 0 receives every rank's per-member result dicts, ordered by member index
    (``index`` key); the other ranks receive None."""
    import torch.distributed as dist
    rank, world = rank_world(group)
    if world == 1:
        return sorted(local, key=lambda d: d["index"])
    bucket = [None] * world if rank == 0 else None
    dist.gather_object(local, bucket, dst=0, group=group)
    if rank != 0:
        return None
    return sorted((d for part in bucket for d in part), key=lambda d: d["index"])


def run_sharded(make_case: Callable[[int], object], n_members: int, costs: Sequence[float] | None = None,
                device: int = 0, group=None, autotune_steps: int = 8, launches_per_poll: int = 512,
                maxima: bool = False, ensemble_factory=None, member_factory=None) -> dict | None:
    """Runs members 0..n_members-1 over all ranks of ``group`` and returns, on rank 0, a
    summary with the per-member results ({index, steps, t, cells, and the peak-depth map in
    metres when ``maxima``}); None on the other ranks.

    ``make_case(i)`` builds member i (a ``synthetic.Case``); only the members of this rank's
    share are built.  ``costs`` balance the shares (default: cells, which needs every case
    built on every rank -- pass a cheap estimate such as ``synthetic.ensemble_member_cost``).
    Timing: CUDA events on each rank's ensemble stream around every launch until its last
    member reaches its routing time; the job's time is the maximum over ranks, so
    ``members_per_h`` is the whole job's throughput."""
    rank, world = rank_world(group)
    if costs is None:
        costs = [float(make_case(i).z.size) for i in range(n_members)]
    if len(costs) != n_members:
        raise ValueError("one cost per member")
    mine = shard(costs, world)[rank]
    if ensemble_factory is None or member_factory is None:
        from .ensemble import Ensemble
        from .surface import SurfaceFlow
        ensemble_factory = ensemble_factory or Ensemble
        member_factory = member_factory or (
            lambda c: SurfaceFlow(*c.shape, c.resolution, "fp32", device=device, **c.params))
    ens = ensemble_factory(device)
    for i in mine:
        c = make_case(i)
        m = member_factory(c)
        c.apply(m)
        ens.add(m)
    ms_total, launches, rpw = 0.0, 0, None
    try:
        if mine:
            rpw = ens.autotune(autotune_steps)
            active = len(mine)
            while active:
                active, ms = ens.steps_timed(launches_per_poll)
                ms_total += ms
                launches += launches_per_poll
        local = []
        for i, m in zip(mine, ens.members):
            d = m.diag()
            r = {"index": i, "rank": rank, "steps": int(d["k"]) - 1, "t": float(d["t"]),
                 "cells": int(m.ny * m.nx)}
            if maxima:
                r["max_depth_m"] = m.download("dmax") / 1000.0
            local.append(r)
    finally:
        ens.close()
    seconds = max_over_ranks(ms_total / 1e3, group, device=_collective_device(device, group))
    results = gather_results(local, group)
    if rank != 0:
        return None
    cu = sum(r["cells"] * r["steps"] for r in results)
    return {"members": n_members, "ranks": world, "seconds": seconds,
            "members_per_h": n_members / seconds * 3600.0 if seconds > 0 else float("inf"),
            "gcups": cu / seconds / 1e9 if seconds > 0 else float("inf"),
            "launches_rank0": launches, "rows_per_warp_rank0": rpw,
            "members_per_rank": [len(p) for p in shard(costs, world)],
            "results": results}


def _collective_device(device: int, group=None):
    """Tensors of a collective live on this rank's GPU under NCCL and on the host under
    gloo."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_backend(group) == "nccl":
        return f"cuda:{device}"
    return "cpu"
