"""Ensemble members across ranks (hydropol2d_b200.sharding): the partition, and the
multi-rank orchestration run as two and three gloo ranks on the CPU with a stand-in
ensemble (the GPU ensemble itself is covered by test_gpu_ensemble.py)."""
import json
import os
import socket

import numpy as np
import pytest

from hydropol2d_b200.sharding import gather_results, max_over_ranks, run_sharded, shard


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shard_is_a_balanced_partition(world):
    rng = np.random.default_rng(world)
    costs = rng.lognormal(0.0, 1.0, 97)
    parts = shard(costs, world)
    assert len(parts) == world
    flat = [i for p in parts for i in p]
    assert sorted(flat) == list(range(97))
    assert all(p == sorted(p) for p in parts)
    loads = [sum(costs[i] for i in p) for p in parts]
    # greedy LPT: no rank exceeds the mean load by more than the largest single cost
    assert max(loads) <= sum(costs) / world + max(costs) + 1e-9
    assert shard(costs, world) == parts   # deterministic: every rank computes the same


def test_shard_more_ranks_than_members():
    parts = shard([3.0, 1.0], 4)
    assert parts == [[0], [1], [], []]


def test_synthetic_member_costs_balance_the_benchmark_ensemble():
    from hydropol2d_b200 import synthetic as S
    costs = [S.ensemble_member_cost(i) for i in range(256)]
    for world in (2, 4, 8):
        loads = [sum(costs[i] for i in p) for p in shard(costs, world)]
        assert max(loads) / (sum(costs) / world) < 1.05
    spec = S.ensemble_member_spec(5)
    case = S.ensemble_member(5)
    assert case.shape == (spec["ny"], spec["nx"]) and case.meta["kind"] == spec["kind"]


# ---- multi-rank orchestration with a stand-in ensemble ------------------------------

class _Member:
    def __init__(self, case):
        self.ny, self.nx = case.shape
        self.index = case.index
        self.k = 1

    def diag(self):
        return {"k": self.k, "t": 10.0 * self.index}

    def download(self, field):
        assert field == "dmax"
        return np.full((self.ny, self.nx), 1000.0 * self.index)


class _Ensemble:
    """Advances every member 7 steps per poll until each has run 3 * (index + 1) steps;
    reports a device time of 1 ms per poll per member on this rank."""

    def __init__(self, device):
        self.members = []

    def add(self, m):
        self.members.append(m)

    def autotune(self, n):
        return 40

    def steps_timed(self, n):
        for m in self.members:
            m.k = min(m.k + 7, 3 * (m.index + 1) + 1)
        active = sum(m.k < 3 * (m.index + 1) + 1 for m in self.members)
        return active, float(len(self.members))

    def close(self):
        pass


class _Case:
    def __init__(self, i):
        self.index = i
        self.shape = (2 + i % 3, 5)

    def apply(self, m):
        m.applied = True


def _rank_main(rank, world, port, n_members, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assert max_over_ranks(float(rank + 1)) == float(world)
        g = gather_results([{"index": 10 * rank + 1, "rank": rank}])
        if rank == 0:
            assert [d["rank"] for d in g] == list(range(world))
        else:
            assert g is None
        costs = [float(n_members - i) for i in range(n_members)]
        res = run_sharded(_Case, n_members, costs=costs, device=0, ensemble_factory=_Ensemble,
                          member_factory=_Member, maxima=True, launches_per_poll=1)
        if rank == 0:
            res["results"] = [{k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in r.items()}
                              for r in res["results"]]
            with open(out, "w") as f:
                json.dump(res, f)
        else:
            assert res is None
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,n_members", [(2, 9), (3, 2)])
def test_run_sharded_over_gloo_ranks(tmp_path, world, n_members):
    import torch.multiprocessing as mp
    out = str(tmp_path / "res.json")
    mp.spawn(_rank_main, args=(world, _free_port(), n_members, out), nprocs=world, join=True)
    res = json.load(open(out))
    parts = shard([float(n_members - i) for i in range(n_members)], world)
    assert res["members_per_rank"] == [len(p) for p in parts]
    got = res["results"]
    assert [r["index"] for r in got] == list(range(n_members))          # each member once, in order
    for r in got:
        assert parts[r["rank"]].count(r["index"]) == 1                   # run where it was assigned
        assert r["steps"] == 3 * (r["index"] + 1)                        # ran to its own end
        assert r["t"] == 10.0 * r["index"]
        assert np.all(np.asarray(r["max_depth_m"]) == r["index"])         # mm -> m
    # job time = the slowest rank's: polls until its longest member ends x members on it
    per_rank = []
    for p in parts:
        polls = max((-(-3 * (i + 1) // 7) for i in p), default=0)
        per_rank.append(polls * len(p) / 1e3)
    assert res["seconds"] == pytest.approx(max(per_rank))
    assert res["members_per_h"] == pytest.approx(n_members / max(per_rank) * 3600)
