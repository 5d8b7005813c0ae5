"""The ragged batch sharded over ranks: LPT partition, the one gather, and the sharded step.

CPU: the partition's invariants and its balance against an exhaustive optimum, and a world-size-2 `gloo`
job that partitions and gathers like the multi-GPU run does.  GPU: two ranks' shares stepped one after the
other on one device (instances are independent, so nothing waits across shares) equal each instance
stepped alone with the same SM share, bit for bit.
"""
import itertools
import os
import socket

import numpy as np
import pytest

from ding_nsch_core_solver_b200.ensemble import (ShardedEnsemble, droplet_cfgs, estimated_cost, gather_records,
                                                 lpt_partition)


def _check_partition(parts, n, world):
    assert len(parts) == world
    flat = [i for p in parts for i in p]
    assert sorted(flat) == list(range(n))
    for p in parts:
        assert p == sorted(p)


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_lpt_partition_covers_each_instance_once(world):
    rng = np.random.default_rng(world)
    costs = rng.uniform(1, 100, size=37)
    parts = lpt_partition(costs, world)
    _check_partition(parts, len(costs), world)
    assert parts == lpt_partition(list(costs), world)  # a pure function: every rank computes the same


def test_lpt_partition_within_graham_bound():
    """LPT's makespan is at most (4/3 - 1/(3m)) of the optimum (Graham 1969): checked by enumeration."""
    rng = np.random.default_rng(3)
    for trial in range(40):
        world = int(rng.integers(2, 4))
        costs = rng.integers(1, 50, size=int(rng.integers(world, 9))).astype(float)
        parts = lpt_partition(costs, world)
        _check_partition(parts, len(costs), world)
        lpt = max(sum(costs[i] for i in p) for p in parts)
        opt = min(max(sum(costs[i] for i, a in enumerate(assign) if a == r) for r in range(world))
                  for assign in itertools.product(range(world), repeat=len(costs)))
        assert lpt <= (4 / 3 - 1 / (3 * world)) * opt + 1e-9, (trial, costs, parts)


def test_lpt_balances_the_droplet_batch():
    cfgs = droplet_cfgs(512)
    costs = [estimated_cost(c) for c in cfgs]
    for world in (2, 4, 8):
        parts = lpt_partition(costs, world)
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) / (sum(loads) / world) < 1.02, (world, loads)


def test_lpt_rejects_an_empty_world():
    with pytest.raises(ValueError):
        lpt_partition([1.0], 0)


def test_gather_without_process_group_keeps_order():
    assert gather_records(None, [0, 2, 5], ["a", "b", "c"]) == ["a", "b", "c"]
    with pytest.raises(RuntimeError):
        gather_records(None, [1, 1], ["a", "b"])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, out_dir):
    import json
    from datetime import timedelta

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        cfgs = droplet_cfgs(23, seed=9)
        parts = lpt_partition([estimated_cost(c) for c in cfgs], world)
        mine = parts[rank]
        recs = [{"instance": i, "rank": rank, "cells": cfgs[i]["nx"] * cfgs[i]["ny"]} for i in mine]
        allrec = gather_records(dist, mine, recs)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"parts": parts, "records": allrec}, f)
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_partition_and_gather(tmp_path):
    import json

    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_gloo_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    assert res[0] == res[1]  # both ranks hold the same partition and the same gathered list
    parts, recs = res[0]["parts"], res[0]["records"]
    _check_partition(parts, 23, world)
    cfgs = droplet_cfgs(23, seed=9)
    assert [r["instance"] for r in recs] == list(range(23))
    for r in recs:
        assert r["instance"] in parts[r["rank"]]
        assert r["cells"] == cfgs[r["instance"]]["nx"] * cfgs[r["instance"]]["ny"]


@pytest.mark.gpu
def test_sharded_steps_equal_each_instance_alone():
    from ding_nsch_core_solver_b200 import capi

    cfgs = droplet_cfgs(6, seed=7)
    world = 2
    for rank in range(world):  # one rank's share after the other: the shares never wait on each other
        shard = ShardedEnsemble(cfgs, rank, world)
        twins = [capi.Solver(dict(cfgs[i], device_share=m.config.device_share)) for i, m in
                 zip(shard.mine, shard.members)]
        try:
            shard.initialize()
            for t in twins:
                t.initialize()
                t.set_initial_mass(t.compute_mass("c"))
            for step in range(2):
                reps = shard.step(step)
                for k, t in enumerate(twins):
                    assert reps[k] == t.step(step), (rank, k, step)
            for k, t in enumerate(twins):
                for name in ("c", "u", "v", "p"):
                    assert np.array_equal(shard.members[k].get_field(name), t.get_field(name)), (rank, k, name)
        finally:
            shard.close()
            for t in twins:
                t.close()
