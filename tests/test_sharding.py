"""Ensemble sharding across ranks: partition, gather and max-over-ranks timing,
on CPU with world_size-2 ``gloo`` process groups (the GPU ranks use NCCL)."""

from __future__ import annotations

import datetime
import json
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _cells():
    rng = np.random.default_rng(0)
    sizes = [256 * 256, 512 * 512, 1024 * 1024, 768 * 1536]
    return [sizes[int(i)] for i in rng.integers(0, 4, size=64)]


def test_shard_members_partition_and_balance():
    from hybrid_flood_b200.sharding import shard_loads, shard_members

    cells = _cells()
    for world in (1, 2, 3, 4, 8):
        shards = shard_members(cells, world)
        assert len(shards) == world
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(cells)))
        loads = shard_loads(cells, shards)
        assert max(loads) <= sum(cells) / world + max(cells)
        assert shards == shard_members(cells, world)  # deterministic
    assert shard_members([5, 5], 4) == [[0], [1], [], []]
    with pytest.raises(ValueError):
        shard_members(cells, 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir, drop):
    from hybrid_flood_b200.sharding import max_over_ranks, run_sharded

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        cells = _cells()

        def advance(idx):
            res = {i: {"rank": rank, "steps": 10 + i, "ledger": cells[i] * 0.5} for i in idx}
            if drop and rank == 1 and idx:
                res.pop(idx[0])
            return res

        try:
            results, mine = run_sharded(cells, advance, rank, world)
            err = None
        except RuntimeError as e:
            results, mine, err = None, [], str(e)
        ms = max_over_ranks(1.5 + rank)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"results": results, "mine": mine, "ms": ms, "err": err}, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("drop", [False, True])
def test_gloo_world2_gather_and_max(tmp_path, drop):
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path), drop), nprocs=world, join=True)
    outs = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    cells = _cells()
    for o in outs:
        assert o["ms"] == 2.5
    if drop:
        assert all(o["err"] and "reported by no rank" in o["err"] for o in outs)
        return
    assert outs[0]["results"] == outs[1]["results"]
    res = outs[0]["results"]
    assert [r["steps"] for r in res] == [10 + i for i in range(len(cells))]
    owner = {i: r for r, o in enumerate(outs) for i in o["mine"]}
    assert all(res[i]["rank"] == owner[i] for i in range(len(cells)))
    assert sorted(owner) == list(range(len(cells)))
