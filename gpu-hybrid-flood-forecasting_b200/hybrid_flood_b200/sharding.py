"""Ensemble members across GPUs: one process per GPU, no per-step collective.

Members of an ensemble are independent domains, so scaling out is a partition
of the member list: each rank builds a :class:`B200Ensemble` over its share and
advances it alone.  The only communication is after the run: per-member results
(final time, steps, FP64 ledger) are gathered into member order on every rank,
and timings are reduced as the maximum over ranks.

The partition is a longest-processing-time bin-pack on cell counts: members in
decreasing size go to the currently lightest rank (ties to the lower rank), so
the busiest rank carries at most the mean load plus the largest member.
"""

from __future__ import annotations

from collections.abc import Callable, Sequence

import torch
import torch.distributed as dist


def shard_members(cells: Sequence[int], world: int) -> list[list[int]]:
    """Member indices per rank (each list ascending), balanced by cell count."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(cells)), key=lambda i: (-int(cells[i]), i))
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += int(cells[i])
    return [sorted(s) for s in out]


def shard_loads(cells: Sequence[int], shards: list[list[int]]) -> list[int]:
    return [sum(int(cells[i]) for i in s) for s in shards]


def _group_device(group=None) -> torch.device:
    backend = dist.get_backend(group)
    if backend == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(value: float, group=None) -> float:
    """The largest ``value`` over all ranks (every rank gets it)."""
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_group_device(group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_member_results(local: dict, n_members: int, group=None) -> list:
    """Combine ``{member_index: result}`` from every rank into one list in member order.

    Every member must be reported by exactly one rank; raises ``RuntimeError`` otherwise.
    """
    if dist.is_available() and dist.is_initialized():
        parts: list = [None] * dist.get_world_size(group)
        dist.all_gather_object(parts, dict(local), group=group)
    else:
        parts = [dict(local)]
    merged: dict = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise RuntimeError(f"member {k} reported by two ranks")
            merged[int(k)] = v
    missing = [i for i in range(n_members) if i not in merged]
    if missing:
        raise RuntimeError(f"members {missing} were reported by no rank")
    return [merged[i] for i in range(n_members)]


def run_sharded(cells: Sequence[int], advance: Callable[[list[int]], dict], rank: int, world: int,
                group=None) -> tuple[list, list[int]]:
    """Advance this rank's share with ``advance(indices) -> {index: result}`` and gather.

    Returns ``(results in member order, this rank's indices)``.
    """
    mine = shard_members(cells, world)[rank]
    local = advance(mine) if mine else {}
    return gather_member_results(local, len(cells), group), mine
