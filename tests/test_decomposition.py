"""Row-strip decomposition of one domain: layout on CPU, and the full algorithm
(strip steps, CFL maximum over ranks, halo exchange) with world_size-2 and -3
``gloo`` process groups stepping the C oracle per strip, against the undivided
oracle run -- bit for bit, since every owned cell sees the same neighbours and
every strip the same dt."""

from __future__ import annotations

import datetime
import json
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def test_row_ranges_and_local_rows():
    from hybrid_flood_b200.decomposition import local_rows, row_ranges

    for rows in (1, 2, 7, 64, 1000):
        for parts in range(1, min(rows, 9) + 1):
            r = row_ranges(rows, parts)
            assert r[0][0] == 0 and r[-1][1] == rows
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [hi - lo for lo, hi in r]
            assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
    assert local_rows(10, 0, 4) == (0, 5) and local_rows(10, 4, 7) == (3, 8) and local_rows(10, 7, 10) == (6, 10)
    with pytest.raises(ValueError):
        row_ranges(3, 4)


def _case():
    from hybrid_flood_b200.workloads import tilted_bumps
    from oracle import swe_numpy as O

    w = tilted_bumps(23, 37, seed=4)
    mask = np.ones(w.shape, bool)
    mask[9:12, 10:20] = False  # an inactive block across a strip boundary for 2 and 3 strips
    kw = w.solver_kwargs()
    kw["boundary"] = (0, 1, 1, 0)  # open east and south edges
    p = O.make_params(w.bed, w.manning_n, mask, **kw)
    rng = np.random.default_rng(1)
    h = np.where(mask, np.maximum(1.2 - w.bed, 0.0) + rng.uniform(0, 0.05, w.shape), 0).astype(np.float32)
    hu = np.where(mask, rng.normal(0, 0.05, w.shape), 0).astype(np.float32)
    hv = np.where(mask, rng.normal(0, 0.05, w.shape), 0).astype(np.float32)
    return p, (h, hu, hv)


def _strip_params(p, a, b):
    from oracle import swe_numpy as O

    return O.Params(**{**p.__dict__, "bed": p.bed[a:b], "manning_n": p.manning_n[a:b],
                       "domain_mask": p.domain_mask[a:b], "rainfall_multiplier": p.rainfall_multiplier[a:b]})


STEPS = 25


def _worker(rank, world, port, out_dir):
    from hybrid_flood_b200.decomposition import local_rows, row_ranges
    from oracle import cport
    from oracle import swe_numpy as O

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        p, state = _case()
        rows = p.bed.shape[0]
        lo, hi = row_ranges(rows, world)[rank]
        a, b = local_rows(rows, lo, hi)
        dom = cport.Domain(_strip_params(p, a, b))
        st = O.State(*(x[a:b].copy() for x in state))
        below = rank - 1 if lo > 0 else -1
        above = rank + 1 if hi < rows else -1
        t, dts = 0.0, []
        for _ in range(STEPS):
            m = torch.tensor([dom.max_inverse_dt(st)], dtype=torch.float32)
            dist.all_reduce(m, op=dist.ReduceOp.MAX)
            maximum = float(m.item())
            dt = min(p.cfl / maximum, p.max_dt) if maximum > 0.0 else p.max_dt
            st = dom.step(st, dt, t)
            t += dt
            dts.append(dt)
            fields = [np.array(x) for x in st]
            reqs = []
            recv_lo = [torch.empty(fields[0].shape[1]) for _ in range(3)]
            recv_hi = [torch.empty(fields[0].shape[1]) for _ in range(3)]
            for q in range(3):
                if below >= 0:
                    reqs.append(dist.isend(torch.from_numpy(fields[q][lo - a].copy()), below))
                    reqs.append(dist.irecv(recv_lo[q], below))
                if above >= 0:
                    reqs.append(dist.isend(torch.from_numpy(fields[q][hi - 1 - a].copy()), above))
                    reqs.append(dist.irecv(recv_hi[q], above))
            for r in reqs:
                r.wait()
            for q in range(3):
                if below >= 0:
                    fields[q][0] = recv_lo[q].numpy()
                if above >= 0:
                    fields[q][-1] = recv_hi[q].numpy()
            st = O.State(*fields)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), h=st.h[lo - a:hi - a], hu=st.hu[lo - a:hi - a],
                 hv=st.hv[lo - a:hi - a], dts=np.array(dts))
    finally:
        dist.destroy_process_group()


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_strips_equal_the_undivided_oracle(tmp_path, world):
    from oracle import cport
    from oracle import swe_numpy as O

    mp.spawn(_worker, args=(world, _port(), str(tmp_path)), nprocs=world, join=True)
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    p, state = _case()
    dom = cport.Domain(p)
    st, t, dts = O.State(*state), 0.0, []
    for _ in range(STEPS):
        dt = dom.cfl_dt(st)
        st = dom.step(st, dt, t)
        t += dt
        dts.append(dt)
    for r in range(world):
        np.testing.assert_array_equal(parts[r]["dts"], np.array(dts))
    for q, name in enumerate(("h", "hu", "hv")):
        np.testing.assert_array_equal(np.concatenate([x[name] for x in parts]), st[q])


def _agree_worker(rank, world, port, out_dir, failing):
    from hybrid_flood_b200.decomposition import agree_on_errors

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    try:
        err = ValueError(f"rank {rank}: bad strip state") if rank in failing else None
        try:
            agree_on_errors(err, world)
            outcome = "ok"
        except ValueError as e:
            outcome = str(e)
        # every rank is still in step: one more collective completes
        t = torch.ones(1)
        dist.all_reduce(t)
        with open(os.path.join(out_dir, f"agree{rank}.json"), "w") as f:
            json.dump({"outcome": outcome, "after": float(t.item())}, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("failing", [(), (1,), (0, 2)])
def test_ranks_agree_before_the_collective_steps(tmp_path, failing):
    """A rank whose argument check fails does not leave the others waiting in
    NCCL: every rank learns of the failure from one all-reduce and raises, and
    all ranks stay in step for the next collective."""
    world = 3
    mp.spawn(_agree_worker, args=(world, _port(), str(tmp_path), failing), nprocs=world, join=True)
    out = [json.loads((tmp_path / f"agree{r}.json").read_text()) for r in range(world)]
    for r, o in enumerate(out):
        assert o["after"] == world
        if not failing:
            assert o["outcome"] == "ok"
        elif r in failing:
            assert o["outcome"] == f"rank {r}: bad strip state"
        else:
            assert o["outcome"] == "another rank's strip arguments are invalid"
