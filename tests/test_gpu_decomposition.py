"""Row strips on the GPU: the strip kernels (owned-row updates, halo rows read as
neighbours), the CFL maximum over strips and the halo exchange reproduce the
undivided run, for all strips in one process and for one strip over NCCL (a
single-rank communicator: this pool gives one GPU per run).

Exact arithmetic: bit for bit.  Fast arithmetic: the march body is compiled
twice (two register rotations) and the compiler may contract multiply-adds
differently in the two copies, so a row stepped at the other parity of its chunk
can differ in the last bit; the strips then agree with the undivided run to
1e-6 relative L2 after 40 steps."""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _member(arith_rows=97, cols=130):
    from hybrid_flood_b200.workloads import as_member, urban

    w = urban(arith_rows, cols, seed=31, duration_s=3600.0, rain_scale=5.0)
    m = as_member(w)
    mask = np.asarray(m["domain_mask"]).copy()
    mask[40:47, 30:70] = False
    m["domain_mask"] = mask
    m["boundary"] = (0, 1, 1, 0)
    rng = np.random.default_rng(3)
    h = np.where(mask, rng.uniform(0.0, 0.2, mask.shape), 0.0).astype(np.float32)
    return m, h


def _single(m, h, arith, steps, device):
    from hybrid_flood_b200.solver import B200ShallowWaterSolver

    kw = {k: v for k, v in m.items() if k not in ("bed", "manning_n", "domain_mask")}
    s = B200ShallowWaterSolver(m["bed"], m["manning_n"], m["domain_mask"], **kw, arithmetic=arith, device=device)
    st = s.initial_state(depth_m=h, x_velocity_m_s=0.1)
    t, n, led = s.advance_(st, steps, 3.0)
    init = s.initial_state(depth_m=h, x_velocity_m_s=0.1)
    return init, st, t, n, led


@pytest.mark.parametrize("arith", ["fast", "exact"])
@pytest.mark.parametrize("parts", [1, 2, 3])
def test_strip_set_equals_the_undivided_run(cuda_device, arith, parts):
    from hybrid_flood_b200.decomposition import StripSet

    m, h = _member()
    init, want, t, n, led = _single(m, h, arith, 40, cuda_device)
    strips = StripSet(m, parts, arithmetic=arith, device=cuda_device)
    local = strips.split(init)
    res = strips.advance_(local, 40, 3.0)
    got = strips.join(local)
    for a, b in zip(got, want):
        if arith == "exact" or parts == 1:
            assert torch.equal(a, b)
        else:
            assert float((a.double() - b.double()).norm() / b.double().norm()) < 1e-6
    assert all(r[1] == n for r in res)
    assert all((r[0] == t) if arith == "exact" else r[0] == pytest.approx(t, rel=1e-6) for r in res)
    vol = sum(r[2]["volume"] for r in res)
    assert vol == pytest.approx(led["volume"], rel=1e-6)
    outflow = sum(r[2]["outflow"] for r in res)
    assert outflow == pytest.approx(led["outflow"], rel=1e-5, abs=1e-9)


def test_single_rank_nccl_strip_equals_the_undivided_run(cuda_device):
    from hybrid_flood_b200.decomposition import NcclStrip

    m, h = _member(64, 96)
    init, want, t, n, _ = _single(m, h, "fast", 30, cuda_device)
    strip = NcclStrip(m, rank=0, world=1, arithmetic="fast", device=cuda_device)
    local = strip.local_state(init)
    t1, n1, _ = strip.advance_(local, 30, 3.0)
    assert (t1, n1) == (t, n)
    for a, b in zip(local, want):
        assert torch.equal(a, b)
