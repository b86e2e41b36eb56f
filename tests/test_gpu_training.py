"""Training through the solver (GPU): the interval autograd nodes against float64
central differences of the oracle replaying the same dts, the torch restatements
of features/correction against the kernels, and a few optimiser steps.

dt is a stop-gradient: the finite differences replay the logged dt sequence, so
they measure the same derivative.  Tolerance 2e-3 relative over ~10 steps (the
reverse step runs in float32)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import max_ulp
from oracle import cport
from oracle import swe_numpy as O

pytestmark = pytest.mark.gpu


def _member(rows, cols, seed):
    from hybrid_flood_b200.workloads import as_member, tilted_bumps

    w = tilted_bumps(rows, cols, seed=seed)
    m = as_member(w)
    rng = np.random.default_rng(seed)
    m["manning_n"] = rng.uniform(0.02, 0.05, w.shape).astype(np.float32)
    m["cfl"] = 0.9
    depth = np.maximum(1.6 - w.bed, 0.3).astype(np.float32)
    hu = (0.3 * depth).astype(np.float32)
    hv = (rng.normal(0, 0.02, w.shape) * depth).astype(np.float32)
    return m, (depth, hu, hv)


def _solver(m, arith="exact"):
    from hybrid_flood_b200.solver import B200ShallowWaterSolver

    kw = {k: v for k, v in m.items() if k not in ("bed", "manning_n", "domain_mask")}
    return B200ShallowWaterSolver(m["bed"], m["manning_n"], m["domain_mask"], **kw, arithmetic=arith)


def _replay64(m, state, dts, t0):
    kw = {k: v for k, v in m.items() if k not in ("bed", "manning_n", "domain_mask")}
    p = O.make_params(m["bed"], m["manning_n"], m["domain_mask"], dtype=np.float64, **kw)
    d = cport.Domain(p)
    st = O.State(*[np.asarray(a, np.float64) for a in state])
    t = t0
    for dt in dts:
        st = d.step(st, float(dt), t)
        t += float(dt)
    return st


def test_physics_interval_gradient_matches_replayed_differences(cuda_device):
    from hybrid_flood_b200.training import PhysicsInterval

    m, state = _member(24, 40, 3)
    s = _solver(m)
    x = [torch.tensor(a, device=cuda_device, requires_grad=True) for a in state]
    h, hu, hv, n = PhysicsInterval.apply(*x, s, 10.0, 13.0, 100)
    n = int(n)
    assert n > 3
    rng = np.random.default_rng(1)
    wts = [rng.normal(0, 1, m["bed"].shape) for _ in range(3)]
    loss = sum((o * torch.tensor(w, dtype=torch.float32, device=cuda_device)).sum() for o, w in zip((h, hu, hv), wts))
    loss.backward()
    # the logged dts, read back from a second forward
    log = torch.empty(100, dtype=torch.float64, device=cuda_device)
    from hybrid_flood_b200.solver import SWEState

    st = SWEState(*(torch.tensor(a, device=cuda_device) for a in state))
    t_end, n2, _ = s.advance_to_(st, 10.0, 13.0, 100, dt_log=log)
    assert n2 == n and abs(t_end - 13.0) < 1e-7
    dts = log[:n].cpu().numpy()
    assert abs(10.0 + dts.sum() - 13.0) < 1e-9

    def J(U):
        out = _replay64(m, U, dts, 10.0)
        return sum(float((a * w).sum()) for a, w in zip(out, wts))

    U = [a.astype(np.float64) for a in state]
    dU = [rng.normal(0, 1, m["bed"].shape) * 1e-3 for _ in range(3)]
    eps = 1e-6
    fd = (J([a + eps * b for a, b in zip(U, dU)]) - J([a - eps * b for a, b in zip(U, dU)])) / (2 * eps)
    ad = sum(float((g.grad.cpu().numpy().astype(np.float64) * d).sum()) for g, d in zip(x, dU))
    assert ad == pytest.approx(fd, rel=2e-3)


def test_ensemble_interval_gradients_equal_single_domain(cuda_device):
    from hybrid_flood_b200.ensemble import B200Ensemble
    from hybrid_flood_b200.training import EnsembleInterval, PhysicsInterval

    mems = [_member(24, 40, 5), _member(24, 40, 6)]
    ens = B200Ensemble([m for m, _ in mems], arithmetic="exact")
    flat = [torch.tensor(a, device=cuda_device, requires_grad=True) for _, st in mems for a in st]
    out = EnsembleInterval.apply(ens, 0.0, 4.0, 200, *flat)
    rng = np.random.default_rng(2)
    wts = [torch.tensor(rng.normal(0, 1, (24, 40)), dtype=torch.float32, device=cuda_device) for _ in range(6)]
    sum((o * w).sum() for o, w in zip(out[:6], wts)).backward()
    for i, (m, st) in enumerate(mems):
        s = _solver(m)
        x = [torch.tensor(a, device=cuda_device, requires_grad=True) for a in st]
        h, hu, hv, n = PhysicsInterval.apply(*x, s, 0.0, 4.0, 200)
        assert int(n) == int(out[-1][i])
        sum((o * w).sum() for o, w in zip((h, hu, hv), wts[3 * i:3 * i + 3])).backward()
        for a, b in zip(x, flat[3 * i:3 * i + 3]):
            assert torch.equal(a.grad, b.grad)


def test_torch_features_and_correction_match_kernels(cuda_device):
    from hybrid_flood_b200.hybrid import HybridInputs, apply_residual_correction, network_features, rain_feature
    from hybrid_flood_b200.solver import SWEState
    from hybrid_flood_b200.training import correction_torch, features_torch

    m, state = _member(32, 48, 7)
    m["domain_mask"] = m["domain_mask"].copy()
    m["domain_mask"][5:9, 10:20] = False
    s = _solver(m, "fast")
    st = SWEState(*(torch.tensor(np.where(m["domain_mask"], a, 0), dtype=torch.float32, device=cuda_device)
                    for a in state))
    mask = torch.tensor(m["domain_mask"], device=cuda_device)
    bed = torch.tensor(m["bed"], device=cuda_device)
    hi = HybridInputs(None, None, [0.5, 0.1, 0.0, 1.0, 2.0], [0.3, 0.2, 0.1, 2.0, 3.0], 25.0, [0.01])
    k = network_features(s, st, hi, 100.0, layout="state5")[0].permute(2, 0, 1)
    from hybrid_flood_b200.hybrid import _domain

    t = features_torch(st, mask, bed, hi, rain_feature(_domain(s), hi, 100.0, "state5"), "state5",
                       s.params.dry_tolerance)
    assert torch.equal(k, t)
    res = torch.tensor(np.random.default_rng(3).normal(0, 0.05, (1, 32, 48)), dtype=torch.float32,
                       device=cuda_device)
    kc = apply_residual_correction(s, st, res.permute(1, 2, 0), correction_relaxation=0.5, clip_limits=[0.06])
    tc = correction_torch(st, res, mask, s.params.dry_tolerance, 0.5, [0.06])
    for a, b in zip(kc, tc):
        assert max_ulp(a.cpu().numpy(), b.detach().cpu().numpy()) <= 2


def test_train_steps_reduce_loss_against_refined_targets(cuda_device):
    from hybrid_flood_b200.ensemble import B200Ensemble
    from hybrid_flood_b200.hybrid import HybridInputs
    from hybrid_flood_b200.training import refined_targets, train_step
    from hybrid_flood_b200.unet import ResidualUNet
    from hybrid_flood_b200.workloads import as_member, street_depth, urban

    members, states, targets = [], [], []
    times = np.array([0.0, 20.0, 40.0])
    for sd in (11, 12):
        w = urban(32, 32, seed=sd, duration_s=3600.0, rain_scale=20.0)
        mem = as_member(w)
        d0 = street_depth(w, 0.05)
        members.append(mem)
        states.append((d0, np.zeros_like(d0), np.zeros_like(d0)))
        targets.append(refined_targets(mem, d0, times, device=cuda_device))
    ens = B200Ensemble(members, arithmetic="fast")
    hi = HybridInputs(None, None, [0.05, 0.0, 0.0, 5.0, 10.0], [0.05, 0.02, 0.02, 5.0, 10.0], 25.0, [0.01])
    torch.manual_seed(0)
    net = ResidualUNet(input_channels=5, depth=2, channels=(8, 16), output_channels=1).to(cuda_device)
    opt = torch.optim.Adam(net.parameters(), lr=3e-3)
    kw = dict(max_substeps_per_interval=2000, correction_relaxation=0.5)
    losses = []
    for _ in range(6):
        loss, steps = train_step(ens, states, net, opt, hi, times, targets, **kw)
        losses.append(loss)
    assert all(np.isfinite(losses)) and int(steps.min()) > 0
    assert all(p.grad is not None and bool(torch.isfinite(p.grad).all()) for p in net.parameters())
    assert float(net.residual_head.weight.grad.abs().sum()) > 0
    assert min(losses[1:]) < losses[0]
