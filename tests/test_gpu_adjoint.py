"""The hand-written adjoint against float64 finite differences of the oracle (GPU).

The reference has no gradients, so the oracle is the float64 C restatement of
the step: central differences (relative step 1e-6) of its outputs / of a gauge
loss.  States are kept wet (no wet/dry fronts) so the step is smooth there.

Tolerances: the adjoint runs in float32, so a directional derivative agrees
with the float64 difference quotient to ~1e-4 relative per step; a 60-step
rollout gradient to 1e-2 relative (the float32 forward trajectory itself moves
the linearisation point).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import cport
from oracle import gauge_loss as GL
from oracle import swe_numpy as O

pytestmark = pytest.mark.gpu


def _case(rows, cols, bnd, masked, seed):
    from hybrid_flood_b200.workloads import tilted_bumps

    w = tilted_bumps(rows, cols, seed=seed)
    rng = np.random.default_rng(seed)
    mask = np.ones(w.shape, bool)
    if masked:
        mask[rows // 3: rows // 3 + 4, cols // 2: cols // 2 + 5] = False
    n = rng.uniform(0.02, 0.05, w.shape).astype(np.float32)
    kw = w.solver_kwargs()
    kw["boundary"] = bnd
    depth = np.maximum(1.6 - w.bed, 0.3).astype(np.float32)
    u = rng.normal(0.0, 0.05, w.shape).astype(np.float32)
    v = rng.normal(0.0, 0.05, w.shape).astype(np.float32)
    return w, mask, n, kw, depth, u, v


def _f64_step(w, mask, n, kw, state, dt, t, rain_scale=1.0):
    kw = dict(kw)
    kw["rainfall_rates_m_s"] = np.asarray(kw["rainfall_rates_m_s"], np.float64) * rain_scale
    p = O.make_params(w.bed, n, mask, dtype=np.float64, **kw)
    return cport.Domain(p).step(O.State(*[np.asarray(a, np.float64) for a in state]), dt, t)


@pytest.mark.parametrize("bnd,masked", [((0, 0, 0, 0), False), ((0, 1, 0, 0), True), ((1, 1, 1, 1), True)])
def test_adjoint_step_dot_product(cuda_device, bnd, masked):
    from hybrid_flood_b200.adjoint import adjoint_step, set_manning
    from hybrid_flood_b200.solver import B200ShallowWaterSolver, SWEState

    w, mask, n, kw, depth, u, v = _case(24, 40, bnd, masked, seed=3)
    s = B200ShallowWaterSolver(w.bed, n, mask, **kw)
    st = s.initial_state(depth_m=depth, x_velocity_m_s=u, y_velocity_m_s=v)
    U = [a.cpu().numpy().astype(np.float64) for a in st]
    rng = np.random.default_rng(11)
    lam = [rng.normal(0, 1, w.shape) for _ in range(3)]
    lam = [np.where(mask, a, 0.0) for a in lam]
    dt, t = 0.2, 30.0
    gn2 = torch.zeros(w.shape, device=cuda_device)
    gr = torch.zeros(1, dtype=torch.float64, device=cuda_device)
    lam_t = SWEState(*(torch.tensor(a, dtype=torch.float32, device=cuda_device) for a in lam))
    set_manning(s, n)
    out = adjoint_step(s, st, lam_t, dt, t, gn2, gr)
    got = [a.cpu().numpy().astype(np.float64) for a in out]

    def J(state, nn=n, scale=1.0):
        o = _f64_step(w, mask, nn, kw, state, dt, t, scale)
        return sum(float((a * b).sum()) for a, b in zip(lam, o))

    # state direction
    dU = [np.where(mask, rng.normal(0, 1, w.shape), 0.0) * sc for sc in (1e-3, 1e-3, 1e-3)]
    eps = 1e-6
    plus = [a + eps * b for a, b in zip(U, dU)]
    minus = [a - eps * b for a, b in zip(U, dU)]
    fd = (J(plus) - J(minus)) / (2 * eps)
    ad = sum(float((a * b).sum()) for a, b in zip(got, dU))
    assert ad == pytest.approx(fd, rel=2e-4, abs=1e-9)
    # Manning-n direction (gradient is returned for n^2)
    dn = rng.normal(0, 1, w.shape) * 1e-3
    n64 = n.astype(np.float64)
    fd_n = (J(U, n64 + eps * dn) - J(U, n64 - eps * dn)) / (2 * eps)
    ad_n = float((gn2.cpu().numpy().astype(np.float64) * 2.0 * n64 * dn).sum())
    assert ad_n == pytest.approx(fd_n, rel=2e-3, abs=1e-12)
    # rain scale
    fd_s = (J(U, n64, 1.0 + eps) - J(U, n64, 1.0 - eps)) / (2 * eps)
    assert float(gr.item()) == pytest.approx(fd_s, rel=1e-3, abs=1e-12)


def test_rollout_gradient_matches_finite_differences(cuda_device):
    from hybrid_flood_b200.adjoint import gauge_rollout
    from hybrid_flood_b200.solver import B200ShallowWaterSolver

    w, mask, n, kw, _, _, _ = _case(48, 64, (0, 1, 0, 0), False, seed=5)
    # A flowing start: a tilted free surface and a uniform current.
    yy, xx = np.mgrid[0:48, 0:64]
    depth = np.maximum(1.6 + 0.004 * xx - 0.002 * yy - w.bed, 0.3).astype(np.float32)
    hu0 = (0.4 * depth).astype(np.float32)
    hv0 = (-0.1 * depth).astype(np.float32)
    n_truth = (n * 1.3).astype(np.float32)
    rng = np.random.default_rng(2)
    gauges = rng.choice(48 * 64, size=6, replace=False)
    steps, dt, every = 60, 0.2, 10
    obs = GL.rollout_gauges(w.bed, n_truth, mask, kw, depth, steps, dt, gauges, every, hu0=hu0, hv0=hv0)
    s = B200ShallowWaterSolver(w.bed, n, mask, **kw)
    dev = cuda_device
    n_t = torch.tensor(n, device=dev, requires_grad=True)
    h0_t = torch.tensor(depth, device=dev, requires_grad=True)
    s_t = torch.tensor(1.0, device=dev, requires_grad=True)
    pred = gauge_rollout(s, n_t, h0_t, s_t, hu0=torch.tensor(hu0, device=dev), hv0=torch.tensor(hv0, device=dev),
                         n_steps=steps, dt=dt, gauge_index=gauges, obs_every=every, checkpoint_every=25)
    loss = torch.mean((pred - torch.tensor(obs, dtype=torch.float32, device=dev)) ** 2)
    loss.backward()
    want_loss = GL.gauge_mse(GL.rollout_gauges(w.bed, n, mask, kw, depth, steps, dt, gauges, every,
                                               hu0=hu0, hv0=hv0), obs)
    assert want_loss > 1e-8  # the case is not degenerate
    assert float(loss.detach()) == pytest.approx(want_loss, rel=1e-3)

    def L(nn=n.astype(np.float64), h0=depth.astype(np.float64), scale=1.0):
        return GL.gauge_mse(GL.rollout_gauges(w.bed, nn, mask, kw, h0, steps, dt, gauges, every, scale,
                                              hu0=hu0, hv0=hv0), obs)

    eps = 1e-6
    dn = rng.normal(0, 1, n.shape) * 1e-3
    fd = (L(nn=n + eps * dn) - L(nn=n - eps * dn)) / (2 * eps)
    ad = float((n_t.grad.cpu().numpy().astype(np.float64) * dn).sum())
    assert ad == pytest.approx(fd, rel=1e-2)
    dh = rng.normal(0, 1, n.shape) * 1e-2
    fd = (L(h0=depth + eps * dh) - L(h0=depth - eps * dh)) / (2 * eps)
    ad = float((h0_t.grad.cpu().numpy().astype(np.float64) * dh).sum())
    assert ad == pytest.approx(fd, rel=1e-2)
    fd = (L(scale=1.0 + eps) - L(scale=1.0 - eps)) / (2 * eps)
    assert float(s_t.grad) == pytest.approx(fd, rel=1e-2)


def test_step_function_autograd_chain_matches_finite_differences(cuda_device):
    """Two chained autograd steps (state and Manning-n gradients) against float64
    central differences of the oracle."""
    from hybrid_flood_b200.adjoint import swe_step
    from hybrid_flood_b200.solver import B200ShallowWaterSolver

    w, mask, n, kw, depth, u, v = _case(24, 40, (0, 1, 0, 0), True, seed=7)
    s = B200ShallowWaterSolver(w.bed, n, mask, **kw)
    st0 = s.initial_state(depth_m=depth, x_velocity_m_s=u, y_velocity_m_s=v)
    U = [a.cpu().numpy().astype(np.float64) for a in st0]
    rng = np.random.default_rng(4)
    wts = [np.where(mask, rng.normal(0, 1, w.shape), 0.0) for _ in range(3)]
    dt, t = 0.15, 12.0
    x = [a.clone().requires_grad_(True) for a in st0]
    n_t = torch.tensor(n, device=cuda_device, requires_grad=True)
    mid = swe_step(s, x, dt, t, manning_n=n_t)
    out = swe_step(s, mid, dt, t + dt, manning_n=n_t)
    loss = sum((o * torch.tensor(wt, dtype=torch.float32, device=cuda_device)).sum() for o, wt in zip(out, wts))
    loss.backward()

    def J(state, nn=n.astype(np.float64)):
        a = _f64_step(w, mask, nn, kw, state, dt, t)
        b = _f64_step(w, mask, nn, kw, a, dt, t + dt)
        return sum(float((p * q).sum()) for p, q in zip(wts, b))

    eps = 1e-6
    dU = [np.where(mask, rng.normal(0, 1, w.shape), 0.0) * 1e-3 for _ in range(3)]
    fd = (J([a + eps * b for a, b in zip(U, dU)]) - J([a - eps * b for a, b in zip(U, dU)])) / (2 * eps)
    ad = sum(float((g.grad.cpu().numpy().astype(np.float64) * d).sum()) for g, d in zip(x, dU))
    assert ad == pytest.approx(fd, rel=5e-4, abs=1e-9)
    dn = rng.normal(0, 1, w.shape) * 1e-3
    n64 = n.astype(np.float64)
    fd_n = (J(U, n64 + eps * dn) - J(U, n64 - eps * dn)) / (2 * eps)
    ad_n = float((n_t.grad.cpu().numpy().astype(np.float64) * dn).sum())
    assert ad_n == pytest.approx(fd_n, rel=5e-3, abs=1e-12)


def test_rollout_backward_matches_stepwise_reverse(cuda_device):
    """The rollout's reverse steps rebuild each cell update from the step's own output
    (or from the faces where strong friction makes that inexact); the standalone
    reverse step always rebuilds it from the faces.  Both must give the same
    gradients, here on a shallow, rough case where both branches occur."""
    from hybrid_flood_b200.adjoint import adjoint_step, set_manning
    from hybrid_flood_b200.solver import B200ShallowWaterSolver, SWEState, _ptr, _stream

    w, mask, n, kw, _, _, _ = _case(32, 48, (0, 1, 0, 0), True, seed=8)
    rng = np.random.default_rng(8)
    n = rng.uniform(0.03, 0.3, w.shape).astype(np.float32)
    depth = rng.uniform(0.002, 0.3, w.shape).astype(np.float32)
    s = B200ShallowWaterSolver(w.bed, n, mask, **kw)
    set_manning(s, n)
    st = s.initial_state(depth_m=depth, x_velocity_m_s=0.2, y_velocity_m_s=-0.1)
    steps, dt, t0, every = 12, 0.05, 5.0, 4
    H, W = w.shape
    dev = cuda_device
    # forward, keeping every state
    states = [SWEState(*(a.clone() for a in st))]
    for k in range(steps):
        states.append(s.step(states[-1], dt, t0 + k * dt))
    g_final = [torch.tensor(rng.normal(0, 1, w.shape), dtype=torch.float32, device=dev) for _ in range(3)]
    # stepwise reverse (faces recomputed in every reverse step)
    lam = SWEState(*(g.clone() for g in g_final))
    gn2_a = torch.zeros((H, W), device=dev)
    gr_a = torch.zeros(1, dtype=torch.float64, device=dev)
    t = [t0]
    for k in range(steps - 1):
        t.append(t[-1] + dt)
    for k in range(steps - 1, -1, -1):
        lam = adjoint_step(s, states[k], lam, dt, t[k], gn2_a, gr_a)
    # the rollout's reverse pass from one checkpoint, final-state gradient on entry
    ckpt = torch.stack(list(states[0]))[None].contiguous()
    seg = torch.empty((steps, 3, H, W), device=dev)
    lb = [g.clone() for g in g_final]
    gn2_b = torch.zeros((H, W), device=dev)
    gr_b = torch.zeros(1, dtype=torch.float64, device=dev)
    with torch.cuda.device(dev):
        rc = s._lib.swe_rollout_backward(s._handle, _ptr(ckpt), steps, steps, dt, t0, None, None, 0, 1, None,
                                         _ptr(lb[0]), _ptr(lb[1]), _ptr(lb[2]), W, 1, _ptr(gn2_b), _ptr(gr_b),
                                         _ptr(seg), _stream(dev))
    assert rc == 0
    for a, b in zip(lam, lb):
        a, b = a.cpu().numpy().astype(np.float64), b.cpu().numpy().astype(np.float64)
        assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(a)
    ga, gb = gn2_a.cpu().numpy().astype(np.float64), gn2_b.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(ga - gb) <= 1e-3 * np.linalg.norm(ga)


def test_gauge_loss_gradients_at_the_adjoint_configuration(cuda_device):
    """The adjoint configuration at full size: 512x512 (dx = 2 m), log-normal
    Manning n, 16 gauges every 10 steps, 2000 fixed 0.2 s steps, a checkpoint
    every 50 steps.  Directional derivatives of the gauge MSE in three random
    directions for the n field and for the initial depth, and the rain-scale
    derivative, against central differences of the float64 C oracle with a
    relative step of 1e-3.  The state stays wet (depth >= 0.2 m), away from
    wet/dry fronts.  Tolerance 5 % relative: a float32 forward and an adjoint on
    approximate division/square root over 2000 steps."""
    from hybrid_flood_b200.adjoint import gauge_rollout
    from hybrid_flood_b200.solver import B200ShallowWaterSolver
    from hybrid_flood_b200.workloads import adjoint_case

    w, n_truth, n_est, gauges = adjoint_case(512, 512)
    kw = w.solver_kwargs()
    depth = np.maximum(1.0 - w.bed, 0.2).astype(np.float32)
    steps, dt, every, ckpt = 2000, 0.2, 10, 50
    obs = GL.rollout_gauges(w.bed, n_truth, w.domain_mask, kw, depth, steps, dt, gauges, every)
    s = B200ShallowWaterSolver(w.bed, n_est, w.domain_mask, **kw, arithmetic="exact")
    dev = cuda_device
    n_t = torch.tensor(n_est, device=dev, requires_grad=True)
    h_t = torch.tensor(depth, device=dev, requires_grad=True)
    s_t = torch.tensor(1.0, device=dev, requires_grad=True)
    pred = gauge_rollout(s, n_t, h_t, s_t, n_steps=steps, dt=dt, gauge_index=gauges, obs_every=every,
                         checkpoint_every=ckpt)
    loss = torch.mean((pred - torch.tensor(obs, dtype=torch.float32, device=dev)) ** 2)
    loss.backward()
    gn, gh, gs = (n_t.grad.cpu().numpy().astype(np.float64), h_t.grad.cpu().numpy().astype(np.float64),
                  float(s_t.grad))

    def L(nn=n_est.astype(np.float64), h0=depth.astype(np.float64), scale=1.0):
        return GL.gauge_mse(GL.rollout_gauges(w.bed, nn, w.domain_mask, kw, h0, steps, dt, gauges, every, scale),
                            obs)

    assert float(loss.detach()) == pytest.approx(L(), rel=1e-2)
    eps = 1e-3
    rng = np.random.default_rng(21)
    rel = []
    for _ in range(3):
        v = rng.normal(0.0, 1.0, w.shape)
        dn = eps * n_est.astype(np.float64) * v  # relative step of the n field
        fd = (L(nn=n_est + dn) - L(nn=n_est - dn)) / 2.0
        ad = float((gn * dn).sum())
        rel.append(abs(ad - fd) / abs(fd))
        assert ad == pytest.approx(fd, rel=5e-2)
        dh = eps * depth.astype(np.float64) * rng.normal(0.0, 1.0, w.shape)  # relative step of h0
        fd = (L(h0=depth + dh) - L(h0=depth - dh)) / 2.0
        ad = float((gh * dh).sum())
        rel.append(abs(ad - fd) / abs(fd))
        assert ad == pytest.approx(fd, rel=5e-2)
    fd = (L(scale=1.0 + eps) - L(scale=1.0 - eps)) / (2.0 * eps)
    rel.append(abs(gs - fd) / abs(fd))
    assert gs == pytest.approx(fd, rel=5e-2)
    print(f"config-2 directional derivatives: max relative difference {max(rel):.3g}")
