"""Differentiable rollouts: the hand-written adjoint behind ``torch.autograd``.

The reference never differentiates its solver.  This module adds what the
hybrid training needs: gradients of a loss on gauge depths with respect to
the Manning-n field, the initial depth and a scalar rain scale, through a
sequence of fixed-dt steps of
``src/hybrid_flood/numpy_solver/shallow_water_2d.py:277-327``.

dt is held fixed (a stop-gradient).  The forward pass keeps one state per
``checkpoint_every`` steps.  The backward pass walks the segments in reverse:
it recomputes a segment's states from its checkpoint and applies the
hand-written reverse step (``swe_adjoint_step``, two sm_100a kernels) to each
of them, injecting the gauge-loss gradient at each observation step.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .solver import SWEState, _ptr, _stream


def set_manning(solver, manning_n) -> None:
    """Replace the solver's Manning-n field (the domain mask is kept)."""
    n = torch.as_tensor(manning_n, dtype=torch.float32, device=solver.device).contiguous()
    if tuple(n.shape) != solver.shape:
        raise ValueError(f"Manning field must have shape {solver.shape}")
    with torch.cuda.device(solver.device):
        _lib.check(solver._lib.swe_domain_set_manning(solver._handle, _ptr(n), 0, _stream(solver.device)),
                   "set_manning")


def set_rain_scale(solver, scale: float) -> None:
    """Scale every hyetograph rate of the solver by ``scale``."""
    _lib.check(solver._lib.swe_domain_set_rain_scale(solver._handle, float(scale)), "set_rain_scale")


def adjoint_step(solver, state: SWEState, lam: SWEState, dt: float, time_s: float,
                 grad_n2: torch.Tensor, grad_rain: torch.Tensor) -> SWEState:
    """dL/dU_k from dL/dU_{k+1} for the step U_{k+1} = step(U_k, dt, time_s).

    Adds dL/d(n^2) into ``grad_n2`` ([rows, cols] float32) and dL/d(rain scale)
    into ``grad_rain`` (one float64 element).
    """
    out = [torch.empty(solver.shape, dtype=torch.float32, device=solver.device) for _ in range(3)]
    with torch.cuda.device(solver.device):
        rc = solver._lib.swe_adjoint_step(
            solver._handle, _ptr(state.h), _ptr(state.hu), _ptr(state.hv), int(state.h.stride(0)),
            _ptr(lam.h), _ptr(lam.hu), _ptr(lam.hv), int(lam.h.stride(0)),
            _ptr(out[0]), _ptr(out[1]), _ptr(out[2]), int(out[0].stride(0)),
            _ptr(grad_n2), _ptr(grad_rain), float(dt), float(time_s), _stream(solver.device))
    _lib.check(rc, "swe_adjoint_step")
    return SWEState(*out)


class SWEStepFunction(torch.autograd.Function):
    """One fixed-dt step ``finite_volume_step(state, params, dt, time_s)``
    (``src/hybrid_flood/jax_solver/numerics.py:312-369``) as an autograd node.

    forward(h, hu, hv, manning_n or None, solver, dt, time_s) -> (h', hu', hv').
    Backward is the hand-written reverse step: gradients for the state and, when
    ``manning_n`` is given, for the Manning field (dt is a stop-gradient).
    """

    @staticmethod
    def forward(ctx, h, hu, hv, manning_n, solver, dt, time_s):
        if manning_n is not None:
            set_manning(solver, manning_n.detach())
        state = SWEState(*(t.detach().to(torch.float32).contiguous() for t in (h, hu, hv)))
        out = solver.step(state, float(dt), float(time_s))
        ctx.solver = solver
        ctx.meta = (float(dt), float(time_s))
        ctx.save_for_backward(state.h, state.hu, state.hv, manning_n)
        return out.h, out.hu, out.hv

    @staticmethod
    def backward(ctx, gh, ghu, ghv):
        solver = ctx.solver
        h, hu, hv, manning_n = ctx.saved_tensors
        dt, t = ctx.meta
        if manning_n is not None:
            set_manning(solver, manning_n.detach())
        lam = SWEState(*(torch.zeros_like(h) if g is None else g.detach().to(torch.float32).contiguous()
                         for g in (gh, ghu, ghv)))
        gn2 = torch.zeros_like(h)
        gr = torch.zeros(1, dtype=torch.float64, device=h.device)
        out = adjoint_step(solver, SWEState(h, hu, hv), lam, dt, t, gn2, gr)
        grad_n = None
        if manning_n is not None and ctx.needs_input_grad[3]:
            grad_n = gn2 * 2.0 * manning_n.detach().to(torch.float32)
        return out.h, out.hu, out.hv, grad_n, None, None, None


def swe_step(solver, state, dt: float, time_s: float, manning_n=None) -> SWEState:
    """Differentiable :meth:`B200ShallowWaterSolver.step` (see :class:`SWEStepFunction`)."""
    return SWEState(*SWEStepFunction.apply(state[0], state[1], state[2], manning_n, solver, dt, time_s))


class GaugeRollout(torch.autograd.Function):
    """Gauge depths of a fixed-dt rollout, differentiable in (n, h0, rain scale).

    forward(manning_n [H,W], h0 [H,W], rain_scale [], solver, hu0, hv0, n_steps,
            dt, gauge_index (flat cell indices), obs_every, checkpoint_every,
            start_time_s) -> depths [n_steps // obs_every, n_gauges]

    Both passes run as native loops (``swe_rollout_forward`` /
    ``swe_rollout_backward``): no Python work per step.
    """

    @staticmethod
    def forward(ctx, manning_n, h0, rain_scale, solver, hu0, hv0, n_steps, dt, gauge_index,
                obs_every, checkpoint_every, start_time_s):
        set_manning(solver, manning_n.detach())
        set_rain_scale(solver, float(rain_scale))
        dev = solver.device
        H, W = solver.shape
        state = [t.detach().to(device=dev, dtype=torch.float32).contiguous().clone() for t in (h0, hu0, hv0)]
        n_obs = n_steps // obs_every
        obs = torch.empty((n_obs, gauge_index.numel()), dtype=torch.float32, device=dev)
        n_ckpt = (n_steps + checkpoint_every - 1) // checkpoint_every
        ckpt = torch.empty((max(n_ckpt, 1), 3, H, W), dtype=torch.float32, device=dev)
        with torch.cuda.device(dev):
            rc = solver._lib.swe_rollout_forward(
                solver._handle, _ptr(state[0]), _ptr(state[1]), _ptr(state[2]), W, int(n_steps), float(dt),
                float(start_time_s), None, _ptr(gauge_index), int(gauge_index.numel()), int(obs_every), _ptr(obs),
                _ptr(ckpt), int(checkpoint_every), _stream(dev))
        _lib.check(rc, "swe_rollout_forward")
        ctx.solver = solver
        ctx.meta = (int(n_steps), float(dt), int(obs_every), int(checkpoint_every), float(start_time_s))
        ctx.save_for_backward(manning_n, gauge_index, ckpt)
        return obs

    @staticmethod
    def backward(ctx, grad_obs):
        solver = ctx.solver
        manning_n, gauge_index, ckpt = ctx.saved_tensors
        n_steps, dt, obs_every, ckpt_every, t0 = ctx.meta
        dev = solver.device
        H, W = solver.shape
        lam = [torch.empty((H, W), dtype=torch.float32, device=dev) for _ in range(3)]
        grad_n2 = torch.zeros((H, W), dtype=torch.float32, device=dev)
        grad_rain = torch.zeros(1, dtype=torch.float64, device=dev)
        seg = torch.empty((ckpt_every, 3, H, W), dtype=torch.float32, device=dev)
        g = grad_obs.detach().to(torch.float32).contiguous()
        with torch.cuda.device(dev):
            rc = solver._lib.swe_rollout_backward(
                solver._handle, _ptr(ckpt), ckpt_every, n_steps, dt, t0, None, _ptr(gauge_index),
                int(gauge_index.numel()), obs_every, _ptr(g), _ptr(lam[0]), _ptr(lam[1]), _ptr(lam[2]), W, 0,
                _ptr(grad_n2), _ptr(grad_rain), _ptr(seg), _stream(dev))
        _lib.check(rc, "swe_rollout_backward")
        grad_n = grad_n2 * 2.0 * manning_n.detach().to(torch.float32)
        return grad_n, lam[0], grad_rain[0].to(torch.float32), None, None, None, None, None, None, None, None, None


def gauge_rollout(solver, manning_n, h0, rain_scale, *, hu0=None, hv0=None, n_steps: int, dt: float,
                  gauge_index, obs_every: int = 10, checkpoint_every: int = 50, start_time_s: float = 0.0):
    """Differentiable gauge depths (see :class:`GaugeRollout`)."""
    hu0 = torch.zeros_like(h0) if hu0 is None else hu0
    hv0 = torch.zeros_like(h0) if hv0 is None else hv0
    if not torch.is_tensor(rain_scale):
        rain_scale = torch.tensor(float(rain_scale), device=h0.device)
    gauge_index = torch.as_tensor(gauge_index, dtype=torch.long, device=h0.device)
    return GaugeRollout.apply(manning_n, h0, rain_scale, solver, hu0, hv0, int(n_steps), float(dt),
                              gauge_index, int(obs_every), int(checkpoint_every), float(start_time_s))
