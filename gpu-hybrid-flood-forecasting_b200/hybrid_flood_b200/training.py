"""Training the corrector through the solver.

The reference trains its residual U-Net offline on saved transitions
(``ml/train.py``) and never differentiates the solver.  Here the coupled
rollout of ``hybrid/coupled_forecast.py:164-225`` is differentiable end to end,
so a loss on corrected states at the correction times trains the corrector
through the physics that follows each correction:

* physics to the next correction time is a :class:`PhysicsInterval` (single
  domain) or :class:`EnsembleInterval` (all members in one batched advance)
  autograd node.  Forward: ``swe_advance_to`` / ``swe_ensemble_advance_to`` with
  the adaptive dts logged on the device.  Backward: the interval is replayed
  with the logged dts (dt is a stop-gradient) by ``swe_rollout_backward``: its
  states are recomputed into one device segment (or, past a memory budget,
  from sqrt-spaced checkpoints) and the hand-written reverse step runs back
  through them;
* features and the volume-preserving correction are restated in torch ops
  (:func:`features_torch`, :func:`correction_torch`) so autograd differentiates
  them, including the two global volume sums;
* the corrector runs under activation checkpointing, so one interval's
  activations are alive at a time.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch
import torch.nn.functional as F
from torch.utils.checkpoint import checkpoint

from . import _lib
from .hybrid import LAYOUTS, HybridInputs, _domain, _host_f32, ensemble_domains, rain_feature
from .solver import SWEState, _ptr, _stream

F32_EPS = float(np.finfo(np.float32).eps)
SEGMENT_BUDGET_BYTES = 8 << 30


def _replay_backward(dom, x0: SWEState, dts: np.ndarray, t0: float, grad_out: SWEState,
                     budget: int = SEGMENT_BUDGET_BYTES) -> SWEState:
    """dL/d(interval input) from dL/d(interval output) by replaying the logged dts."""
    n = int(dts.size)
    lam = [g.detach().to(torch.float32).contiguous().clone() for g in grad_out]
    if n == 0:
        return SWEState(*lam)
    H, W = dom.shape
    dev = dom.device
    plane = H * W
    seg_len = int(max(1, min(n, budget // (12 * plane))))
    dts = np.ascontiguousarray(dts, dtype=np.float64)
    if seg_len >= n:
        ckpt = torch.stack([t.detach().contiguous() for t in x0])[None]
    else:
        n_ckpt = (n + seg_len - 1) // seg_len
        ckpt = torch.empty((n_ckpt, 3, H, W), dtype=torch.float32, device=dev)
        work = [t.detach().clone().contiguous() for t in x0]
        with torch.cuda.device(dev):
            rc = dom._lib.swe_rollout_forward(dom._handle, _ptr(work[0]), _ptr(work[1]), _ptr(work[2]), W, n, 0.0,
                                              float(t0), dts.ctypes.data, None, 0, 1, None, _ptr(ckpt), seg_len,
                                              _stream(dev))
        _lib.check(rc, "interval checkpoint pass")
    seg = torch.empty((seg_len, 3, H, W), dtype=torch.float32, device=dev)
    gn2 = torch.zeros((H, W), dtype=torch.float32, device=dev)
    gr = torch.zeros(1, dtype=torch.float64, device=dev)
    with torch.cuda.device(dev):
        rc = dom._lib.swe_rollout_backward(dom._handle, _ptr(ckpt), seg_len, n, 0.0, float(t0), dts.ctypes.data,
                                           None, 0, 1, None, _ptr(lam[0]), _ptr(lam[1]), _ptr(lam[2]), W, 1,
                                           _ptr(gn2), _ptr(gr), _ptr(seg), _stream(dev))
    _lib.check(rc, "interval backward")
    return SWEState(*lam)


_SIDE_STREAMS: dict = {}
SIDE_STREAMS = 4  # concurrent member replays in an ensemble interval's backward


def _side_streams(dev: torch.device) -> list:
    key = (dev.index, SIDE_STREAMS)
    if key not in _SIDE_STREAMS:
        _SIDE_STREAMS[key] = [torch.cuda.Stream(dev) for _ in range(SIDE_STREAMS)]
    return _SIDE_STREAMS[key]


def _nan_if_short(state, t: float, target: float) -> None:
    if not t >= target - 1.0e-6:
        for x in state:
            x.fill_(float("nan"))


class PhysicsInterval(torch.autograd.Function):
    """forward(h, hu, hv, solver, t0, t1, max_steps) -> (h', hu', hv', steps) (steps: int64 scalar)."""

    @staticmethod
    def forward(ctx, h, hu, hv, solver, t0, t1, max_steps):
        x0 = SWEState(*(t.detach().to(torch.float32).contiguous().clone() for t in (h, hu, hv)))
        out = SWEState(*(t.clone() for t in x0))
        log = torch.empty(max(int(max_steps), 1), dtype=torch.float64, device=solver.device)
        t, n, _ = solver.advance_to_(out, float(t0), float(t1), int(max_steps), dt_log=log)
        _nan_if_short(out, t, float(t1))
        ctx.dom = _domain(solver)
        ctx.meta = (float(t0), log[:n].cpu().numpy())
        ctx.save_for_backward(*x0)
        return out.h, out.hu, out.hv, torch.tensor(n, dtype=torch.int64)

    @staticmethod
    def backward(ctx, gh, ghu, ghv, _gn):
        t0, dts = ctx.meta
        x0 = SWEState(*ctx.saved_tensors)
        g = SWEState(*(torch.zeros_like(x0.h) if a is None else a for a in (gh, ghu, ghv)))
        lam = _replay_backward(ctx.dom, x0, dts, t0, g)
        return lam.h, lam.hu, lam.hv, None, None, None, None


def physics_interval(solver, state, t0: float, t1: float, max_steps: int) -> tuple[SWEState, int]:
    """Differentiable ``advance_physics_to_time`` (see :class:`PhysicsInterval`)."""
    h, hu, hv, n = PhysicsInterval.apply(state[0], state[1], state[2], solver, t0, t1, max_steps)
    return SWEState(h, hu, hv), int(n)


class EnsembleInterval(torch.autograd.Function):
    """forward(ensemble, t0, t1, max_steps, *flat_states) -> (*flat_states', steps[M])."""

    @staticmethod
    def forward(ctx, ens, t0, t1, max_steps, *flat):
        M = len(ens)
        x0 = [t.detach().to(torch.float32).contiguous().clone() for t in flat]
        cur = [SWEState(*(t.clone() for t in x0[3 * m:3 * m + 3])) for m in range(M)]
        logs = [torch.empty(max(int(max_steps), 1), dtype=torch.float64, device=ens.device) for _ in range(M)]
        res = ens.advance_to_(cur, float(t0), float(t1), int(max_steps), dt_logs=logs)
        steps = []
        dts = []
        for m, (t, n, _) in enumerate(res):
            _nan_if_short(cur[m], t, float(t1))
            steps.append(n)
            dts.append(logs[m][:n].cpu().numpy())
        ctx.doms = ensemble_domains(ens)
        ctx.meta = (float(t0), dts)
        ctx.save_for_backward(*x0)
        out = [x for s in cur for x in s]
        return (*out, torch.tensor(steps, dtype=torch.int64))

    @staticmethod
    def backward(ctx, *grads):
        # The members' replays are independent, so they run on a few side streams
        # at once: a member's steps fill the GPU only between their starts and
        # tails, which the other members' kernels fill in.
        t0, dts = ctx.meta
        x0 = ctx.saved_tensors
        dev = x0[0].device
        main = torch.cuda.current_stream(dev)
        streams = _side_streams(dev)
        out = []
        for m, dom in enumerate(ctx.doms):
            xm = SWEState(*x0[3 * m:3 * m + 3])
            g = SWEState(*(torch.zeros_like(xm.h) if a is None else a for a in grads[3 * m:3 * m + 3]))
            s = streams[m % len(streams)]
            s.wait_stream(main)
            for t in (*xm, *g):
                t.record_stream(s)  # made on the main stream, read on this one
            with torch.cuda.stream(s):
                lam = _replay_backward(dom, xm, dts[m], t0, g)
            for t in lam:
                t.record_stream(main)  # made on this stream, read on the main one
            out.extend(lam)
        for s in streams:
            main.wait_stream(s)
        return (None, None, None, None, *out)


def _vel(m, h, dry):
    return torch.where(h > dry, m / torch.clamp_min(h, dry), torch.zeros((), device=h.device))


def features_torch(state: SWEState, mask: torch.Tensor, bed: torch.Tensor | None, hybrid_inputs: HybridInputs,
                   rain_value: float, layout: str, dry: float, planes=None) -> torch.Tensor:
    """Differentiable features ``[C, rows, cols]`` (float32), the same values as ``features_kernel``."""
    nstat = 3 if layout == "reference6" else 5
    dev = state.h.device
    mean = torch.from_numpy(_host_f32(hybrid_inputs.state_mean, nstat, "state_mean")).to(dev)
    std = torch.from_numpy(_host_f32(hybrid_inputs.state_std, nstat, "state_std")).to(dev)
    zero = torch.zeros((), device=dev)
    if layout == "reference6":
        dyn = torch.stack((state.h, _vel(state.hu, state.h, dry), _vel(state.hv, state.h, dry)))
        dyn = (dyn - mean[:, None, None]) / std[:, None, None]
        dyn = torch.where(mask[None], dyn, zero)
        terrain, rough = planes
        rain = torch.full_like(state.h, float(rain_value))
        extra = [rain, terrain if terrain is not None else torch.zeros_like(state.h),
                 rough if rough is not None else torch.zeros_like(state.h)]
        return torch.cat((dyn, torch.stack(extra)))
    src = torch.stack((state.h, state.hu, state.hv, bed, torch.full_like(state.h, float(rain_value))))
    f = (src - mean[:, None, None]) / std[:, None, None]
    return torch.where(mask[None], f, zero)


def correction_torch(pred: SWEState, residual: torch.Tensor, mask: torch.Tensor, dry: float, relaxation: float,
                     clip_limits=None) -> SWEState:
    """Differentiable ``apply_residual_correction`` (coupled_forecast.py:82-120) with the clip of
    ``:199-200``; ``residual`` is ``[C, rows, cols]``."""
    r = residual.float()
    if clip_limits is not None:
        lim = torch.as_tensor(np.asarray(clip_limits, np.float32)[: r.shape[0]], device=r.device)[:, None, None]
        r = torch.maximum(torch.minimum(r, lim), -lim)
    zero = torch.zeros((), device=r.device)
    u = _vel(pred.hu, pred.h, dry)
    v = _vel(pred.hv, pred.h, dry)
    prov = torch.where(mask, F.relu(pred.h + relaxation * r[0]), zero)
    target = torch.where(mask, pred.h, zero).double().sum()
    provisional = prov.double().sum()
    scale = torch.where(provisional > F32_EPS, target / provisional, torch.ones((), dtype=torch.float64,
                                                                                  device=r.device)).float()
    ch = torch.where(target > F32_EPS, prov * scale, pred.h)
    if r.shape[0] >= 3:
        u = u + relaxation * r[1]
        v = v + relaxation * r[2]
    wet = mask & (ch > dry)
    return SWEState(ch, torch.where(wet, ch * u, zero), torch.where(wet, ch * v, zero))


def coupled_loss(ensemble, initial_states, model, hybrid_inputs: HybridInputs, output_times_s, targets, *,
                 max_substeps_per_interval: int, correction_relaxation: float = 0.5,
                 correction_clip_sigma: float = 5.0, feature_layout: str = "state5",
                 loss_fn=None, checkpoint_model: bool = True):
    """Differentiable coupled rollout of every ensemble member and its loss.

    ``targets[m][k]`` is member m's target depth ``[rows, cols]`` at output time
    k >= 1 (e.g. a refined run block-averaged to this grid).  The default loss
    is the mean squared depth error over active cells and all intervals.
    Returns ``(loss, final_states, physics_steps [M])``.
    """
    times = np.asarray(output_times_s, dtype=np.float64).reshape(-1)
    if times.size < 2:
        raise ValueError("At least two output times are required.")
    if max_substeps_per_interval < 1:
        raise ValueError("At least one physics substep per correction interval is required.")
    M = len(ensemble)
    dev = ensemble.device
    doms = ensemble_domains(ensemble)
    masks = ensemble.masks
    beds = [torch.as_tensor(b, dtype=torch.float32, device=dev) for b in ensemble.beds]
    his = [hybrid_inputs] * M if isinstance(hybrid_inputs, HybridInputs) else list(hybrid_inputs)
    planes = [(None, None)] * M
    if feature_layout == "reference6":
        planes = [tuple(None if p is None else torch.as_tensor(p, dtype=torch.float32, device=dev)
                        for p in (hi.terrain_standardized, hi.roughness_standardized)) for hi in his]
    lims = []
    for hi in his:
        std = None if hi.residual_std is None else np.asarray(torch.as_tensor(hi.residual_std).cpu(), np.float32)
        lims.append(None if std is None else np.float32(correction_clip_sigma) * std.reshape(-1))
    mdtype = next(model.parameters()).dtype
    cur = [SWEState(*(torch.as_tensor(t, dtype=torch.float32, device=dev) for t in s)) for s in initial_states]
    loss = torch.zeros((), dtype=torch.float32, device=dev)
    steps = torch.zeros(M, dtype=torch.int64)
    count = 0
    for k in range(1, times.size):
        feats = torch.stack([
            features_torch(cur[m], masks[m], beds[m], his[m], rain_feature(doms[m], his[m], times[k - 1],
                                                                              feature_layout),
                           feature_layout, doms[m].dry, planes[m]) for m in range(M)])
        feats = feats.to(mdtype).contiguous(memory_format=torch.channels_last)
        flat = [x for s in cur for x in s]
        out = EnsembleInterval.apply(ensemble, float(times[k - 1]), float(times[k]),
                                     int(max_substeps_per_interval), *flat)
        steps += out[-1]
        adv = [SWEState(*out[3 * m:3 * m + 3]) for m in range(M)]
        residual = checkpoint(model, feats, use_reentrant=False) if checkpoint_model else model(feats)
        cur = [correction_torch(adv[m], residual[m], masks[m], doms[m].dry, correction_relaxation, lims[m])
               for m in range(M)]
        for m in range(M):
            tgt = torch.as_tensor(targets[m][k], dtype=torch.float32, device=dev)
            if loss_fn is None:
                d = torch.where(masks[m], cur[m].h - tgt, torch.zeros((), device=dev))
                loss = loss + (d * d).sum() / masks[m].sum()
            else:
                loss = loss + loss_fn(cur[m], tgt, masks[m])
            count += 1
    return loss / max(count, 1), cur, steps


def train_step(ensemble, initial_states, model, optimizer, hybrid_inputs, output_times_s, targets, **kw):
    """One optimiser step on :func:`coupled_loss`; returns the loss value."""
    model.train()
    optimizer.zero_grad(set_to_none=True)
    loss, _, steps = coupled_loss(ensemble, initial_states, model, hybrid_inputs, output_times_s, targets, **kw)
    loss.backward()
    optimizer.step()
    return float(loss.detach()), steps


def refine2(a: np.ndarray) -> np.ndarray:
    """Each cell split into 2x2 cells of the same value (a 2x refined grid)."""
    return np.repeat(np.repeat(np.asarray(a), 2, axis=0), 2, axis=1)


def coarsen2(a) -> np.ndarray:
    """2x2 block means (back to the coarse grid)."""
    a = np.asarray(a, dtype=np.float64)
    return (0.25 * (a[0::2, 0::2] + a[1::2, 0::2] + a[0::2, 1::2] + a[1::2, 1::2])).astype(np.float32)


def refined_targets(member: dict, depth0: np.ndarray, output_times_s, *, arithmetic: str = "fast",
                    device=None, max_steps: int = 200_000) -> list[np.ndarray]:
    """Target depths at every output time from a run on the 2x refined grid.

    The member's bed, roughness, mask and initial depth are refined 2x (dx
    halved), run with the same forcing, and block-averaged back; entry 0 is the
    initial depth.
    """
    from .solver import B200ShallowWaterSolver

    kw = {k: v for k, v in member.items() if k not in ("bed", "manning_n", "domain_mask", "rainfall_multiplier")}
    kw["resolution_m"] = float(member["resolution_m"]) / 2.0
    if member.get("rainfall_multiplier") is not None:
        kw["rainfall_multiplier"] = refine2(member["rainfall_multiplier"])
    s = B200ShallowWaterSolver(refine2(member["bed"]), refine2(member["manning_n"]),
                               refine2(member["domain_mask"]), **kw, arithmetic=arithmetic, device=device)
    init = s.initial_state(depth_m=refine2(depth0))
    times = np.asarray(output_times_s, dtype=np.float32)
    r = s.run(init, times, max_steps=max_steps)
    return [coarsen2(r.states.h[k].cpu().numpy()) for k in range(times.size)]
