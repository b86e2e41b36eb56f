"""Physics-AI coupled rollout on the sm_100a solver.

Drop-in for ``src/hybrid_flood/hybrid/coupled_forecast.py``: the same
functions, arguments and failure behaviour, with a torch ``nn.Module`` as the
corrector instead of a Flax ``apply_fn``.

One correction interval (``run_coupled_forecast``'s ``coupled_step``,
``coupled_forecast.py:188-207``) is, all on one CUDA stream:

1. ``features_kernel``: the network features of the pre-advance state,
   written channels-last (NHWC) in the network's dtype;
2. ``swe_advance_to``: CFL-limited physics steps to the correction time, the
   run-mode step kernel with its on-device clock (``advance_physics_to_time``,
   ``:123-161``);
3. the corrector (cuDNN convolutions in bfloat16, ``channels_last``);
4. ``correction_sums_kernel`` + ``correction_apply_kernel``: the clip to
   ``clip_sigma * residual_std`` fused with the volume-preserving correction
   (``:82-120`` and ``:199-200``), reading the residual in place.

Two feature layouts: ``"reference6"`` (the reference's six channels) and
``"state5"`` ((h, hu, hv, z, rain in mm/h) standardised, the input of the
4-level depth-only corrector).
"""

from __future__ import annotations

import ctypes
from typing import Any, NamedTuple

import numpy as np
import torch

from . import _lib
from .solver import SWEState, _ptr, _stream

M_S_TO_MM_HR = 3.6e6  # coupled_forecast.py:27

LAYOUTS = {"reference6": (0, 6), "state5": (1, 5)}


class HybridInputs(NamedTuple):
    """Static normalised network inputs and training statistics (coupled_forecast.py:30-38).

    ``state_mean``/``state_std`` hold 3 values (h, u, v) for ``"reference6"`` or
    5 values (h, hu, hv, z, rain mm/h) for ``"state5"``; ``residual_std`` one
    value per residual channel.  ``terrain_standardized`` and
    ``roughness_standardized`` are [rows, cols] (``"reference6"`` only).
    """

    terrain_standardized: Any
    roughness_standardized: Any
    state_mean: Any
    state_std: Any
    rainfall_scale_mm_hr: float
    residual_std: Any


class CoupledRolloutResult(NamedTuple):
    """Corrected conserved states at the output times (coupled_forecast.py:41-46)."""

    states: SWEState  # [T, rows, cols] each
    output_times_s: np.ndarray
    physics_steps_used: int


def _host_f32(values, n: int, what: str) -> np.ndarray:
    if isinstance(values, torch.Tensor):
        values = values.detach().cpu().numpy()
    a = np.asarray(values, dtype=np.float32).reshape(-1)
    if a.size == 1 and n > 1:
        a = np.repeat(a, n)
    if a.size < n:
        raise ValueError(f"{what} needs {n} values, got {a.size}")
    return np.ascontiguousarray(a[:n])


def _dev_plane(values, solver) -> torch.Tensor | None:
    if values is None:
        return None
    t = torch.as_tensor(values, dtype=torch.float32, device=solver.device).contiguous()
    if tuple(t.shape) != tuple(solver.shape):
        raise ValueError(f"static feature planes must have shape {tuple(solver.shape)}")
    return t


def _check_state(state, solver) -> SWEState:
    for t in state:
        if not (isinstance(t, torch.Tensor) and t.device == solver.device and t.dtype == torch.float32
                and tuple(t.shape) == tuple(solver.shape) and t.stride(-1) == 1):
            raise ValueError("states must be device float32 [rows, cols] tensors with unit column stride")
    if not (state.h.stride(0) == state.hu.stride(0) == state.hv.stride(0)):
        raise ValueError("h, hu and hv must share one row pitch")
    return SWEState(*state)


class _Domain:
    """What the coupling kernels need of a solver or of an ensemble member."""

    def __init__(self, lib, handle, shape, device, dry) -> None:
        self._lib, self._handle, self.shape, self.device, self.dry = lib, handle, tuple(shape), device, dry

    def rainfall_rate(self, time_s: float) -> float:
        out = ctypes.c_double()
        _lib.check(self._lib.swe_rainfall_rate(self._handle, float(time_s), ctypes.byref(out)), "rainfall_rate")
        return float(out.value)


def _domain(solver) -> _Domain:
    if isinstance(solver, _Domain):
        return solver
    return _Domain(solver._lib, solver._handle, solver.shape, solver.device, solver.params.dry_tolerance)


def rain_feature(dom, hybrid_inputs: HybridInputs, time_s: float, layout: str) -> float:
    """The rain channel's value at ``time_s`` (coupled_forecast.py:65-69)."""
    rate = dom.rainfall_rate(time_s)
    mm_hr = np.float32(rate * M_S_TO_MM_HR)
    if layout == "reference6":
        return float(mm_hr / np.float32(hybrid_inputs.rainfall_scale_mm_hr))
    return float(mm_hr)


def network_features(solver, state, hybrid_inputs: HybridInputs, time_s: float, *, layout: str = "reference6",
                     dtype: torch.dtype = torch.float32, out: torch.Tensor | None = None,
                     _planes=None) -> torch.Tensor:
    """Network input features, ``[1, rows, cols, C]`` (NHWC) in ``dtype`` (coupled_forecast.py:53-79).

    ``out`` may be a preallocated ``[rows, cols, C]`` (or ``[1, rows, cols, C]``)
    contiguous tensor, e.g. one member's slice of a batch.
    """
    if layout not in LAYOUTS:
        raise ValueError(f"unknown feature layout {layout!r}; choose one of {sorted(LAYOUTS)}")
    if dtype not in (torch.float32, torch.bfloat16):
        raise ValueError("features are float32 or bfloat16")
    dom = _domain(solver)
    state = _check_state(state, dom)
    code, C = LAYOUTS[layout]
    H, W = dom.shape
    if out is None:
        out = torch.empty((1, H, W, C), dtype=dtype, device=dom.device)
    if out.dtype != dtype or not out.is_contiguous() or out.numel() != H * W * C or out.device != dom.device:
        raise ValueError("out must be a contiguous [rows, cols, C] tensor of the feature dtype on the device")
    nstat = 3 if layout == "reference6" else 5
    mean = _host_f32(hybrid_inputs.state_mean, nstat, "state_mean")
    std = _host_f32(hybrid_inputs.state_std, nstat, "state_std")
    if _planes is None:
        terrain = _dev_plane(hybrid_inputs.terrain_standardized, dom) if layout == "reference6" else None
        rough = _dev_plane(hybrid_inputs.roughness_standardized, dom) if layout == "reference6" else None
    else:
        terrain, rough = _planes
    rf = rain_feature(dom, hybrid_inputs, time_s, layout)
    with torch.cuda.device(dom.device):
        rc = dom._lib.swe_network_features(
            dom._handle, _ptr(state.h), _ptr(state.hu), _ptr(state.hv), int(state.h.stride(0)), code,
            mean.ctypes.data, std.ctypes.data, ctypes.c_float(rf),
            _ptr(terrain) if terrain is not None else None, _ptr(rough) if rough is not None else None,
            _ptr(out), 1 if dtype == torch.bfloat16 else 0, _stream(dom.device))
    _lib.check(rc, "network_features")
    return out if out.dim() == 4 else out.view(1, H, W, C)


def _residual_view(residual: torch.Tensor, shape) -> torch.Tensor:
    """[rows, cols, C] view of a residual given as NHWC [rows, cols, C], [1, rows, cols, C] or NCHW [1, C, rows, cols]."""
    H, W = shape
    r = residual
    if r.dim() == 4:
        if r.shape[0] != 1:
            raise ValueError("a 4-D residual must have batch 1")
        r = r[0]
        if tuple(r.shape[1:]) == (H, W):  # [C, H, W] (NCHW model output)
            r = r.permute(1, 2, 0)
    if r.dim() != 3 or tuple(r.shape[:2]) != (H, W):
        raise ValueError(f"residual must be [rows, cols, C] for shape {(H, W)}, got {tuple(residual.shape)}")
    return r


def apply_residual_correction(solver, predicted, residual: torch.Tensor, *, correction_relaxation: float,
                              clip_limits=None, out: SWEState | None = None) -> SWEState:
    """Volume-preserving correction of ``predicted`` by ``residual`` (coupled_forecast.py:82-120).

    ``residual`` channels: (depth, u, v) or depth only; any strides, float32 or
    bfloat16, read in place.  ``clip_limits`` (one per channel) clips the
    residual first (``:199-200``); ``out`` may alias ``predicted``.
    """
    dom = _domain(solver)
    predicted = _check_state(predicted, dom)
    r = _residual_view(residual, dom.shape)
    if r.device != dom.device:
        raise ValueError("residual must be on the solver's device")
    if r.dtype not in (torch.float32, torch.bfloat16):
        r = r.float()
    nch = int(r.shape[2])
    if nch not in (1, 3):
        raise ValueError("residual must have 1 (depth) or 3 (depth, u, v) channels")
    lim = None if clip_limits is None else _host_f32(clip_limits, nch, "clip_limits")
    if out is None:
        out = SWEState(*(torch.empty(dom.shape, dtype=torch.float32, device=dom.device) for _ in range(3)))
    out = _check_state(out, dom)
    with torch.cuda.device(dom.device):
        rc = dom._lib.swe_apply_correction(
            dom._handle, _ptr(predicted.h), _ptr(predicted.hu), _ptr(predicted.hv), int(predicted.h.stride(0)),
            _ptr(r), 1 if r.dtype == torch.bfloat16 else 0, int(r.stride(0)), int(r.stride(1)), int(r.stride(2)),
            nch, lim.ctypes.data if lim is not None else None, float(correction_relaxation),
            _ptr(out.h), _ptr(out.hu), _ptr(out.hv), int(out.h.stride(0)), _stream(dom.device))
    _lib.check(rc, "apply_residual_correction")
    return out


def _nan_fill(state: SWEState) -> None:
    for t in state:
        t.fill_(float("nan"))


def advance_physics_to_time(solver, state, start_time_s: float, target_time_s: float, *,
                            max_substeps: int) -> tuple[SWEState, int]:
    """Adaptive physics to one correction time (coupled_forecast.py:123-161).

    Returns ``(state, steps)``; the state is NaN-filled when ``max_substeps``
    steps did not reach the target within 1e-6 s, as in the reference.
    """
    if max_substeps < 1:
        raise ValueError("At least one physics substep per correction interval is required.")
    st = SWEState(*(t.to(device=solver.device, dtype=torch.float32).contiguous().clone() for t in state))
    t, steps, _ = solver.advance_to_(st, float(start_time_s), float(target_time_s), int(max_substeps))
    if not t >= float(target_time_s) - 1.0e-6:
        _nan_fill(st)
    return st, steps


class _Corrector:
    """Runs the corrector on a side stream so that it overlaps the physics advance.

    The residual of interval k depends only on the features of the state before
    the advance (coupled_forecast.py:190-198), so it is computed while the
    physics of the same interval runs; the correction waits for both.
    """

    def __init__(self, model, device, overlap: bool) -> None:
        self.model = model
        self.side = torch.cuda.Stream(device=device) if overlap else None
        self.done = torch.cuda.Event() if overlap else None

    def start(self, x: torch.Tensor):
        if self.side is None:
            return None
        main = torch.cuda.current_stream(x.device)
        self.side.wait_stream(main)
        with torch.cuda.stream(self.side):
            y = self.model(x)
        self.done.record(self.side)
        return y

    def finish(self, x: torch.Tensor, started):
        if self.side is None:
            return self.model(x)
        main = torch.cuda.current_stream(x.device)
        main.wait_event(self.done)
        started.record_stream(main)
        x.record_stream(self.side)
        return started


def _model_dtype(model) -> torch.dtype:
    for p in model.parameters():
        return p.dtype
    return torch.float32


def _clip_limits(hybrid_inputs: HybridInputs, clip_sigma: float):
    if hybrid_inputs.residual_std is None:
        return None
    std = np.asarray(torch.as_tensor(hybrid_inputs.residual_std).detach().cpu(), np.float32).reshape(-1)
    return (np.float32(clip_sigma) * std).astype(np.float32)


def _check_times(output_times_s) -> np.ndarray:
    times = np.asarray(output_times_s, dtype=np.float64).reshape(-1)
    if times.shape[0] < 2:
        raise ValueError("At least two output times are required.")
    return times


def run_coupled_forecast(solver, initial_state, model, hybrid_inputs: HybridInputs, output_times_s, *,
                         max_substeps_per_interval: int, correction_relaxation: float = 0.05,
                         correction_clip_sigma: float = 5.0, feature_layout: str = "reference6",
                         overlap: bool = False) -> CoupledRolloutResult:
    """Autoregressive physics + corrector rollout, device-resident (coupled_forecast.py:164-225).

    ``model`` maps NCHW features ``[1, C, rows, cols]`` to a NCHW residual; it
    runs in its own parameter dtype (bfloat16 models get bfloat16 NHWC features
    with no conversion) under ``torch.no_grad``; with ``overlap`` it runs on a
    side stream while the interval's physics runs (same results; on 16 x 1024^2
    members it saved nothing, both parts already fill the GPU).
    An interval that does not reach its time leaves NaN states, as in the
    reference.
    """
    if max_substeps_per_interval < 1:
        raise ValueError("At least one physics substep per correction interval is required.")
    times = _check_times(output_times_s)
    if feature_layout not in LAYOUTS:
        raise ValueError(f"unknown feature layout {feature_layout!r}")
    dom = _domain(solver)
    dev = dom.device
    H, W = dom.shape
    T = times.shape[0]
    init = SWEState(*(torch.as_tensor(t, dtype=torch.float32, device=dev) for t in initial_state))
    states = SWEState(*(torch.empty((T, H, W), dtype=torch.float32, device=dev) for _ in range(3)))
    for k in range(3):
        states[k][0].copy_(init[k])
    fdtype = _model_dtype(model)
    fdtype = fdtype if fdtype in (torch.float32, torch.bfloat16) else torch.float32
    feats = torch.empty((1, H, W, LAYOUTS[feature_layout][1]), dtype=fdtype, device=dev)
    planes = None
    if feature_layout == "reference6":
        planes = (_dev_plane(hybrid_inputs.terrain_standardized, dom),
                  _dev_plane(hybrid_inputs.roughness_standardized, dom))
    lim = _clip_limits(hybrid_inputs, correction_clip_sigma)
    corrector = _Corrector(model, dev, overlap)
    total = 0
    with torch.no_grad():
        for k in range(1, T):
            prev = SWEState(states.h[k - 1], states.hu[k - 1], states.hv[k - 1])
            cur = SWEState(states.h[k], states.hu[k], states.hv[k])
            network_features(dom, prev, hybrid_inputs, times[k - 1], layout=feature_layout, dtype=fdtype,
                             out=feats, _planes=planes)
            x = feats.permute(0, 3, 1, 2)
            started = corrector.start(x)
            for a, b in zip(cur, prev):
                a.copy_(b)
            t, steps, _ = solver.advance_to_(cur, times[k - 1], times[k], int(max_substeps_per_interval))
            total += steps
            if not t >= times[k] - 1.0e-6:
                _nan_fill(cur)
            residual = corrector.finish(x, started)
            apply_residual_correction(dom, cur, residual, correction_relaxation=correction_relaxation,
                                      clip_limits=lim, out=cur)
    return CoupledRolloutResult(states, times, total)


def select_relaxation_by_validation(candidate_metrics: dict) -> tuple[float, float]:
    """The relaxation with the lowest finite validation score; ties go to the smaller value.

    Same contract as ``src/hybrid_flood/hybrid/rollout.py:49-68``: candidates
    with a non-finite score or a negative relaxation are ignored; ``ValueError``
    when none is left.
    """
    if not candidate_metrics:
        raise ValueError("At least one correction-relaxation candidate is required.")
    best = None
    for relax, score in candidate_metrics.items():
        score, relax = float(score), float(relax)
        if not (np.isfinite(score) and relax >= 0.0):
            continue
        if best is None or (score, relax) < best:
            best = (score, relax)
    if best is None:
        raise ValueError("No candidate produced a finite validation metric.")
    return best[1], best[0]


def ensemble_domains(ensemble) -> list[_Domain]:
    """Borrowed per-member domains of a :class:`B200Ensemble` for the coupling kernels."""
    out = []
    for m, shape in enumerate(ensemble.shapes):
        h = ctypes.c_void_p()
        _lib.check(ensemble._lib.swe_ensemble_member(ensemble._handle, m, ctypes.byref(h)), "swe_ensemble_member")
        out.append(_Domain(ensemble._lib, h, shape, ensemble.device, ensemble.dry_tolerances[m]))
    return out


def _ptrs(tensors) -> ctypes.Array:
    return (ctypes.c_void_p * len(tensors))(*[None if t is None else t.data_ptr() for t in tensors])


def _pitches(states) -> ctypes.Array:
    return (ctypes.c_int64 * len(states))(*[int(s.h.stride(0)) for s in states])


def ensemble_network_features(ensemble, states, hybrid_inputs, time_s: float, *, layout: str = "state5",
                              out: torch.Tensor, doms=None, planes=None) -> torch.Tensor:
    """:func:`network_features` of every member of ``ensemble`` into ``out``
    (``[M, rows, cols, C]`` channels-last, contiguous) in one library call.

    ``hybrid_inputs``: one :class:`HybridInputs` or one per member; ``planes``:
    per member ``(terrain, roughness)`` device planes (``reference6``).
    """
    if layout not in LAYOUTS:
        raise ValueError(f"unknown feature layout {layout!r}; choose one of {sorted(LAYOUTS)}")
    M = len(ensemble)
    doms = ensemble_domains(ensemble) if doms is None else doms
    his = [hybrid_inputs] * M if isinstance(hybrid_inputs, HybridInputs) else list(hybrid_inputs)
    if len(his) != M or len(states) != M:
        raise ValueError(f"expected {M} states and one HybridInputs or {M} of them")
    if any(d.shape != doms[0].shape for d in doms):
        raise ValueError("ensemble_network_features needs members of one grid shape")
    states = [_check_state(st, d) for st, d in zip(states, doms)]
    code, C = LAYOUTS[layout]
    H, W = doms[0].shape
    if (out.dtype not in (torch.float32, torch.bfloat16) or not out.is_contiguous() or out.device != ensemble.device
            or tuple(out.shape) != (M, H, W, C)):
        raise ValueError(f"out must be a contiguous [{M}, {H}, {W}, {C}] float32 or bfloat16 tensor on the device")
    nstat = 3 if layout == "reference6" else 5
    stats = np.zeros((2, M, 5), np.float32)
    stats[1] = 1.0
    for m, hi in enumerate(his):
        stats[0, m, :nstat] = _host_f32(hi.state_mean, nstat, "state_mean")
        stats[1, m, :nstat] = _host_f32(hi.state_std, nstat, "state_std")
    rain = np.array([rain_feature(d, hi, time_s, layout) for d, hi in zip(doms, his)], np.float32)
    if layout == "reference6":
        if planes is None:
            planes = [(_dev_plane(hi.terrain_standardized, d), _dev_plane(hi.roughness_standardized, d))
                      for hi, d in zip(his, doms)]
        terrain, rough = _ptrs([p[0] for p in planes]), _ptrs([p[1] for p in planes])
    else:
        terrain = rough = None
    with torch.cuda.device(ensemble.device):
        rc = ensemble._lib.swe_ensemble_network_features(
            ensemble._handle, _ptrs([st.h for st in states]), _ptrs([st.hu for st in states]),
            _ptrs([st.hv for st in states]), _pitches(states), code, stats[0].ctypes.data, stats[1].ctypes.data,
            rain.ctypes.data, terrain, rough, _ptr(out), H * W * C, 1 if out.dtype == torch.bfloat16 else 0,
            _stream(ensemble.device))
    _lib.check(rc, "ensemble_network_features")
    return out


def ensemble_apply_correction(ensemble, predicted, residual: torch.Tensor, *, correction_relaxation: float,
                              clip_limits=None, out=None, doms=None) -> list[SWEState]:
    """:func:`apply_residual_correction` of every member in one library call.

    ``residual``: ``[M, C, rows, cols]`` (the corrector's NCHW output, any
    strides) or ``[M, rows, cols, C]``, float32 or bfloat16, read in place;
    ``clip_limits``: ``None`` or one limit array per member; ``out`` may alias
    ``predicted``.
    """
    M = len(ensemble)
    doms = ensemble_domains(ensemble) if doms is None else doms
    if any(d.shape != doms[0].shape for d in doms):
        raise ValueError("ensemble_apply_correction needs members of one grid shape")
    if len(predicted) != M:
        raise ValueError(f"expected {M} predicted states")
    predicted = [_check_state(st, d) for st, d in zip(predicted, doms)]
    H, W = doms[0].shape
    r = residual
    if r.dim() != 4 or r.shape[0] != M:
        raise ValueError(f"residual must be [{M}, C, rows, cols] or [{M}, rows, cols, C]")
    if tuple(r.shape[2:]) == (H, W):
        r = r.permute(0, 2, 3, 1)
    if tuple(r.shape[1:3]) != (H, W):
        raise ValueError(f"residual must be [{M}, C, rows, cols] or [{M}, rows, cols, C] for shape {(H, W)}")
    if r.device != ensemble.device:
        raise ValueError("residual must be on the ensemble's device")
    if r.dtype not in (torch.float32, torch.bfloat16):
        r = r.float()
    nch = int(r.shape[3])
    if nch not in (1, 3):
        raise ValueError("residual must have 1 (depth) or 3 (depth, u, v) channels")
    lim = None
    if clip_limits is not None and any(c is not None for c in clip_limits):
        lim = np.stack([np.full(nch, np.inf, np.float32) if c is None else _host_f32(c, nch, "clip_limits")
                        for c in clip_limits])
    if out is None:
        out = [SWEState(*(torch.empty((H, W), dtype=torch.float32, device=ensemble.device) for _ in range(3)))
               for _ in range(M)]
    out = [_check_state(st, d) for st, d in zip(out, doms)]
    with torch.cuda.device(ensemble.device):
        rc = ensemble._lib.swe_ensemble_apply_correction(
            ensemble._handle, _ptrs([st.h for st in predicted]), _ptrs([st.hu for st in predicted]),
            _ptrs([st.hv for st in predicted]), _pitches(predicted), _ptr(r), 1 if r.dtype == torch.bfloat16 else 0,
            int(r.stride(0)), int(r.stride(1)), int(r.stride(2)), int(r.stride(3)), nch,
            lim.ctypes.data if lim is not None else None, float(correction_relaxation),
            _ptrs([st.h for st in out]), _ptrs([st.hu for st in out]), _ptrs([st.hv for st in out]), _pitches(out),
            _stream(ensemble.device))
    _lib.check(rc, "ensemble_apply_correction")
    return out


def run_coupled_ensemble(ensemble, initial_states, model, hybrid_inputs: HybridInputs, output_times_s, *,
                         max_substeps_per_interval: int, correction_relaxation: float = 0.05,
                         correction_clip_sigma: float = 5.0, feature_layout: str = "state5",
                         keep_states: bool = True, timings: dict | None = None, overlap: bool = False):
    """The coupled rollout of every member of an ensemble, the corrector batched over members.

    All members must share one grid shape (the corrector runs on one
    ``[M, C, rows, cols]`` batch).  Per interval: features of every member
    into one NHWC batch, one ensemble ``advance_to`` (50-step graphs of the
    persistent multi-member kernel), one batched corrector call, and the
    correction of each member.  Returns ``(states, physics_steps_per_member)``
    where ``states[m]`` is that member's ``[T, rows, cols]`` trajectory (or its
    final state only when ``keep_states`` is false).  With ``timings`` (a dict)
    and ensemble timing on (``set_timing``), the device time of the physics
    advances is summed into ``timings["physics_ms"]``.
    """
    if max_substeps_per_interval < 1:
        raise ValueError("At least one physics substep per correction interval is required.")
    times = _check_times(output_times_s)
    shapes = set(ensemble.shapes)
    if len(shapes) != 1:
        raise ValueError("run_coupled_ensemble needs members of one grid shape")
    H, W = ensemble.shapes[0]
    M = len(ensemble)
    dev = ensemble.device
    doms = ensemble_domains(ensemble)
    T = times.shape[0]
    nkeep = T if keep_states else 1
    traj = [SWEState(*(torch.empty((nkeep, H, W), dtype=torch.float32, device=dev) for _ in range(3)))
            for _ in range(M)]
    cur = [SWEState(*(torch.as_tensor(t, dtype=torch.float32, device=dev).clone().contiguous() for t in s))
           for s in initial_states]
    if keep_states:
        for m in range(M):
            for k in range(3):
                traj[m][k][0].copy_(cur[m][k])
    fdtype = _model_dtype(model)
    fdtype = fdtype if fdtype in (torch.float32, torch.bfloat16) else torch.float32
    feats = torch.empty((M, H, W, LAYOUTS[feature_layout][1]), dtype=fdtype, device=dev)
    his = [hybrid_inputs] * M if isinstance(hybrid_inputs, HybridInputs) else list(hybrid_inputs)
    if len(his) != M:
        raise ValueError(f"expected one HybridInputs or {M} of them")
    planes = [None] * M
    if feature_layout == "reference6":
        planes = [(_dev_plane(hi.terrain_standardized, d), _dev_plane(hi.roughness_standardized, d))
                  for hi, d in zip(his, doms)]
    lims = [_clip_limits(hi, correction_clip_sigma) for hi in his]
    steps = np.zeros(M, dtype=np.int64)
    corrector = _Corrector(model, dev, overlap)
    with torch.no_grad():
        for k in range(1, T):
            ensemble_network_features(ensemble, cur, his, times[k - 1], layout=feature_layout, out=feats,
                                      doms=doms, planes=planes)
            x = feats.permute(0, 3, 1, 2)
            started = corrector.start(x)
            res = ensemble.advance_to_(cur, times[k - 1], times[k], int(max_substeps_per_interval))
            if timings is not None:
                ms, launches = ensemble.last_step_time()
                timings["physics_ms"] = timings.get("physics_ms", 0.0) + ms
                timings["physics_launches"] = timings.get("physics_launches", 0) + launches
            for m, (t, n, _) in enumerate(res):
                steps[m] += n
                if not t >= times[k] - 1.0e-6:
                    _nan_fill(cur[m])
            residual = corrector.finish(x, started)
            ensemble_apply_correction(ensemble, cur, residual, correction_relaxation=correction_relaxation,
                                      clip_limits=lims, out=cur, doms=doms)
            for m in range(M):
                if keep_states:
                    for q in range(3):
                        traj[m][q][k].copy_(cur[m][q])
    if not keep_states:
        for m in range(M):
            for q in range(3):
                traj[m][q][0].copy_(cur[m][q])
    return traj, steps
