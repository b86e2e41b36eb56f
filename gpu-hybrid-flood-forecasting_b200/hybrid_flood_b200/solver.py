"""Drop-in B200 solver behind the reference's ``run``/``step`` entry points.

Mirrors, name for name, the reference's solver surface:

* ``B200ShallowWaterSolver(bed, manning_n, domain_mask, *, resolution_m,
  rainfall_times_s, rainfall_rates_m_s, default_rainfall_m_s, gravity_m_s2,
  cfl, dry_tolerance_m, max_dt_s)`` -- the constructor of
  ``NumpyShallowWaterSolver`` (``src/hybrid_flood/numpy_solver/shallow_water_2d.py:333-365``)
  plus ``rainfall_multiplier`` and ``boundaries`` from the JAX wrapper
  (``src/hybrid_flood/jax_solver/shallow_water_2d.py:213-253``).
* ``.initial_state(depth_m, x_velocity_m_s, y_velocity_m_s)`` (``:367-380``).
* ``.run(initial_state, output_times_s, *, max_steps=20_000)`` (``:382-424``),
  same validation, same ``ValueError``/``RuntimeError``, same result fields
  (``states``, ``output_times_s``, ``final_time_s``, ``outputs_written``,
  ``steps_used``) plus the FP64 mass ``ledger``.
* module functions ``finite_volume_step(state, params, dt, time_s)``,
  ``compute_cfl_dt(state, params)`` and ``rainfall_rate(params, time_s)``
  (``:254-327``; ``jax_solver/numerics.py:286-369``).

State lives in device memory as torch float32 tensors ``[rows, cols]``; torch
is used for allocation and streams only -- every step runs in the sm_100a
kernels of ``libswe_b200.so`` through its C ABI.  ``run`` also accepts host
(NumPy) initial states and copies them in, as a drop-in for the NumPy solver.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import NamedTuple

import numpy as np
import torch

from . import _lib
from .boundary import BoundaryConfig, codes

_OUTPUT_TIMES_MSG = "Output times must be one-dimensional, start at zero, and increase."


class SWEState(NamedTuple):
    """Cell-average conserved variables ``(h, hu, hv)`` on the device."""

    h: torch.Tensor
    hu: torch.Tensor
    hv: torch.Tensor


class RunResult(NamedTuple):
    """States recorded at fixed output times (fields of the reference's result types)."""

    states: SWEState
    output_times_s: np.ndarray
    final_time_s: float
    outputs_written: int
    steps_used: int
    ledger: dict

    def to_numpy(self) -> "RunResult":
        """Copy the stacked states to host NumPy arrays."""
        st = SWEState(*(t.detach().cpu().numpy() for t in self.states))
        return self._replace(states=st)


LEDGER_KEYS = ("volume0", "volume", "rain_in", "outflow", "clip_gain", "mask_loss")


def ledger_error(ledger: dict) -> float:
    """Relative closing error of the FP64 ledger (see ``oracle``-independent definition).

    ``volume - (volume0 + rain_in - outflow + clip_gain - mask_loss)`` over the
    gross volume moved, the form of ``anuga_solver/run_simulation.py:100-116``.
    """
    expected = (ledger["volume0"] + ledger["rain_in"] - ledger["outflow"] + ledger["clip_gain"]
                - ledger["mask_loss"])
    scale = max(abs(ledger["volume0"]) + abs(ledger["rain_in"]) + abs(ledger["outflow"]), 1e-300)
    return abs(ledger["volume"] - expected) / scale


@dataclass(frozen=True)
class DeviceParams:
    """Static controls of a domain plus its native handle (reference ``NumpyParams``)."""

    handle: int
    shape: tuple
    dx: float
    dy: float
    gravity: float
    cfl: float
    dry_tolerance: float
    max_dt: float
    default_rainfall_m_s: float
    boundary: tuple
    arithmetic: str
    device: torch.device


def _stream(device: torch.device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _ptr(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _as_state(state, device: torch.device, shape) -> SWEState:
    """Device float32 views of a state given as tensors or host arrays."""
    out = []
    for a in state:
        if isinstance(a, torch.Tensor):
            t = a
            if t.device != device or t.dtype != torch.float32:
                t = t.to(device=device, dtype=torch.float32, non_blocking=True)
        else:
            host = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32))
            if torch.cuda.is_available():
                host = host.pin_memory()
            t = host.to(device, non_blocking=True)
        if tuple(t.shape) != tuple(shape):
            raise ValueError(f"State arrays must have shape {tuple(shape)}, got {tuple(t.shape)}.")
        if t.stride(-1) != 1:
            t = t.contiguous()
        out.append(t)
    return SWEState(*out)


def _pitch(t: torch.Tensor) -> int:
    return int(t.stride(0)) if t.dim() == 2 else int(t.shape[-1])


class B200ShallowWaterSolver:
    """sm_100a finite-volume shallow-water solver with the reference's API."""

    def __init__(
        self,
        bed,
        manning_n,
        domain_mask,
        *,
        resolution_m: float,
        rainfall_times_s,
        rainfall_rates_m_s,
        default_rainfall_m_s: float = 0.0,
        rainfall_multiplier=None,
        boundaries: BoundaryConfig | None = None,
        boundary=None,
        gravity_m_s2: float = 9.81,
        cfl: float = 0.45,
        dry_tolerance_m: float = 1.0e-4,
        max_dt_s: float = 10.0,
        arithmetic: str = "exact",
        device: torch.device | str | int | None = None,
    ) -> None:
        if not torch.cuda.is_available():
            raise RuntimeError("B200ShallowWaterSolver needs a CUDA device (sm_100a); none is visible.")
        lib = _lib.load()
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        # Fields already in this device's memory (e.g. from hybrid_flood_b200.generators)
        # are packed from there; anything else goes through the host.
        on_dev = all(isinstance(a, torch.Tensor) and a.is_cuda and a.device == self.device
                     for a in (bed, manning_n, domain_mask)) and (
            rainfall_multiplier is None or (isinstance(rainfall_multiplier, torch.Tensor)
                                            and rainfall_multiplier.device == self.device))
        if on_dev:
            bed_h = bed.detach().to(torch.float32).contiguous()
            man_h = manning_n.detach().to(torch.float32).contiguous()
            mask_h = domain_mask.detach().to(torch.bool).contiguous()
            mult_h = (rainfall_multiplier.detach().to(torch.float32).contiguous()
                      if rainfall_multiplier is not None else None)
        else:
            to_np = lambda a, dt: (a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)).astype(dt)  # noqa: E731
            bed_h = np.ascontiguousarray(to_np(bed, np.float32))
            man_h = np.ascontiguousarray(to_np(manning_n, np.float32))
            mask_h = np.ascontiguousarray(to_np(domain_mask, bool))
            mult_h = (np.ascontiguousarray(to_np(rainfall_multiplier, np.float32))
                      if rainfall_multiplier is not None else None)
        shape = tuple(bed_h.shape)
        if tuple(man_h.shape) != shape or tuple(mask_h.shape) != shape:
            raise ValueError("Bed, roughness, and domain mask must have identical shapes.")
        if len(shape) != 2:
            raise ValueError("Fields must be two-dimensional [rows, cols].")
        if mult_h is not None and tuple(mult_h.shape) != shape:
            raise ValueError("Rainfall multiplier must match the structured-grid shape.")
        rt = np.ascontiguousarray(np.asarray(rainfall_times_s, dtype=np.float32).reshape(-1))
        rr = np.ascontiguousarray(np.asarray(rainfall_rates_m_s, dtype=np.float32).reshape(-1))
        if rt.size < 1 or rt.size != rr.size:
            raise ValueError("Rainfall times and rates must be non-empty and of equal length.")
        bnd = codes(boundary if boundary is not None else boundaries)
        if arithmetic not in ("exact", "fast"):
            raise ValueError("arithmetic must be 'exact' or 'fast'")
        if on_dev:
            mask_u8 = mask_h.to(torch.uint8)
            ptr = lambda t: t.data_ptr()  # noqa: E731
        else:
            mask_u8 = mask_h.astype(np.uint8)
            ptr = lambda a: a.ctypes.data  # noqa: E731
        desc = _lib.DomainDesc()
        desc.rows, desc.cols = shape
        desc.dx = desc.dy = float(resolution_m)
        desc.gravity = float(gravity_m_s2)
        desc.cfl = float(cfl)
        desc.dry_tolerance = float(dry_tolerance_m)
        desc.max_dt = float(max_dt_s)
        desc.default_rainfall = float(default_rainfall_m_s)
        desc.boundary[:] = list(bnd)
        desc.n_rain = rt.size
        desc.rain_times = rt.ctypes.data
        desc.rain_rates = rr.ctypes.data
        desc.bed = ptr(bed_h)
        desc.manning_n = ptr(man_h)
        desc.domain_mask = ptr(mask_u8)
        desc.rainfall_multiplier = ptr(mult_h) if mult_h is not None else None
        desc.fields_on_host = 0 if on_dev else 1
        desc.arithmetic = _lib.SWE_ARITH_FAST if arithmetic == "fast" else _lib.SWE_ARITH_EXACT
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(lib.swe_domain_create(ctypes.byref(desc), ctypes.byref(handle)), "swe_domain_create")
        self._lib = lib
        self._handle = handle
        self.params = DeviceParams(
            handle=handle.value, shape=tuple(shape), dx=float(resolution_m), dy=float(resolution_m),
            gravity=float(gravity_m_s2), cfl=float(cfl), dry_tolerance=float(dry_tolerance_m),
            max_dt=float(max_dt_s), default_rainfall_m_s=float(default_rainfall_m_s), boundary=bnd,
            arithmetic=arithmetic, device=self.device,
        )
        self.domain_mask = mask_h if on_dev else torch.from_numpy(mask_h).to(self.device)
        self._bed = bed_h  # the output schema's elevation (host array or device tensor)
        self.shape = tuple(shape)

    @property
    def bed(self) -> np.ndarray:
        """Bed elevation as a host float32 array."""
        b = self._bed
        return b.cpu().numpy() if isinstance(b, torch.Tensor) else b

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                self._lib.swe_domain_destroy(h)
            except Exception:  # noqa: BLE001 - interpreter shutdown
                pass
            self._handle = None

    # -- reference surface --------------------------------------------------
    def initial_state(self, *, depth_m=0.0, x_velocity_m_s=0.0, y_velocity_m_s=0.0) -> SWEState:
        """Masked conserved fields from depth and velocity inputs (scalars, arrays or tensors)."""
        f32 = dict(dtype=torch.float32, device=self.device)

        def field(x):
            if isinstance(x, torch.Tensor):
                return x.to(**f32).broadcast_to(self.shape)
            return torch.as_tensor(np.asarray(x, dtype=np.float32), **f32).broadcast_to(self.shape)

        depth, u, v = field(depth_m), field(x_velocity_m_s), field(y_velocity_m_s)
        depth = torch.where(self.domain_mask, torch.clamp_min(depth, 0.0), torch.zeros((), **f32))
        return SWEState(depth.contiguous(), (depth * u).contiguous(), (depth * v).contiguous())

    def run(self, initial_state, output_times_s, *, max_steps: int = 20_000) -> RunResult:
        """Integrate adaptively to the requested output times on the device."""
        times = np.asarray(output_times_s, dtype=np.float32)
        if times.ndim != 1 or not len(times) or times[0] != 0 or np.any(np.diff(times) <= 0):
            raise ValueError(_OUTPUT_TIMES_MSG)
        times = np.ascontiguousarray(times)
        st = _as_state(initial_state, self.device, self.shape)
        n = len(times)
        outs = [torch.empty((n, *self.shape), dtype=torch.float32, device=self.device) for _ in range(3)]
        res = _lib.RunResult()
        with torch.cuda.device(self.device):
            rc = self._lib.swe_run(
                self._handle, _ptr(st.h), _ptr(st.hu), _ptr(st.hv), _pitch(st.h),
                times.ctypes.data, n, int(max_steps), _ptr(outs[0]), _ptr(outs[1]), _ptr(outs[2]),
                ctypes.byref(res), _stream(self.device),
            )
        _lib.check(rc, "run")
        return RunResult(
            SWEState(*outs), times, float(res.final_time_s), int(res.outputs_written),
            int(res.steps_used), dict(zip(LEDGER_KEYS, list(res.ledger))),
        )

    def run_to_host(self, initial_state, output_times_s, *, max_steps: int = 20_000, out=None) -> RunResult:
        """``run`` from and to host memory: the reference's NumPy-in, NumPy-out call.

        ``initial_state``: three host arrays ``[rows, cols]`` (NumPy or CPU
        tensors).  The outputs come back as NumPy arrays ``[n_out, rows, cols]``;
        each is copied to the host as soon as it is recorded, while the run
        continues.  ``out``: three preallocated CPU float32 tensors of that
        shape (pinned memory overlaps the copies); by default pinned ones are
        allocated.
        """
        times = np.asarray(output_times_s, dtype=np.float32)
        if times.ndim != 1 or not len(times) or times[0] != 0 or np.any(np.diff(times) <= 0):
            raise ValueError(_OUTPUT_TIMES_MSG)
        times = np.ascontiguousarray(times)
        n = len(times)
        host = []
        for a in initial_state:
            t = a if isinstance(a, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32))
            if t.is_cuda or t.dtype != torch.float32 or tuple(t.shape) != self.shape or t.stride(-1) != 1:
                raise ValueError(f"run_to_host needs host float32 arrays of shape {self.shape}")
            host.append(t)
        if out is None:
            out = [torch.empty((n, *self.shape), dtype=torch.float32).pin_memory() for _ in range(3)]
        for t in out:
            if t.is_cuda or t.dtype != torch.float32 or tuple(t.shape) != (n, *self.shape) or not t.is_contiguous():
                raise ValueError("out must be three contiguous host float32 tensors [n_out, rows, cols]")
        res = _lib.RunResult()
        with torch.cuda.device(self.device):
            rc = self._lib.swe_run_host(
                self._handle, *(ctypes.c_void_p(t.data_ptr()) for t in host), int(host[0].stride(0)),
                times.ctypes.data, n, int(max_steps), *(ctypes.c_void_p(t.data_ptr()) for t in out),
                ctypes.byref(res), _stream(self.device))
        _lib.check(rc, "run_to_host")
        return RunResult(SWEState(*(t.numpy() for t in out)), times, float(res.final_time_s),
                         int(res.outputs_written), int(res.steps_used), dict(zip(LEDGER_KEYS, list(res.ledger))))

    def step(self, state, dt: float, time_s: float) -> SWEState:
        return finite_volume_step(state, self.params, dt, time_s)

    def cfl_dt(self, state) -> float:
        return compute_cfl_dt(state, self.params)

    def max_inverse_dt(self, state) -> float:
        st = _as_state(state, self.device, self.shape)
        out = ctypes.c_float()
        with torch.cuda.device(self.device):
            rc = self._lib.swe_max_inverse_dt(self._handle, _ptr(st.h), _ptr(st.hu), _ptr(st.hv),
                                              _pitch(st.h), ctypes.byref(out), _stream(self.device))
        _lib.check(rc, "max_inverse_dt")
        return float(out.value)

    def rainfall_rate(self, time_s: float) -> float:
        return rainfall_rate(self.params, time_s)

    def advance_(self, state: SWEState, n_steps: int, start_time_s: float = 0.0) -> tuple[float, int, dict]:
        """Advance ``state`` IN PLACE by ``n_steps`` CFL-limited steps.

        Returns ``(final_time_s, steps_used, ledger)``.
        """
        res = _lib.RunResult()
        for t in state:
            if not (isinstance(t, torch.Tensor) and t.device == self.device and t.dtype == torch.float32
                    and tuple(t.shape) == self.shape and t.stride(-1) == 1):
                raise ValueError("advance_ needs device float32 [rows, cols] tensors")
        with torch.cuda.device(self.device):
            rc = self._lib.swe_advance(self._handle, _ptr(state.h), _ptr(state.hu), _ptr(state.hv),
                                       _pitch(state.h), int(n_steps), float(start_time_s),
                                       ctypes.byref(res), _stream(self.device))
        _lib.check(rc, "advance")
        return float(res.final_time_s), int(res.steps_used), dict(zip(LEDGER_KEYS, list(res.ledger)))

    # -- device-resident stepping ------------------------------------------------
    def resident_load(self, state, start_time_s: float = 0.0) -> None:
        """Copy ``state`` into the solver's own device buffers and start the clock.

        The reference's step loop (``numpy_solver/shallow_water_2d.py:402-412``)
        then runs on that resident copy through :meth:`resident_steps`, without
        the state leaving the device between calls.
        """
        st = _as_state(state, self.device, self.shape)
        with torch.cuda.device(self.device):
            rc = self._lib.swe_resident_load(self._handle, _ptr(st.h), _ptr(st.hu), _ptr(st.hv), _pitch(st.h),
                                             float(start_time_s), _stream(self.device))
        _lib.check(rc, "resident_load")

    def resident_steps(self, n_steps: int) -> None:
        """Enqueue ``n_steps`` CFL-limited steps of the resident state; returns at once."""
        with torch.cuda.device(self.device):
            rc = self._lib.swe_resident_steps(self._handle, int(n_steps), _stream(self.device))
        _lib.check(rc, "resident_steps")

    def resident_prepare(self, n_steps: int) -> None:
        """Capture the step graphs that a call of ``n_steps`` resident steps uses, from either
        ping-pong buffer, without running them."""
        with torch.cuda.device(self.device):
            rc = self._lib.swe_resident_prepare(self._handle, int(n_steps))
        _lib.check(rc, "resident_prepare")

    def resident_store(self, state: SWEState) -> tuple[float, int, dict]:
        """Copy the resident state into ``state`` (device tensors); ``(time, steps since load, ledger)``."""
        for t in state:
            if not (isinstance(t, torch.Tensor) and t.device == self.device and t.dtype == torch.float32
                    and tuple(t.shape) == self.shape and t.stride(-1) == 1):
                raise ValueError("resident_store needs device float32 [rows, cols] tensors")
        res = _lib.RunResult()
        with torch.cuda.device(self.device):
            rc = self._lib.swe_resident_store(self._handle, _ptr(state.h), _ptr(state.hu), _ptr(state.hv),
                                              _pitch(state.h), ctypes.byref(res), _stream(self.device))
        _lib.check(rc, "resident_store")
        return float(res.final_time_s), int(res.steps_used), dict(zip(LEDGER_KEYS, list(res.ledger)))

    def advance_to_(self, state: SWEState, start_time_s: float, target_time_s: float,
                    max_steps: int, dt_log: torch.Tensor | None = None) -> tuple[float, int, dict]:
        """Advance ``state`` IN PLACE from ``start_time_s`` to ``target_time_s``.

        CFL-limited steps with ``dt = min(cfl_dt, target - t)``, at most
        ``max_steps`` of them (``advance_physics_to_time``,
        ``src/hybrid_flood/hybrid/coupled_forecast.py:123-161``).  Returns
        ``(final_time_s, steps_used, ledger)``; when the step cap stops the run
        short, ``final_time_s`` is where it stopped and the state is the one
        reached there.  ``dt_log`` (device float64, at least ``max_steps``
        long) receives the dt of every step taken.
        """
        if dt_log is not None and not (dt_log.device == self.device and dt_log.dtype == torch.float64
                                       and dt_log.is_contiguous() and dt_log.numel() >= max_steps):
            raise ValueError("dt_log must be a contiguous device float64 tensor of at least max_steps")
        res = _lib.RunResult()
        for t in state:
            if not (isinstance(t, torch.Tensor) and t.device == self.device and t.dtype == torch.float32
                    and tuple(t.shape) == self.shape and t.stride(-1) == 1):
                raise ValueError("advance_to_ needs device float32 [rows, cols] tensors")
        with torch.cuda.device(self.device):
            rc = self._lib.swe_advance_to(self._handle, _ptr(state.h), _ptr(state.hu), _ptr(state.hv),
                                          _pitch(state.h), float(start_time_s), float(target_time_s),
                                          int(max_steps), _ptr(dt_log) if dt_log is not None else None,
                                          ctypes.byref(res), _stream(self.device))
        if rc != _lib.SWE_ERR_MAX_STEPS:
            _lib.check(rc, "advance_to")
        return float(res.final_time_s), int(res.steps_used), dict(zip(LEDGER_KEYS, list(res.ledger)))

    def advance(self, state, n_steps: int, start_time_s: float = 0.0):
        """Functional form of :meth:`advance_`: returns ``(new_state, final_time_s, steps_used, ledger)``."""
        st = _as_state(state, self.device, self.shape)
        st = SWEState(*(t.clone() for t in st))
        t, n, ledger = self.advance_(st, n_steps, start_time_s)
        return st, t, n, ledger

    def last_launch_count(self) -> int:
        return int(self._lib.swe_last_launch_count(self._handle))

    def set_timing(self, enable: bool = True) -> None:
        """Time the step kernels of subsequent run/advance calls with CUDA events."""
        _lib.check(self._lib.swe_set_timing(self._handle, 1 if enable else 0), "set_timing")

    def last_step_time(self) -> tuple[float, int]:
        """``(milliseconds, step launches)`` of the last timed run/advance."""
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        _lib.check(self._lib.swe_last_step_time(self._handle, ctypes.byref(ms), ctypes.byref(n)),
                   "last_step_time")
        return float(ms.value), int(n.value)


# -- module-level functional API (reference numerics) -------------------------
def _solver_call(params: DeviceParams):
    return _lib.load(), ctypes.c_void_p(params.handle)


def finite_volume_step(state, params: DeviceParams, dt: float, time_s: float) -> SWEState:
    """One conservative, well-balanced HLL step (new tensors; inputs untouched)."""
    lib, h = _solver_call(params)
    st = _as_state(state, params.device, params.shape)
    out = [torch.empty(params.shape, dtype=torch.float32, device=params.device) for _ in range(3)]
    with torch.cuda.device(params.device):
        rc = lib.swe_step(h, _ptr(st.h), _ptr(st.hu), _ptr(st.hv), _pitch(st.h),
                          _ptr(out[0]), _ptr(out[1]), _ptr(out[2]), _pitch(out[0]),
                          float(dt), float(time_s), _stream(params.device))
    _lib.check(rc, "finite_volume_step")
    return SWEState(*out)


def compute_cfl_dt(state, params: DeviceParams) -> float:
    """Unsplit two-dimensional CFL time step (float64, as the reference's host code)."""
    lib, h = _solver_call(params)
    st = _as_state(state, params.device, params.shape)
    out = ctypes.c_double()
    with torch.cuda.device(params.device):
        rc = lib.swe_cfl_dt(h, _ptr(st.h), _ptr(st.hu), _ptr(st.hv), _pitch(st.h),
                            ctypes.byref(out), _stream(params.device))
    _lib.check(rc, "compute_cfl_dt")
    return float(out.value)


def rainfall_rate(params: DeviceParams, time_s: float) -> float:
    """Linearly interpolated uniform rainfall (m/s) at ``time_s``."""
    lib, h = _solver_call(params)
    out = ctypes.c_double()
    _lib.check(lib.swe_rainfall_rate(h, float(time_s), ctypes.byref(out)), "rainfall_rate")
    return float(out.value)


def benchmark_compiled_steps(solver: "B200ShallowWaterSolver", state, *, iterations: int = 100, dt_s: float = 1.0,
                             output_directory=None) -> dict:
    """Fixed-dt step timing (``src/hybrid_flood/jax_solver/benchmarking.py:17-97``).

    ``iterations`` steps of ``dt_s`` from t = 0 (step k at time k*dt), run once
    untimed and then timed with CUDA events on the solver's stream; the report
    has the reference's fields.  The B200 path has no CPU backend, so the
    ``cpu`` record says it is unavailable.
    """
    import datetime
    import json
    import pathlib

    if iterations < 1:
        raise ValueError("Benchmark iterations must be positive.")
    dev = solver.device
    base = _as_state(state, dev, solver.shape)
    work = SWEState(*(t.clone().contiguous() for t in base))
    lib = solver._lib

    def once():
        for t, b in zip(work, base):
            t.copy_(b)
        with torch.cuda.device(dev):
            rc = lib.swe_rollout_forward(solver._handle, _ptr(work.h), _ptr(work.hu), _ptr(work.hv),
                                         _pitch(work.h), int(iterations), float(dt_s), 0.0, None, None, 0, 1, None,
                                         None, 1, _stream(dev))
        _lib.check(rc, "benchmark_compiled_steps")

    once()
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for t, b in zip(work, base):
        t.copy_(b)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    with torch.cuda.device(dev):
        rc = lib.swe_rollout_forward(solver._handle, _ptr(work.h), _ptr(work.hu), _ptr(work.hv), _pitch(work.h),
                                     int(iterations), float(dt_s), 0.0, None, None, 0, 1, None, None, 1, _stream(dev))
    e1.record(stream)
    torch.cuda.synchronize(dev)
    _lib.check(rc, "benchmark_compiled_steps")
    elapsed = e0.elapsed_time(e1) / 1e3
    records = [
        {"platform": "cpu", "available": False, "reason": "The B200 solver has no CPU backend."},
        {"platform": "gpu", "available": True, "device": torch.cuda.get_device_name(dev),
         "iterations": int(iterations), "total_seconds": elapsed, "seconds_per_step": elapsed / iterations,
         "steps_per_second": iterations / elapsed, "grid_shape": list(solver.shape), "dtype": "float32",
         "includes_jit_compilation": False, "arithmetic": solver.params.arithmetic},
    ]
    report = {
        "generated_at": datetime.datetime.now(datetime.timezone.utc).isoformat(),
        "library_version": lib.swe_version().decode(),
        "default_backend": "gpu",
        "devices": [torch.cuda.get_device_name(dev)],
        "gpu_benchmark_available": True,
        "benchmarks": records,
    }
    if output_directory is not None:
        directory = pathlib.Path(output_directory)
        directory.mkdir(parents=True, exist_ok=True)
        stamp = datetime.datetime.now(datetime.timezone.utc).strftime("%Y%m%dT%H%M%S%fZ")
        path = directory / f"benchmark_{stamp}.json"
        path.write_text(json.dumps(report, indent=2, sort_keys=True), encoding="utf-8")
        report["output_path"] = str(path)
    return report
