"""Batched ensemble: many shallow-water domains of uneven size in one launch per step.

The reference runs one solver per scenario (``NumpyShallowWaterSolver.run``,
``src/hybrid_flood/numpy_solver/shallow_water_2d.py:382-424``).  An ensemble of
rainfall/roughness scenarios is many such runs.  ``B200Ensemble`` advances all
of them together: every member keeps its own float64 clock, CFL dt and mass
ledger, and one kernel launch (``ensemble_step_kernel``, a persistent grid
over a flattened work list of all members) advances every member by one of its
own steps.  Sequences of 50 steps are replayed from a captured CUDA graph.

The work-list granularity (rows each warp marches per item) is tuned by
:meth:`B200Ensemble.autotune`, which times the candidates on the live members
and caches the winner per member-shape set in a JSON file.
"""

from __future__ import annotations

import ctypes
import hashlib
import json
import os
import pathlib

import numpy as np
import torch

from . import _lib
from .boundary import codes
from .solver import LEDGER_KEYS, SWEState, _ptr, _stream

DEFAULT_CACHE = pathlib.Path(os.environ.get("SWE_TUNE_CACHE", pathlib.Path.home() / ".cache" / "swe_b200_tune.json"))


def _on_device(member: dict) -> bool:
    fields = [member["bed"], member["manning_n"], member["domain_mask"]]
    if member.get("rainfall_multiplier") is not None:
        fields.append(member["rainfall_multiplier"])
    return all(isinstance(a, torch.Tensor) and a.is_cuda for a in fields)


def _desc(member: dict, arithmetic: str, keep: list) -> _lib.DomainDesc:
    """A ``swe_domain_desc`` for one member (keyword arguments of B200ShallowWaterSolver).

    Members whose fields are device tensors (``hybrid_flood_b200.generators``)
    are packed from device memory; others from host arrays."""
    f32 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float32))  # noqa: E731
    on_dev = _on_device(member)
    if on_dev:
        bed = member["bed"].detach().to(torch.float32).contiguous()
        man = member["manning_n"].detach().to(torch.float32).contiguous()
        mask = member["domain_mask"].detach().to(torch.uint8).contiguous()
        ptr = lambda t: t.data_ptr()  # noqa: E731
    else:
        bed = f32(member["bed"])
        man = f32(member["manning_n"])
        mask = np.ascontiguousarray(np.asarray(member["domain_mask"], dtype=bool).astype(np.uint8))
        ptr = lambda a: a.ctypes.data  # noqa: E731
    shape = tuple(bed.shape)
    if tuple(man.shape) != shape or tuple(mask.shape) != shape:
        raise ValueError("Bed, roughness, and domain mask must have identical shapes.")
    rt = f32(member["rainfall_times_s"]).reshape(-1)
    rr = f32(member["rainfall_rates_m_s"]).reshape(-1)
    if rt.size < 1 or rt.size != rr.size:
        raise ValueError("Rainfall times and rates must be non-empty and of equal length.")
    mult = member.get("rainfall_multiplier")
    if mult is not None:
        mult = mult.detach().to(torch.float32).contiguous() if on_dev else f32(mult)
    keep.extend([bed, man, mask, rt, rr, mult])
    d = _lib.DomainDesc()
    d.rows, d.cols = shape
    d.dx = d.dy = float(member["resolution_m"])
    d.gravity = float(member.get("gravity_m_s2", 9.81))
    d.cfl = float(member.get("cfl", 0.45))
    d.dry_tolerance = float(member.get("dry_tolerance_m", 1.0e-4))
    d.max_dt = float(member.get("max_dt_s", 10.0))
    d.default_rainfall = float(member.get("default_rainfall_m_s", 0.0))
    d.boundary[:] = list(codes(member.get("boundary", member.get("boundaries"))))
    d.n_rain = rt.size
    d.rain_times, d.rain_rates = rt.ctypes.data, rr.ctypes.data
    d.bed, d.manning_n, d.domain_mask = ptr(bed), ptr(man), ptr(mask)
    d.rainfall_multiplier = ptr(mult) if mult is not None else None
    d.fields_on_host = 0 if on_dev else 1
    d.arithmetic = _lib.SWE_ARITH_FAST if arithmetic == "fast" else _lib.SWE_ARITH_EXACT
    return d


class B200Ensemble:
    """Members advanced together, each with its own CFL dt, clock and FP64 ledger."""

    def __init__(self, members: list[dict], *, arithmetic: str = "fast", device=None) -> None:
        if not torch.cuda.is_available():
            raise RuntimeError("B200Ensemble needs a CUDA device (sm_100a); none is visible.")
        if not members:
            raise ValueError("An ensemble needs at least one member.")
        if arithmetic not in ("exact", "fast"):
            raise ValueError("arithmetic must be 'exact' or 'fast'")
        self._lib = _lib.load()
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        keep: list = []
        descs = (_lib.DomainDesc * len(members))(*[_desc(m, arithmetic, keep) for m in members])
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self._lib.swe_ensemble_create(descs, len(members), ctypes.byref(handle)),
                       "swe_ensemble_create")
        self._handle = handle
        self.shapes = [tuple(m["bed"].shape) for m in members]
        self.masks = [torch.as_tensor(m["domain_mask"]).to(device=self.device, dtype=torch.bool) for m in members]
        self.arithmetic = arithmetic
        self.rows_per_warp = int(self._lib.swe_ensemble_rows_per_warp(handle))  # the library's one-round default
        self.dry_tolerances = [float(m.get("dry_tolerance_m", 1.0e-4)) for m in members]
        self.beds = [m["bed"].detach().cpu().numpy().astype(np.float32) if isinstance(m["bed"], torch.Tensor)
                     else np.asarray(m["bed"], dtype=np.float32) for m in members]

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                self._lib.swe_ensemble_destroy(h)
            except Exception:  # noqa: BLE001 - interpreter shutdown
                pass
            self._handle = None

    def __len__(self) -> int:
        return len(self.shapes)

    @property
    def cells(self) -> int:
        return int(sum(r * c for r, c in self.shapes))

    def initial_states(self, depths=None) -> list[SWEState]:
        """Masked still-water states (``depths``: scalar or one array per member)."""
        out = []
        for i, shape in enumerate(self.shapes):
            dep = 0.0 if depths is None else (depths[i] if isinstance(depths, (list, tuple)) else depths)
            d = torch.as_tensor(np.asarray(dep, dtype=np.float32), device=self.device).broadcast_to(shape)
            d = torch.where(self.masks[i], torch.clamp_min(d, 0.0), torch.zeros((), device=self.device))
            out.append(SWEState(d.contiguous(), torch.zeros(shape, device=self.device),
                                torch.zeros(shape, device=self.device)))
        return out

    def advance_(self, states: list[SWEState], n_steps: int, start_times=None) -> list[tuple]:
        """Advance every member IN PLACE by ``n_steps`` of its own CFL dt.

        Returns one ``(final_time_s, steps_used, ledger)`` per member.
        """
        n = len(self.shapes)
        if len(states) != n:
            raise ValueError(f"expected {n} states, got {len(states)}")
        arr = lambda typ, vals: (typ * n)(*vals)  # noqa: E731
        for st, shape in zip(states, self.shapes):
            for t in st:
                if not (isinstance(t, torch.Tensor) and t.device == self.device and t.dtype == torch.float32
                        and tuple(t.shape) == shape and t.stride(-1) == 1):
                    raise ValueError("advance_ needs device float32 [rows, cols] tensors per member")
        hs = arr(ctypes.c_void_p, [s.h.data_ptr() for s in states])
        hus = arr(ctypes.c_void_p, [s.hu.data_ptr() for s in states])
        hvs = arr(ctypes.c_void_p, [s.hv.data_ptr() for s in states])
        pitches = arr(ctypes.c_int64, [int(s.h.stride(0)) for s in states])
        starts = None if start_times is None else arr(ctypes.c_double, [float(t) for t in start_times])
        res = (_lib.RunResult * n)()
        with torch.cuda.device(self.device):
            rc = self._lib.swe_ensemble_advance(self._handle, hs, hus, hvs, pitches, int(n_steps),
                                                starts, res, _stream(self.device))
        _lib.check(rc, "swe_ensemble_advance")
        return [(float(r.final_time_s), int(r.steps_used), dict(zip(LEDGER_KEYS, list(r.ledger)))) for r in res]

    def advance_to_(self, states: list[SWEState], start_times, target_time_s: float,
                    max_steps: int, dt_logs: list | None = None) -> list[tuple]:
        """Advance every member IN PLACE from its start time to ``target_time_s``.

        At most ``max_steps`` CFL-limited steps per member; 50-step graphs are
        replayed until every member is done.  Returns one
        ``(final_time_s, steps_used, ledger)`` per member; a member stopped
        short by the cap reports where it stopped.  ``dt_logs``: one device
        float64 tensor of at least ``max_steps`` per member, receiving its dts.
        """
        n = len(self.shapes)
        if len(states) != n:
            raise ValueError(f"expected {n} states, got {len(states)}")
        self._check_states(states)
        starts = [float(start_times)] * n if np.isscalar(start_times) else [float(t) for t in start_times]
        arr = lambda typ, vals: (typ * n)(*vals)  # noqa: E731
        logs = None
        if dt_logs is not None:
            if len(dt_logs) != n or not all(t.device == self.device and t.dtype == torch.float64
                                            and t.is_contiguous() and t.numel() >= max_steps for t in dt_logs):
                raise ValueError("dt_logs: one contiguous device float64 tensor of >= max_steps per member")
            logs = arr(ctypes.c_void_p, [t.data_ptr() for t in dt_logs])
        res = (_lib.RunResult * n)()
        with torch.cuda.device(self.device):
            rc = self._lib.swe_ensemble_advance_to(
                self._handle, arr(ctypes.c_void_p, [s.h.data_ptr() for s in states]),
                arr(ctypes.c_void_p, [s.hu.data_ptr() for s in states]),
                arr(ctypes.c_void_p, [s.hv.data_ptr() for s in states]),
                arr(ctypes.c_int64, [int(s.h.stride(0)) for s in states]), arr(ctypes.c_double, starts),
                float(target_time_s), int(max_steps), logs, res, _stream(self.device))
        if rc != _lib.SWE_ERR_MAX_STEPS:
            _lib.check(rc, "swe_ensemble_advance_to")
        return [(float(r.final_time_s), int(r.steps_used), dict(zip(LEDGER_KEYS, list(r.ledger)))) for r in res]

    def _check_states(self, states) -> None:
        for st, shape in zip(states, self.shapes):
            for t in st:
                if not (isinstance(t, torch.Tensor) and t.device == self.device and t.dtype == torch.float32
                        and tuple(t.shape) == shape and t.stride(-1) == 1):
                    raise ValueError("ensemble states must be device float32 [rows, cols] tensors per member")

    def set_rows_per_warp(self, rows: int) -> None:
        with torch.cuda.device(self.device):
            _lib.check(self._lib.swe_ensemble_set_rows_per_warp(self._handle, int(rows)), "set_rows_per_warp")
        self.rows_per_warp = int(rows)

    def set_timing(self, enable: bool = True) -> None:
        _lib.check(self._lib.swe_ensemble_set_timing(self._handle, 1 if enable else 0), "set_timing")

    def last_step_time(self) -> tuple[float, int]:
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        _lib.check(self._lib.swe_ensemble_last_step_time(self._handle, ctypes.byref(ms), ctypes.byref(n)),
                   "last_step_time")
        return float(ms.value), int(n.value)

    def last_launch_count(self) -> int:
        return int(self._lib.swe_ensemble_last_launch_count(self._handle))

    def shape_key(self) -> str:
        text = json.dumps({"shapes": sorted(self.shapes), "arith": self.arithmetic,
                           "device": torch.cuda.get_device_name(self.device)})
        return hashlib.sha1(text.encode()).hexdigest()[:16]

    def autotune(self, states: list[SWEState], candidates=(32, 64, 128, 256), steps: int = 50,
                 cache: pathlib.Path | None = DEFAULT_CACHE) -> int:
        """Pick the rows-per-warp of the work list by timing ``steps`` steps per candidate.

        The members' states are advanced by the tuning steps (pass copies to
        keep them).  The winner is cached in ``cache`` (JSON) per member-shape
        set and device, and reused without timing on later calls.
        """
        key = self.shape_key()
        if cache is not None and cache.exists():
            try:
                known = json.loads(cache.read_text())
                if key in known:
                    self.set_rows_per_warp(int(known[key]["rows_per_warp"]))
                    return self.rows_per_warp
            except (ValueError, KeyError, OSError):
                pass
        timings = {}
        self.set_timing(True)
        for rows in candidates:
            self.set_rows_per_warp(int(rows))
            self.advance_(states, 2)  # warm-up: graph capture, caches
            self.advance_(states, steps)
            ms, n = self.last_step_time()
            timings[int(rows)] = ms / max(n, 1)
        best = min(timings, key=timings.get)
        self.set_rows_per_warp(best)
        if cache is not None:
            try:
                cache.parent.mkdir(parents=True, exist_ok=True)
                known = json.loads(cache.read_text()) if cache.exists() else {}
                known[key] = {"rows_per_warp": best, "ms_per_step": timings}
                cache.write_text(json.dumps(known, indent=1))
            except OSError:
                pass
        return best
