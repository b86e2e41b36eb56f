"""ctypes wrapper of the C oracle (``oracle/swe_oracle.c``).

TEST INFRASTRUCTURE ONLY -- the checker for sizes the NumPy restatement is too
slow for, and the timed CPU baseline ("port").  Same semantics as
:mod:`oracle.swe_numpy` (which is pinned against the reference's golden
fixtures); float32 results agree with it bit-for-bit except where the friction
``pow`` differs by an ulp.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build
from .swe_numpy import Params, State

_LIB = None


class _Domain(ctypes.Structure):
    _fields_ = [
        ("rows", ctypes.c_int64), ("cols", ctypes.c_int64),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("g", ctypes.c_double),
        ("cfl", ctypes.c_double), ("dry", ctypes.c_double), ("max_dt", ctypes.c_double),
        ("default_rain", ctypes.c_double),
        ("boundary", ctypes.c_int32 * 4), ("n_rain", ctypes.c_int32), ("pad_", ctypes.c_int32),
        ("rain_times", ctypes.c_void_p), ("rain_rates", ctypes.c_void_p),
        ("bed", ctypes.c_void_p), ("manning", ctypes.c_void_p), ("mask", ctypes.c_void_p),
        ("mult", ctypes.c_void_p),
    ]


def lib():
    """Load (building first if needed) the oracle shared library."""
    global _LIB
    if _LIB is None:
        path = _build.build()
        _LIB = ctypes.CDLL(str(path))
        for prec in ("f32", "f64"):
            getattr(_LIB, f"oracle_step_{prec}").restype = ctypes.c_int
            getattr(_LIB, f"oracle_max_inverse_dt_{prec}").restype = ctypes.c_double
            getattr(_LIB, f"oracle_cfl_dt_{prec}").restype = ctypes.c_double
            getattr(_LIB, f"oracle_rain_rate_{prec}").restype = ctypes.c_double
            getattr(_LIB, f"oracle_volume_{prec}").restype = ctypes.c_double
            getattr(_LIB, f"oracle_run_{prec}").restype = ctypes.c_int
        _LIB.oracle_max_threads.restype = ctypes.c_int
    return _LIB


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


class Domain:
    """Oracle domain built from :class:`oracle.swe_numpy.Params` (keeps its arrays alive)."""

    def __init__(self, params: Params):
        self.params = params
        dt_ = np.dtype(params.dtype)
        if dt_ not in (np.dtype(np.float32), np.dtype(np.float64)):
            raise ValueError("oracle precision must be float32 or float64")
        self.prec = "f32" if dt_ == np.float32 else "f64"
        self.dtype = dt_
        c = lambda a: np.ascontiguousarray(a, dtype=dt_)  # noqa: E731
        self._keep = [
            c(params.rainfall_times_s), c(params.rainfall_rates_m_s), c(params.bed),
            c(params.manning_n), np.ascontiguousarray(params.domain_mask, dtype=np.uint8),
            c(params.rainfall_multiplier),
        ]
        rt, rr, bed, man, mask, mult = self._keep
        d = _Domain()
        d.rows, d.cols = bed.shape
        d.dx, d.dy, d.g = params.dx, params.dy, params.gravity
        d.cfl, d.dry, d.max_dt = params.cfl, params.dry_tolerance, params.max_dt
        d.default_rain = params.default_rainfall_m_s
        d.boundary[:] = list(params.boundary)
        d.n_rain = rt.size
        d.rain_times, d.rain_rates = _ptr(rt), _ptr(rr)
        d.bed, d.manning, d.mask, d.mult = _ptr(bed), _ptr(man), _ptr(mask), _ptr(mult)
        self._d = d
        self._fn = lambda name: getattr(lib(), f"oracle_{name}_{self.prec}")

    def _state(self, state):
        return [np.ascontiguousarray(a, dtype=self.dtype) for a in state]

    def step(self, state: State, dt: float, time_s: float, terms: np.ndarray | None = None) -> State:
        h, hu, hv = self._state(state)
        out = [np.empty_like(h) for _ in range(3)]
        tp = None if terms is None else _ptr(terms)
        self._fn("step")(ctypes.byref(self._d), _ptr(h), _ptr(hu), _ptr(hv), *map(_ptr, out),
                         ctypes.c_double(dt), ctypes.c_double(time_s), tp)
        return State(*out)

    def max_inverse_dt(self, state: State) -> float:
        h, hu, hv = self._state(state)
        return float(self._fn("max_inverse_dt")(ctypes.byref(self._d), _ptr(h), _ptr(hu), _ptr(hv)))

    def cfl_dt(self, state: State) -> float:
        h, hu, hv = self._state(state)
        return float(self._fn("cfl_dt")(ctypes.byref(self._d), _ptr(h), _ptr(hu), _ptr(hv)))

    def rain_rate(self, time_s: float) -> float:
        return float(self._fn("rain_rate")(ctypes.byref(self._d), ctypes.c_double(time_s)))

    def run(self, initial: State, output_times_s, *, max_steps: int = 20_000):
        """Adaptive run; returns ``(states[n_out,3,H,W], final_time, steps, written, ledger)``."""
        times = np.ascontiguousarray(output_times_s, dtype=np.float32)
        if times.ndim != 1 or not len(times) or times[0] != 0 or np.any(np.diff(times) <= 0):
            raise ValueError("Output times must be one-dimensional, start at zero, and increase.")
        h, hu, hv = self._state(initial)
        out = np.empty((len(times), 3, *h.shape), dtype=self.dtype)
        ft = ctypes.c_double()
        steps = ctypes.c_int()
        written = ctypes.c_int()
        ledger = np.zeros(6, dtype=np.float64)
        rc = self._fn("run")(ctypes.byref(self._d), _ptr(h), _ptr(hu), _ptr(hv), _ptr(times),
                             ctypes.c_int(len(times)), ctypes.c_int(max_steps), _ptr(out),
                             ctypes.byref(ft), ctypes.byref(steps), ctypes.byref(written),
                             _ptr(ledger))
        if rc != 0:
            raise RuntimeError(
                f"max_steps={max_steps} wrote {written.value}/{len(times)} outputs; "
                f"last time={ft.value:.3f} s."
            )
        names = ("volume0", "volume", "rain_in", "outflow", "clip_gain", "mask_loss")
        return out, ft.value, steps.value, written.value, dict(zip(names, ledger.tolist()))


def default_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
