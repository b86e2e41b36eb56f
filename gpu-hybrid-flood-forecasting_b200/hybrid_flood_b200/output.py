"""Forecast outputs in the reference's common schema, streamed from the device.

The reference converts solver states to one schema shared by all its backends
(``conserved_to_xarray``, ``src/hybrid_flood/structured_io.py:160-209``) and
saves it as NetCDF (``save_netcdf``, ``:212-230``): ``elevation(y, x)`` and
``depth``, ``x_velocity``, ``y_velocity``, ``velocity(time, y, x)``, NaN off the
domain mask, with ``time``/``x``/``y`` coordinates and run attributes.

Here the per-state fields come from ``swe_output_fields`` (one sm_100a kernel,
values equal to the reference's NumPy arrays bit for bit) and are streamed to
the host while the solver goes on: each output time's four planes are copied
into one of two pinned host buffers on a side stream, and the file write of
time k overlaps the device work of time k+1.

The file is NetCDF-3 (64-bit offset) written with ``scipy.io.netcdf_file``:
the image has neither ``netCDF4`` nor ``xarray``, so the variables, dimensions,
coordinates and attributes are the reference's but without zlib compression;
scipy keeps the file's data in host memory until :meth:`ForecastWriter.close`.
"""

from __future__ import annotations

import pathlib
from typing import NamedTuple

import numpy as np
import torch

from . import _lib
from .solver import SWEState, _as_state, _ptr, _stream

FIELDS = ("depth", "x_velocity", "y_velocity", "velocity")


def output_fields(solver, state, out: torch.Tensor | None = None) -> dict:
    """The four schema fields of ``state`` as device tensors ``[rows, cols]`` (NaN off-mask)."""
    st = _as_state(state, solver.device, solver.shape)
    H, W = solver.shape
    if out is None:
        out = torch.empty((4, H, W), dtype=torch.float32, device=solver.device)
    if tuple(out.shape) != (4, H, W) or out.dtype != torch.float32 or not out.is_contiguous():
        raise ValueError(f"out must be a contiguous float32 tensor of shape (4, {H}, {W})")
    with torch.cuda.device(solver.device):
        rc = solver._lib.swe_output_fields(solver._handle, _ptr(st.h), _ptr(st.hu), _ptr(st.hv), int(st.h.stride(0)),
                                           _ptr(out[0]), _ptr(out[1]), _ptr(out[2]), _ptr(out[3]), W,
                                           _stream(solver.device))
    _lib.check(rc, "swe_output_fields")
    return dict(zip(FIELDS, out))


def elevation(solver) -> np.ndarray:
    """Bed elevation with NaN off the domain mask (structured_io.py:185-186)."""
    z = np.array(solver.bed, dtype=np.float32, copy=True)
    z[~solver.domain_mask.cpu().numpy()] = np.nan
    return z


class ForecastWriter:
    """Streams output times of one domain into a common-schema NetCDF file.

    ``append(time_s, state)`` queues the state's fields (kernel + copy to a
    pinned buffer on a side stream) and writes the previously queued time;
    ``close(steps_used)`` writes the last one and the run attributes.
    ``x``/``y`` default to cell centres from 0 with the grid resolution (rows =
    y, northward).
    """

    def __init__(self, path, solver, *, title: str = "B200 shallow-water forecast", backend: str = "b200_cuda",
                 x=None, y=None, crs: str = "", resolution_m: float | None = None) -> None:
        from scipy.io import netcdf_file

        self.solver = solver
        H, W = solver.shape
        dx = float(resolution_m if resolution_m is not None else solver.params.dx)
        self.path = pathlib.Path(path)
        self.path.parent.mkdir(parents=True, exist_ok=True)
        f = netcdf_file(str(self.path), "w", version=2)
        f.title = title
        f.crs = crs
        f.grid_resolution_m = dx
        f.dry_tolerance_m = float(solver.params.dry_tolerance)
        f.numerical_flux = "HLL with hydrostatic reconstruction"
        f.execution_backend = backend
        f.createDimension("time", None)
        f.createDimension("y", H)
        f.createDimension("x", W)
        xs = f.createVariable("x", "f8", ("x",))
        ys = f.createVariable("y", "f8", ("y",))
        xs[:] = np.asarray(x, np.float64) if x is not None else (np.arange(W) + 0.5) * dx
        ys[:] = np.asarray(y, np.float64) if y is not None else (np.arange(H) + 0.5) * dx
        self._time = f.createVariable("time", "f8", ("time",))
        self._time.units = "s"
        ev = f.createVariable("elevation", "f4", ("y", "x"))
        ev[:] = elevation(solver)
        ev.units = "m"
        self._vars = {}
        for name in FIELDS:
            v = f.createVariable(name, "f4", ("time", "y", "x"))
            v.units = "m" if name == "depth" else "m s-1"
            self._vars[name] = v
        self._file = f
        dev = solver.device
        self._stream = torch.cuda.Stream(device=dev)
        self._dev = torch.empty((4, H, W), dtype=torch.float32, device=dev)
        self._host = [torch.empty((4, H, W), dtype=torch.float32).pin_memory() for _ in range(2)]
        self._events = [torch.cuda.Event(), torch.cuda.Event()]
        self._read = torch.cuda.Event()
        self._pending = None  # (slot, time index, time)
        self._n = 0

    def append(self, time_s: float, state) -> None:
        st = SWEState(*(t for t in _as_state(state, self.solver.device, self.solver.shape)))
        slot = self._n % 2
        main = torch.cuda.current_stream(self.solver.device)
        self._stream.wait_stream(main)
        with torch.cuda.stream(self._stream):
            for t in st:
                t.record_stream(self._stream)
            output_fields(self.solver, st, out=self._dev)
            self._read.record(self._stream)
            self._host[slot].copy_(self._dev, non_blocking=True)
            self._events[slot].record(self._stream)
        main.wait_event(self._read)  # the caller may overwrite the state once its fields exist
        self._flush_pending()
        self._pending = (slot, self._n, float(time_s))
        self._n += 1

    def _flush_pending(self) -> None:
        if self._pending is None:
            return
        slot, k, t = self._pending
        self._events[slot].synchronize()
        data = self._host[slot].numpy()
        self._time[k] = t
        for i, name in enumerate(FIELDS):
            self._vars[name][k] = data[i]
        self._pending = None

    def close(self, steps_used: int | None = None) -> pathlib.Path:
        self._flush_pending()
        if steps_used is not None:
            self._file.steps_used = int(steps_used)
        self._file.close()
        return self.path

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        if self._file.fp is not None and not self._file.fp.closed:
            self.close()


class StreamedRun(NamedTuple):
    path: pathlib.Path
    final_time_s: float
    outputs_written: int
    steps_used: int


def run_to_netcdf(solver, initial_state, output_times_s, path, *, max_steps: int = 20_000, **writer_kw) -> StreamedRun:
    """``run`` with every output time streamed to a common-schema file instead of kept on the device.

    Same steps and states as :meth:`B200ShallowWaterSolver.run` (the same float32
    output times, the same clock carried from one output time to the next);
    ``ValueError``/``RuntimeError`` as ``run`` raises them.
    """
    times = np.asarray(output_times_s, dtype=np.float32)
    if times.ndim != 1 or not len(times) or times[0] != 0 or np.any(np.diff(times) <= 0):
        raise ValueError("Output times must be one-dimensional, start at zero, and increase.")
    st = _as_state(initial_state, solver.device, solver.shape)
    cur = SWEState(*(t.clone().contiguous() for t in st))
    writer = ForecastWriter(path, solver, **writer_kw)
    t = float(times[0])
    steps = 0
    try:
        writer.append(t, cur)
        for k in range(1, len(times)):
            target = float(times[k])
            t, n, _ = solver.advance_to_(cur, t, target, max(max_steps - steps, 0))
            steps += n
            if not t >= target - 1.0e-7:
                raise RuntimeError(f"max_steps={max_steps} wrote {k}/{len(times)} outputs; last time={t:.3f} s.")
            writer.append(t, cur)
    except BaseException:
        writer.close(steps)
        raise
    writer.close(steps)
    return StreamedRun(writer.path, t, len(times), steps)


def read_netcdf(path) -> dict:
    """Variables, coordinates and attributes of a file written here, as NumPy arrays."""
    from scipy.io import netcdf_file

    with netcdf_file(str(path), "r", mmap=False) as f:
        out = {name: np.array(v.data) for name, v in f.variables.items()}
        out["attrs"] = {k: (v.decode() if isinstance(v, bytes) else v) for k, v in f._attributes.items()}
    return out
