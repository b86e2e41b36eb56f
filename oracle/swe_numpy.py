"""NumPy restatement of the reference shallow-water finite-volume step (test oracle).

TEST INFRASTRUCTURE ONLY -- imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py``; never by the product package.

What it restates (paths are inside the reference project):

* ``src/hybrid_flood/numpy_solver/shallow_water_2d.py:60-63``  safe velocity
* ``.../shallow_water_2d.py:66-135``   HLL flux in x and y
* ``.../shallow_water_2d.py:138-239``  wall mirroring at active/inactive faces,
  hydrostatic reconstruction, side-specific pressure corrections
* ``.../shallow_water_2d.py:242-251``  ghost layer (edge copy, normal momentum
  negated); generalised to per-side codes as in
  ``src/hybrid_flood/jax_solver/boundary_conditions.py:29-52`` (0 reflective,
  1 open = zero-gradient copy), ordered left, right, bottom, top
* ``.../shallow_water_2d.py:254-264``  rainfall interpolation (``np.interp``)
* ``.../shallow_water_2d.py:267-274``  CFL time step
* ``.../shallow_water_2d.py:277-327``  the step (divergence, rain, positivity
  clip, semi-implicit Manning friction, wet/dry masking)
* ``.../shallow_water_2d.py:333-424``  solver constructor, ``initial_state`` and
  the adaptive ``run`` loop to fixed output times

The code is organised differently from the reference (one axis-generic face
routine instead of two mirrored ones) but performs the same floating-point
operations in the same order, so at float32 it is bit-identical to the
reference: scalar controls stay Python floats, so NumPy's weak-scalar rule
rounds them to float32 exactly where the reference's do, while ``dt * rate``
and ``dt * gravity`` are formed in float64 first, as in the reference.  With
``dtype=np.float64`` the whole step runs in double precision (the reference
hard-casts to float32 and cannot do that).

It adds an FP64 mass ledger that the reference lacks (rain in, boundary
outflow, positivity-clip gain, masked-cell removal), built on the mass-balance
identity of ``src/hybrid_flood/anuga_solver/run_simulation.py:100-116``.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import NamedTuple

import numpy as np

REFLECTIVE = 0
OPEN = 1


class State(NamedTuple):
    """Conserved cell averages ``(h, hu, hv)`` as ``[rows=y, cols=x]`` arrays."""

    h: np.ndarray
    hu: np.ndarray
    hv: np.ndarray


class Result(NamedTuple):
    """Output of :func:`run` (fields of the reference ``NumpyResult`` + ledger)."""

    states: State
    output_times_s: np.ndarray
    final_time_s: float
    outputs_written: int
    steps_used: int
    ledger: dict


@dataclass(frozen=True)
class Params:
    """Static fields and scalar controls (reference ``NumpyParams`` + boundary codes)."""

    bed: np.ndarray
    manning_n: np.ndarray
    domain_mask: np.ndarray
    rainfall_multiplier: np.ndarray
    rainfall_times_s: np.ndarray
    rainfall_rates_m_s: np.ndarray
    default_rainfall_m_s: float
    dx: float
    dy: float
    gravity: float
    cfl: float
    dry_tolerance: float
    max_dt: float
    boundary: tuple = (REFLECTIVE, REFLECTIVE, REFLECTIVE, REFLECTIVE)
    dtype: type = np.float32


def make_params(
    bed,
    manning_n,
    domain_mask,
    *,
    resolution_m: float,
    rainfall_times_s,
    rainfall_rates_m_s,
    default_rainfall_m_s: float = 0.0,
    rainfall_multiplier=None,
    boundary=(REFLECTIVE, REFLECTIVE, REFLECTIVE, REFLECTIVE),
    gravity_m_s2: float = 9.81,
    cfl: float = 0.45,
    dry_tolerance_m: float = 1.0e-4,
    max_dt_s: float = 10.0,
    dtype=np.float32,
) -> Params:
    """Cast inputs the way the reference constructor does (``shallow_water_2d.py:348-365``)."""
    shape = np.asarray(bed).shape
    if np.asarray(manning_n).shape != shape or np.asarray(domain_mask).shape != shape:
        raise ValueError("Bed, roughness, and domain mask must have identical shapes.")
    mask = np.asarray(domain_mask, dtype=bool)
    multiplier = mask if rainfall_multiplier is None else rainfall_multiplier
    if np.asarray(multiplier).shape != shape:
        raise ValueError("Rainfall multiplier must match the grid shape.")
    codes = tuple(int(c) for c in boundary)
    if len(codes) != 4 or any(c not in (REFLECTIVE, OPEN) for c in codes):
        raise ValueError("boundary must hold four codes (left, right, bottom, top), each 0 or 1.")
    return Params(
        bed=np.asarray(bed, dtype=dtype),
        manning_n=np.asarray(manning_n, dtype=dtype),
        domain_mask=mask,
        rainfall_multiplier=np.asarray(multiplier, dtype=dtype),
        rainfall_times_s=np.asarray(rainfall_times_s, dtype=dtype),
        rainfall_rates_m_s=np.asarray(rainfall_rates_m_s, dtype=dtype),
        default_rainfall_m_s=float(default_rainfall_m_s),
        dx=float(resolution_m),
        dy=float(resolution_m),
        gravity=float(gravity_m_s2),
        cfl=float(cfl),
        dry_tolerance=float(dry_tolerance_m),
        max_dt=float(max_dt_s),
        boundary=codes,
        dtype=dtype,
    )


def initial_state(params: Params, *, depth_m=0.0, x_velocity_m_s=0.0, y_velocity_m_s=0.0) -> State:
    """Masked conserved fields from depth and velocity (``shallow_water_2d.py:367-380``)."""
    shape = params.bed.shape
    dt_ = params.dtype
    depth = np.broadcast_to(np.asarray(depth_m, dtype=dt_), shape).copy()
    u = np.broadcast_to(np.asarray(x_velocity_m_s, dtype=dt_), shape)
    v = np.broadcast_to(np.asarray(y_velocity_m_s, dtype=dt_), shape)
    depth = np.where(params.domain_mask, np.maximum(depth, 0.0), 0.0).astype(dt_)
    return State(depth, (depth * u).astype(dt_), (depth * v).astype(dt_))


def _velocity(momentum: np.ndarray, depth: np.ndarray, dry: float) -> np.ndarray:
    """``m / max(h, dry)`` where ``h > dry`` else 0 (``shallow_water_2d.py:60-63``)."""
    out = np.zeros_like(momentum)
    np.divide(momentum, np.maximum(depth, dry), out=out, where=depth > dry)
    return out


def ghost_layer(state: State, boundary) -> State:
    """One ghost ring: edge copy, normal momentum negated on reflective sides.

    Follows ``jax_solver/boundary_conditions.py:29-52`` (which the NumPy
    reference hard-codes to all-reflective at ``shallow_water_2d.py:242-251``).
    """
    h = np.pad(state.h, 1, mode="edge")
    hu = np.pad(state.hu, 1, mode="edge")
    hv = np.pad(state.hv, 1, mode="edge")
    left, right, bottom, top = boundary
    if left == REFLECTIVE:
        hu[:, 0] = -hu[:, 1]
    if right == REFLECTIVE:
        hu[:, -1] = -hu[:, -2]
    if bottom == REFLECTIVE:
        hv[0] = -hv[1]
    if top == REFLECTIVE:
        hv[-1] = -hv[-2]
    return State(h, hu, hv)


def _hll(lo, hi, axis: int, g: float, dry: float):
    """HLL flux between reconstructed states ``(H, Hu, Hv)`` (``shallow_water_2d.py:66-135``).

    ``axis`` 1 is an x-face (normal momentum ``Hu``), 0 a y-face (``Hv``).  The
    velocities are recomputed from the reconstructed momenta, as the reference
    does.  The tangential flux is ``Hu * v`` on both axes (``:84`` and ``:120``).
    """
    H0, X0, Y0 = lo
    H1, X1, Y1 = hi
    n0, n1 = (X0, X1) if axis == 1 else (Y0, Y1)
    un0 = _velocity(n0, H0, dry)
    un1 = _velocity(n1, H1, dry)
    c0 = np.sqrt(g * np.maximum(H0, 0.0))
    c1 = np.sqrt(g * np.maximum(H1, 0.0))
    s0 = np.minimum(un0 - c0, un1 - c1)
    s1 = np.maximum(un0 + c0, un1 + c1)
    p0 = 0.5 * g * H0**2
    p1 = 0.5 * g * H1**2
    if axis == 1:
        f0 = (X0, X0 * un0 + p0, X0 * _velocity(Y0, H0, dry))
        f1 = (X1, X1 * un1 + p1, X1 * _velocity(Y1, H1, dry))
    else:
        f0 = (Y0, X0 * un0, Y0 * un0 + p0)
        f1 = (Y1, X1 * un1, Y1 * un1 + p1)
    u0 = (H0, X0, Y0)
    u1 = (H1, X1, Y1)
    spread = s1 - s0
    den = np.where(spread > 1.0e-12, spread, 1.0)
    flux = []
    for k in range(3):
        middle = (s1 * f0[k] - s0 * f1[k] + (s0 * s1) * (u1[k] - u0[k])) / den
        flux.append(np.where(s0 >= 0.0, f0[k], np.where(s1 <= 0.0, f1[k], middle)))
    return flux


def face_fluxes(h, hu, hv, bed, active, axis: int, g: float, dry: float):
    """Side-specific fluxes on every face along ``axis`` (``shallow_water_2d.py:138-239``).

    Returns ``(lo_side, hi_side)``: three flux components each, the flux seen by
    the lower-index cell and by the higher-index cell of the face.  They differ
    only in the normal-momentum pressure correction.
    """
    if axis == 1:
        lo_ix, hi_ix = (slice(None), slice(None, -1)), (slice(None), slice(1, None))
    else:
        lo_ix, hi_ix = (slice(None, -1), slice(None)), (slice(1, None), slice(None))
    lo = [np.array(a[lo_ix]) for a in (h, hu, hv, bed)]
    hi = [np.array(a[hi_ix]) for a in (h, hu, hv, bed)]
    act_lo, act_hi = active[lo_ix], active[hi_ix]
    normal = 1 if axis == 1 else 2
    # Solid wall where exactly one side is active: mirror the active side onto
    # the inactive one and negate the normal momentum.
    hi_wall = act_lo & ~act_hi
    lo_wall = ~act_lo & act_hi
    for k in range(4):
        hi[k][hi_wall] = -lo[k][hi_wall] if k == normal else lo[k][hi_wall]
        lo[k][lo_wall] = -hi[k][lo_wall] if k == normal else hi[k][lo_wall]
    bed_face = np.maximum(lo[3], hi[3])
    H_lo = np.maximum(lo[0] + lo[3] - bed_face, 0.0)
    H_hi = np.maximum(hi[0] + hi[3] - bed_face, 0.0)
    u_lo, v_lo = _velocity(lo[1], lo[0], dry), _velocity(lo[2], lo[0], dry)
    u_hi, v_hi = _velocity(hi[1], hi[0], dry), _velocity(hi[2], hi[0], dry)
    flux = _hll(
        (H_lo, H_lo * u_lo, H_lo * v_lo),
        (H_hi, H_hi * u_hi, H_hi * v_hi),
        axis,
        g,
        dry,
    )
    relevant = act_lo | act_hi
    flux = [np.where(relevant, f, 0.0) for f in flux]
    corr_lo = np.where(relevant, 0.5 * g * (lo[0] ** 2 - H_lo**2), 0.0)
    corr_hi = np.where(relevant, 0.5 * g * (hi[0] ** 2 - H_hi**2), 0.0)
    lo_side = [f + (corr_lo if k == normal else 0.0) for k, f in enumerate(flux)]
    hi_side = [f + (corr_hi if k == normal else 0.0) for k, f in enumerate(flux)]
    return lo_side, hi_side


def rainfall_rate(params: Params, time_s: float) -> float:
    """Uniform rain rate at ``time_s`` in m/s (``shallow_water_2d.py:254-264``)."""
    return float(
        np.interp(
            time_s,
            params.rainfall_times_s,
            params.rainfall_rates_m_s,
            left=params.default_rainfall_m_s,
            right=params.default_rainfall_m_s,
        )
    )


def max_inverse_dt(state: State, params: Params) -> float:
    """Largest ``(|u|+c)/dx + (|v|+c)/dy`` over active cells (``shallow_water_2d.py:269-273``)."""
    dry = params.dry_tolerance
    u = _velocity(state.hu, state.h, dry)
    v = _velocity(state.hv, state.h, dry)
    wave = np.sqrt(params.gravity * np.maximum(state.h, 0.0))
    inverse = (np.abs(u) + wave) / params.dx + (np.abs(v) + wave) / params.dy
    return float(np.max(np.where(params.domain_mask, inverse, 0.0)))


def compute_cfl_dt(state: State, params: Params) -> float:
    """CFL time step (``shallow_water_2d.py:267-274``)."""
    maximum = max_inverse_dt(state, params)
    return min(params.cfl / maximum, params.max_dt) if maximum > 0.0 else params.max_dt


def finite_volume_step(state: State, params: Params, dt: float, time_s: float, *, terms=None) -> State:
    """Advance one HLL step (``shallow_water_2d.py:277-327``).

    If ``terms`` is a dict, the FP64 ledger increments of this step (m^3) are
    added into it: ``rain_in``, ``outflow``, ``clip_gain``, ``mask_loss``.
    """
    dt = float(dt)
    time_s = float(time_s)
    g, dry = params.gravity, params.dry_tolerance
    ghost = ghost_layer(state, params.boundary)
    bed_g = np.pad(params.bed, 1, mode="edge")
    act_g = np.pad(params.domain_mask, 1, mode="edge")
    x_lo, x_hi = face_fluxes(
        ghost.h[1:-1], ghost.hu[1:-1], ghost.hv[1:-1], bed_g[1:-1], act_g[1:-1], 1, g, dry
    )
    y_lo, y_hi = face_fluxes(
        ghost.h[:, 1:-1], ghost.hu[:, 1:-1], ghost.hv[:, 1:-1], bed_g[:, 1:-1], act_g[:, 1:-1],
        0, g, dry,
    )
    updated = []
    for k, value in enumerate(state):
        div_x = (x_lo[k][:, 1:] - x_hi[k][:, :-1]) / params.dx
        div_y = (y_lo[k][1:] - y_hi[k][:-1]) / params.dy
        updated.append(value - dt * (div_x + div_y))
    rain = dt * rainfall_rate(params, time_s) * params.rainfall_multiplier
    updated[0] = updated[0] + rain
    h = np.maximum(updated[0], 0.0)
    hu, hv = updated[1], updated[2]
    norm = np.hypot(hu, hv)
    den = 1.0 + (dt * g * params.manning_n**2 * norm / np.maximum(h, dry) ** (7.0 / 3.0))
    hu = hu / den
    hv = hv / den
    mask = params.domain_mask
    wet = mask & (h > dry)
    out = State(
        np.where(mask, h, 0.0).astype(params.dtype),
        np.where(wet, hu, 0.0).astype(params.dtype),
        np.where(wet, hv, 0.0).astype(params.dtype),
    )
    if terms is not None:
        area = params.dx * params.dy
        # Mass through the outer faces: x faces carry F0 * dy, y faces F0 * dx.
        fx, fy = x_lo[0].astype(np.float64), y_lo[0].astype(np.float64)
        out_x = fx[:, -1].sum() - fx[:, 0].sum()
        out_y = fy[-1, :].sum() - fy[0, :].sum()
        terms["rain_in"] = terms.get("rain_in", 0.0) + float(rain.astype(np.float64).sum()) * area
        terms["outflow"] = terms.get("outflow", 0.0) + dt * (out_x * params.dy + out_y * params.dx)
        terms["clip_gain"] = terms.get("clip_gain", 0.0) + float(
            np.maximum(-updated[0], 0.0).astype(np.float64).sum()
        ) * area
        terms["mask_loss"] = terms.get("mask_loss", 0.0) + float(
            h[~mask].astype(np.float64).sum()
        ) * area
    return out


def stored_volume(state: State, params: Params) -> float:
    """FP64 water volume over active cells (m^3), as ``hybrid/rollout.py:318-321``."""
    return float(state.h[params.domain_mask].astype(np.float64).sum()) * params.dx * params.dy


def ledger_error(ledger: dict) -> float:
    """Relative closing error of the FP64 ledger.

    ``V - (V0 + rain_in - outflow + clip_gain - mask_loss)`` divided by the
    gross volume moved, following the form of
    ``anuga_solver/run_simulation.py:100-116``.
    """
    expected = (
        ledger["volume0"] + ledger["rain_in"] - ledger["outflow"] + ledger["clip_gain"]
        - ledger["mask_loss"]
    )
    scale = max(abs(ledger["volume0"]) + abs(ledger["rain_in"]) + abs(ledger["outflow"]), 1e-300)
    return abs(ledger["volume"] - expected) / scale


def run(initial: State, params: Params, output_times_s, *, max_steps: int = 20_000) -> Result:
    """Adaptive loop to fixed output times (``shallow_water_2d.py:382-424``)."""
    times = np.asarray(output_times_s, dtype=np.float32)
    if times.ndim != 1 or not len(times) or times[0] != 0 or np.any(np.diff(times) <= 0):
        raise ValueError("Output times must be one-dimensional, start at zero, and increase.")
    shape = (len(times), *initial.h.shape)
    out = [np.zeros(shape, dtype=params.dtype) for _ in range(3)]
    for k in range(3):
        out[k][0] = initial[k]
    state = initial
    time_s = float(times[0])
    index = 1
    steps = 0
    terms: dict = {}
    volume0 = stored_volume(initial, params)
    while index < len(times) and steps < max_steps:
        target = float(times[index])
        dt = min(compute_cfl_dt(state, params), target - time_s)
        state = finite_volume_step(state, params, dt, time_s, terms=terms)
        time_s += dt
        steps += 1
        if time_s >= target - 1.0e-7:
            for k in range(3):
                out[k][index] = state[k]
            index += 1
    if index != len(times):
        raise RuntimeError(
            f"max_steps={max_steps} wrote {index}/{len(times)} outputs; last time={time_s:.3f} s."
        )
    ledger = {
        "volume0": volume0,
        "volume": stored_volume(state, params),
        "rain_in": terms.get("rain_in", 0.0),
        "outflow": terms.get("outflow", 0.0),
        "clip_gain": terms.get("clip_gain", 0.0),
        "mask_loss": terms.get("mask_loss", 0.0),
    }
    return Result(State(*out), times, time_s, index, steps, ledger)


def run_steps(initial: State, params: Params, n_steps: int, *, start_time_s: float = 0.0):
    """``n_steps`` CFL-limited steps with no output target (dt = CFL dt).

    Returns ``(state, time_s, dts)``.  Used for "after N steps" parity checks.
    """
    state = initial
    time_s = float(start_time_s)
    dts = []
    for _ in range(n_steps):
        dt = compute_cfl_dt(state, params)
        state = finite_volume_step(state, params, dt, time_s)
        time_s += dt
        dts.append(dt)
    return state, time_s, dts
