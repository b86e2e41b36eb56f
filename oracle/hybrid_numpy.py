"""NumPy restatement of the reference's physics-AI coupling pieces (test oracle).

TEST INFRASTRUCTURE ONLY.  Restates, in float32 NumPy with the reference's
operation order, ``src/hybrid_flood/hybrid/coupled_forecast.py``:

* ``:49-50``   ``_velocity``
* ``:53-79``   ``network_features`` (six standardised channels, NHWC)
* ``:82-120``  ``apply_residual_correction`` (relaxation, positivity clip,
  projection back to the physics step's water volume, momentum rebuilt on wet
  cells), with the clip of ``:199-200`` applied first
* ``:123-161`` ``advance_physics_to_time`` and ``:164-225``
  ``run_coupled_forecast`` (physics from ``swe_numpy.run_steps`` semantics,
  float64 clock)

The volume sums are taken in float64 here (the reference's ``jnp.sum`` of a
float32 array accumulates pairwise in float32); the tests' tolerances allow for
that.
"""

from __future__ import annotations

import numpy as np

M_S_TO_MM_HR = 3.6e6  # coupled_forecast.py:27


def _velocity(m, h, dry):
    out = np.zeros_like(m)
    np.divide(m, np.maximum(h, np.float32(dry)), out=out, where=h > np.float32(dry))
    return out


def network_features(h, hu, hv, mask, dry, rain_rate_m_s, terrain_std, roughness_std,
                     state_mean, state_std, rainfall_scale_mm_hr):
    """[1, H, W, 6]: (h, u, v) standardised and masked, rain / scale, terrain, roughness."""
    u = _velocity(hu, h, dry)
    v = _velocity(hv, h, dry)
    dyn = np.stack((h, u, v), axis=-1).astype(np.float32)
    dyn = (dyn - np.asarray(state_mean, np.float32)) / np.asarray(state_std, np.float32)
    dyn = np.where(mask[..., None], dyn, np.float32(0.0))
    rain = np.full_like(h, np.float32(rain_rate_m_s * M_S_TO_MM_HR) / np.float32(rainfall_scale_mm_hr))
    feats = np.concatenate((dyn, rain[..., None], terrain_std[..., None].astype(np.float32),
                            roughness_std[..., None].astype(np.float32)), axis=-1)
    return feats[None].astype(np.float32)


def state5_features(h, hu, hv, bed, mask, rain_mm_hr, mean, std):
    """[1, H, W, 5]: (h, hu, hv, bed, rain in mm/h), each standardised, zero off-mask.

    The input layout of the 4-level, 5-channel corrector (no reference counterpart:
    the reference network takes :func:`network_features`)."""
    src = np.stack((h, hu, hv, bed, np.full_like(h, np.float32(rain_mm_hr))), axis=-1).astype(np.float32)
    f = (src - np.asarray(mean, np.float32)) / np.asarray(std, np.float32)
    return np.where(mask[..., None], f, np.float32(0.0))[None].astype(np.float32)


def clip_residual(residual, limits):
    """``jnp.clip(residual, -limits, limits)`` per channel (coupled_forecast.py:199-200)."""
    if limits is None:
        return residual
    lim = np.asarray(limits, np.float32)[: residual.shape[-1]]
    return np.clip(residual, -lim, lim).astype(np.float32)


def apply_residual_correction(h, hu, hv, residual, mask, dry, relaxation, clip_limits=None):
    """Corrected (h, hu, hv); ``residual`` is [H, W, 3] (depth, u, v) or [H, W, 1] (depth)."""
    residual = clip_residual(np.asarray(residual, np.float32), clip_limits)
    r = np.float32(relaxation)
    u = _velocity(hu, h, dry)
    v = _velocity(hv, h, dry)
    prov = np.where(mask, np.maximum(h + r * residual[..., 0], np.float32(0.0)), np.float32(0.0))
    target = float(np.where(mask, h, 0.0).astype(np.float64).sum())
    provisional = float(prov.astype(np.float64).sum())
    eps = float(np.finfo(np.float32).eps)
    scale = np.float32(target / provisional) if provisional > eps else np.float32(1.0)
    ch = (prov * scale).astype(np.float32) if target > eps else h
    if residual.shape[-1] >= 3:
        u = u + r * residual[..., 1]
        v = v + r * residual[..., 2]
    wet = mask & (ch > np.float32(dry))
    return ch, np.where(wet, ch * u, np.float32(0.0)), np.where(wet, ch * v, np.float32(0.0))


def advance_physics_to_time(stepper, state, start_time_s, target_time_s, max_substeps):
    """Adaptive steps to one correction time (coupled_forecast.py:123-161).

    ``stepper`` has ``cfl_dt(state)`` and ``step(state, dt, t)`` (``cport.Domain``).
    The clock is float64 as in the NumPy run loop.  Returns (state, steps);
    the state is NaN-filled when the target was not reached within 1e-6 s.
    """
    t = float(start_time_s)
    target = float(target_time_s)
    steps = 0
    while steps < max_substeps and t < target - 1.0e-7:
        dt = min(stepper.cfl_dt(state), target - t)
        state = stepper.step(state, dt, t)
        t += dt
        steps += 1
    if not t >= target - 1.0e-6:
        state = type(state)(*(np.full_like(a, np.nan) for a in state))
    return state, steps
