"""Float64 gauge-loss oracle for the adjoint (test infrastructure only).

The loss of a fixed-dt rollout of the oracle step (``oracle/swe_oracle.c`` in
float64, restating ``src/hybrid_flood/numpy_solver/shallow_water_2d.py:277-327``):
mean squared difference between the depth at ``gauge_index`` every
``obs_every`` steps and ``obs``.  Central finite differences of this loss are
the gradient oracle; the reference itself has no gradient to compare against.
"""

from __future__ import annotations

import numpy as np

from . import cport
from .swe_numpy import State, make_params


def rollout_gauges(bed, manning_n, mask, kw: dict, h0, n_steps: int, dt: float, gauge_index,
                   obs_every: int, rain_scale: float = 1.0, start_time_s: float = 0.0,
                   hu0=None, hv0=None, dtype=np.float64) -> np.ndarray:
    """Gauge depths [n_steps // obs_every, n_gauges] of a fixed-dt rollout."""
    kw = dict(kw)
    kw["rainfall_rates_m_s"] = np.asarray(kw["rainfall_rates_m_s"], dtype=np.float64) * rain_scale
    p = make_params(bed, manning_n, mask, dtype=dtype, **kw)
    d = cport.Domain(p)
    h0 = np.asarray(h0, dtype=dtype)
    st = State(h0, np.zeros_like(h0) if hu0 is None else np.asarray(hu0, dtype),
               np.zeros_like(h0) if hv0 is None else np.asarray(hv0, dtype))
    obs = []
    t = start_time_s
    for k in range(n_steps):
        st = d.step(st, dt, t)
        t += dt
        if (k + 1) % obs_every == 0:
            obs.append(st.h.reshape(-1)[gauge_index].copy())
    return np.stack(obs)


def gauge_mse(pred: np.ndarray, obs: np.ndarray) -> float:
    return float(np.mean((pred - obs) ** 2))
