"""The coupling oracle against the reference's own coupling code.

``tests/golden/coupling_ref6.npz`` holds outputs of the reference's
``hybrid/coupled_forecast.py`` (``network_features``,
``apply_residual_correction`` after the clip of ``:199-200``, and
``run_coupled_forecast`` with a linear corrector), executed unmodified with a
NumPy stand-in for jax (``tests/golden/make_coupling_golden.py``; jax is not
installed here).  Bars:

* features: bit for bit;
* correction: within 4 float32 ulp (the reference sums the two volumes in
  float32, the oracle in float64, so the projection scale may differ in its
  last bits);
* forecast: the same physics step count and 2e-6 relative L2 per output
  (float32 clock and NumPy's float32 power in the reference's JAX solver,
  float64 clock and the C library's power in the oracle; measured 3.4e-7).
"""

from __future__ import annotations

import numpy as np

from conftest import golden, max_ulp, rel_l2
from oracle import cport
from oracle import hybrid_numpy as HN
from oracle import swe_numpy as O


def _rate(z, t, times="rain_times", rates="rain_rates", default="default_rain"):
    return float(np.interp(float(t), z[times].astype(np.float64), z[rates].astype(np.float64),
                           left=float(z[default]), right=float(z[default])))


def test_features_equal_the_reference_coupling_code():
    z = golden("coupling_ref6")
    h, hu, hv = z["state"]
    for tag in ("break", "past"):
        f = HN.network_features(h, hu, hv, z["domain_mask"], 1.0e-4, _rate(z, z[f"features_{tag}_time"]),
                                z["terrain_std"], z["roughness_std"], z["state_mean"], z["state_std"],
                                float(z["rain_scale"]))
        np.testing.assert_array_equal(f, z[f"features_{tag}"])


def test_correction_matches_the_reference_coupling_code():
    z = golden("coupling_ref6")
    h, hu, hv = z["state"]
    lim = z["clip_sigma"] * z["residual_std"]
    got = HN.apply_residual_correction(h, hu, hv, z["residual"], z["domain_mask"], 1.0e-4, float(z["relaxation"]),
                                       clip_limits=lim)
    for a, q in zip(got, ("h", "hu", "hv")):
        assert max_ulp(a, z[f"corrected_{q}"]) <= 4, q


def forecast_params(z):
    return O.make_params(z["forecast_bed"], z["forecast_manning_n"], z["forecast_mask"], resolution_m=float(z["dx"]),
                         rainfall_times_s=[0.0, 1000.0], rainfall_rates_m_s=[2.0e-5, 2.0e-5],
                         default_rainfall_m_s=0.0, boundary=tuple(int(b) for b in z["boundary"]))


def test_forecast_matches_the_reference_coupling_code():
    z = golden("coupling_ref6")
    params = forecast_params(z)
    dom = cport.Domain(params)
    st = O.State(*z["forecast_state"])
    times = z["forecast_times"].astype(np.float64)
    lim = np.float32(2.0) * z["forecast_residual_std"]
    total = 0
    out = [st]
    for k in range(1, len(times)):
        f = HN.network_features(*st, params.domain_mask, params.dry_tolerance, 2.0e-5, z["forecast_terrain_std"],
                                z["forecast_roughness_std"], z["forecast_state_mean"], z["forecast_state_std"], 25.0)
        adv, n = HN.advance_physics_to_time(dom, st, times[k - 1], times[k], 400)
        total += n
        r = (f[0] @ z["forecast_W"] + z["forecast_b"]).astype(np.float32)
        st = O.State(*HN.apply_residual_correction(*adv, r, params.domain_mask, params.dry_tolerance, 0.5,
                                                   clip_limits=lim))
        out.append(st)
    assert total == int(z["forecast_steps"])
    for k in range(len(times)):
        for q, name in enumerate(("h", "hu", "hv")):
            assert rel_l2(out[k][q], z[f"forecast_{name}"][k]) < 2e-6, (k, name)
