"""The oracle against the reference's own golden vectors (CPU).

The fixtures in tests/golden were produced by running the UNMODIFIED reference
NumPy solver (tests/golden/make_golden.py).  The NumPy restatement must match
them bit-for-bit; the C restatement bit-for-bit on cases without friction
drift and within a few 1e-6 where its libm powf differs from NumPy's pow by an
ulp.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, golden_params, max_ulp, rel_l2
from oracle import cport
from oracle import swe_numpy as O

RUN_CASES = ["lake_sin2_12", "flat_basin_20", "lake_gauss_20", "mask_walls_12"]


def test_numpy_one_step_is_bit_exact():
    z = golden("one_step_7x9")
    p = golden_params(z)
    s0 = O.State(*z["state0"])
    out = O.finite_volume_step(s0, p, float(z["dt"]), float(z["time_s"]))
    for got, want in zip(out, z["state1"]):
        np.testing.assert_array_equal(got, want)
    assert O.compute_cfl_dt(s0, p) == float(z["cfl_dt0"])


@pytest.mark.parametrize("name", RUN_CASES)
def test_numpy_run_is_bit_exact(name):
    z = golden(name)
    p = golden_params(z)
    r = O.run(O.State(*z["state0"]), p, z["output_times"], max_steps=1000)
    for got, key in zip(r.states, ("out_h", "out_hu", "out_hv")):
        np.testing.assert_array_equal(got, z[key])
    assert r.steps_used == int(z["steps_used"])
    assert r.final_time_s == float(z["final_time_s"])
    assert O.ledger_error(r.ledger) < 1e-6


def test_numpy_wetdry_mask_steps_are_bit_exact():
    z = golden("wetdry_mask_33x47")
    p = golden_params(z)
    st, t = O.State(*z["state0"]), 0.0
    for k in range(40):
        dt = O.compute_cfl_dt(st, p)
        assert dt == z["dts"][k]
        st = O.finite_volume_step(st, p, dt, t)
        t += dt
        if (k + 1) % 10 == 0:
            for got, want in zip(st, z["snaps"][(k + 1) // 10 - 1]):
                np.testing.assert_array_equal(got, want)
    assert t == float(z["final_time_s"])


def test_numpy_tilted_bumps_256_is_bit_exact():
    z = golden("tilted_bumps_256")
    p = golden_params(z)
    init = O.initial_state(p)
    st, t, dts = O.run_steps(init, p, 100)
    np.testing.assert_array_equal(np.asarray(dts), z["dts100"])
    for got, want in zip(st, z["state100"]):
        np.testing.assert_array_equal(got, want)
    r = O.run(init, p, z["output_times"])
    assert r.steps_used == int(z["steps_used"])
    for k in range(3):
        np.testing.assert_array_equal(r.states[k][-1], z["out_final"][k])
    assert O.ledger_error(r.ledger) < 1e-6


def test_ghost_cells_known_answer():
    """Restates tests/test_jax_solver_conservation.py:25-41 of the reference."""
    h = np.ones((2, 2), dtype=np.float32)
    hu = np.array([[1.0, 2.0], [3.0, 4.0]], dtype=np.float32)
    hv = np.array([[5.0, 6.0], [7.0, 8.0]], dtype=np.float32)
    refl = O.ghost_layer(O.State(h, hu, hv), (0, 0, 0, 0))
    opn = O.ghost_layer(O.State(h, hu, hv), (1, 1, 1, 1))
    np.testing.assert_array_equal(refl.hu[1:-1, 0], -hu[:, 0])
    np.testing.assert_array_equal(refl.hu[1:-1, -1], -hu[:, -1])
    np.testing.assert_array_equal(refl.hv[0, 1:-1], -hv[0, :])
    np.testing.assert_array_equal(refl.hv[-1, 1:-1], -hv[-1, :])
    np.testing.assert_array_equal(opn.hu[1:-1, 0], hu[:, 0])
    np.testing.assert_array_equal(opn.hv[0, 1:-1], hv[0, :])


def test_rain_interp_matches_numpy_interp():
    z = golden("wetdry_mask_33x47")
    p = golden_params(z)
    d = cport.Domain(p)
    for t in [-1.0, 0.0, 5.0, 7.5, 20.0, 33.3, 55.0, 60.0, 1e9]:
        assert d.rain_rate(t) == O.rainfall_rate(p, t)


def test_c_oracle_one_step_and_runs_are_bit_exact():
    z = golden("one_step_7x9")
    d = cport.Domain(golden_params(z))
    out = d.step(O.State(*z["state0"]), float(z["dt"]), float(z["time_s"]))
    for got, want in zip(out, z["state1"]):
        np.testing.assert_array_equal(got, want)
    for name in RUN_CASES:
        z = golden(name)
        d = cport.Domain(golden_params(z))
        out, ft, steps, written, ledger = d.run(O.State(*z["state0"]), z["output_times"], max_steps=1000)
        for k, key in enumerate(("out_h", "out_hu", "out_hv")):
            np.testing.assert_array_equal(out[:, k], z[key])
        assert steps == int(z["steps_used"]) and ft == float(z["final_time_s"])


def test_c_oracle_tracks_reference_where_pow_rounds_differently():
    z = golden("wetdry_mask_33x47")
    d = cport.Domain(golden_params(z))
    st, t = O.State(*z["state0"]), 0.0
    for k in range(40):
        dt = d.cfl_dt(st)
        st = d.step(st, dt, t)
        t += dt
    want = z["snaps"][-1]
    for q in range(3):
        np.testing.assert_allclose(st[q], want[q], rtol=1e-4, atol=1e-6)
    z = golden("tilted_bumps_256")
    d = cport.Domain(golden_params(z))
    st, t = O.initial_state(golden_params(z)), 0.0
    for _ in range(100):
        dt = d.cfl_dt(st)
        st = d.step(st, dt, t)
        t += dt
    assert rel_l2(st.h, z["state100"][0]) < 1e-5


def test_c_oracle_matches_numpy_oracle_with_open_boundary_and_fp64():
    from hybrid_flood_b200.workloads import tilted_bumps

    w = tilted_bumps(64, 80, seed=3)
    for dtype in (np.float32, np.float64):
        p = O.make_params(w.bed, w.manning_n, w.domain_mask, dtype=dtype, **w.solver_kwargs())
        init = O.initial_state(p, depth_m=0.05)
        d = cport.Domain(p)
        st_n, st_c, t = init, init, 0.0
        for _ in range(20):
            dt = O.compute_cfl_dt(st_n, p)
            assert d.cfl_dt(st_c) == pytest.approx(dt, rel=1e-5)
            st_n = O.finite_volume_step(st_n, p, dt, t)
            st_c = d.step(st_c, dt, t)
            t += dt
        tol = 1e-5 if dtype is np.float32 else 1e-13
        assert rel_l2(st_c.h, st_n.h) < tol
        assert rel_l2(st_c.hu, st_n.hu) < 10 * tol


def test_ledger_closes_with_open_boundary():
    from hybrid_flood_b200.workloads import tilted_bumps

    w = tilted_bumps(48, 48, seed=5)
    p = O.make_params(w.bed, w.manning_n, w.domain_mask, **w.solver_kwargs())
    init = O.initial_state(p, depth_m=0.2)
    r = O.run(init, p, np.asarray([0.0, 60.0], np.float32))
    assert r.ledger["outflow"] > 0.0
    assert O.ledger_error(r.ledger) < 1e-6
    out, ft, steps, written, ledger = cport.Domain(p).run(init, np.asarray([0.0, 60.0], np.float32))
    assert ledger["outflow"] == pytest.approx(r.ledger["outflow"], rel=1e-4)
    assert O.ledger_error(ledger) < 1e-6


def test_max_steps_raises_like_reference():
    z = golden("flat_basin_20")
    p = golden_params(z)
    with pytest.raises(RuntimeError, match="max_steps"):
        O.run(O.State(*z["state0"]), p, z["output_times"], max_steps=3)
    with pytest.raises(RuntimeError, match="max_steps"):
        cport.Domain(p).run(O.State(*z["state0"]), z["output_times"], max_steps=3)
    with pytest.raises(ValueError):
        O.run(O.State(*z["state0"]), p, np.asarray([1.0, 2.0], np.float32))
