"""Parity of the sm_100a step (through the C ABI) with the reference and the oracle.

Tolerances (stated per test):
* exact arithmetic: bit-identical wherever the friction term is inactive
  (no velocity or n = 0); elsewhere within the drift that the one operation
  computed differently -- pow in the friction denominator, which differs from
  NumPy's pow by about an ulp -- produces, the same drift the C oracle shows.
* fast arithmetic: the reference's own NumPy-vs-JAX step tolerance
  (rtol 2e-5, atol 2e-7, tests/test_v1_v2_architecture.py:104) for one step and
  the headline bars for runs: relative L2 depth error <= 1e-5 after 100 steps
  and <= 1e-3 at the end of the run.
"""

from __future__ import annotations

import pathlib

import numpy as np
import pytest
import torch

from conftest import golden, golden_params, golden_solver_kwargs, max_ulp, rel_l2
from oracle import cport
from oracle import swe_numpy as O

pytestmark = pytest.mark.gpu

MODES = ["exact", "fast"]
RUN_CASES = ["lake_sin2_12", "flat_basin_20", "lake_gauss_20", "mask_walls_12"]


def _solver(z, mode, **kw):
    from hybrid_flood_b200.solver import B200ShallowWaterSolver

    return B200ShallowWaterSolver(z["bed"], z["manning_n"], z["domain_mask"],
                                  **golden_solver_kwargs(z, **kw), arithmetic=mode)


def _np(state):
    return [t.detach().cpu().numpy() for t in state]


@pytest.mark.parametrize("mode", MODES)
def test_one_step_matches_reference(cuda_device, mode):
    z = golden("one_step_7x9")
    s = _solver(z, mode)
    st = [torch.from_numpy(a).to(cuda_device) for a in z["state0"]]
    out = _np(s.step(st, float(z["dt"]), float(z["time_s"])))
    for got, want in zip(out, z["state1"]):
        if mode == "exact":
            np.testing.assert_allclose(got, want, rtol=2e-6, atol=1e-9)
        else:
            np.testing.assert_allclose(got, want, rtol=2e-5, atol=2e-7)
    dt = s.cfl_dt(st)
    if mode == "exact":
        assert dt == float(z["cfl_dt0"])
    else:
        assert dt == pytest.approx(float(z["cfl_dt0"]), rel=1e-5)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", RUN_CASES)
def test_run_matches_reference(cuda_device, mode, name):
    z = golden(name)
    s = _solver(z, mode)
    r = s.run([a for a in z["state0"]], z["output_times"], max_steps=1000)
    got = _np(r.states)
    for g, key in zip(got, ("out_h", "out_hu", "out_hv")):
        if mode == "exact":
            np.testing.assert_array_equal(g, z[key])  # friction inactive: bit-identical
        else:
            np.testing.assert_allclose(g, z[key], rtol=2e-5, atol=2e-6)
    assert r.outputs_written == len(z["output_times"])
    if mode == "exact":
        assert r.steps_used == int(z["steps_used"])
        assert r.final_time_s == float(z["final_time_s"])
    else:
        assert abs(r.steps_used - int(z["steps_used"])) <= 1
        assert r.final_time_s == pytest.approx(float(z["final_time_s"]), abs=1e-6)
    from hybrid_flood_b200.solver import ledger_error

    assert ledger_error(r.ledger) < 1e-6


@pytest.mark.parametrize("mode", MODES)
def test_wetdry_mask_steps_track_reference(cuda_device, mode):
    z = golden("wetdry_mask_33x47")
    s = _solver(z, mode)
    st = [torch.from_numpy(a).to(cuda_device) for a in z["state0"]]
    t = 0.0
    for k in range(40):
        dt = s.cfl_dt(st)
        if mode == "exact" and k < 5:
            assert dt == z["dts"][k]
        st = s.step(st, dt, t)
        t += dt
    got = _np(st)
    want = z["snaps"][-1]
    assert rel_l2(got[0], want[0]) < 1e-5
    for q in range(3):
        np.testing.assert_allclose(got[q], want[q], rtol=1e-3, atol=1e-5)


@pytest.mark.parametrize("mode", MODES)
def test_tilted_bumps_256_reference_bars(cuda_device, mode):
    """<= 1e-5 relative L2 depth after 100 steps, <= 1e-3 at the end of the 600 s run."""
    z = golden("tilted_bumps_256")
    s = _solver(z, mode)
    init = s.initial_state()
    st, t, t_ = init, 0.0, 0.0
    final, t_end, n, ledger = s.advance(init, 100, 0.0)
    assert n == 100
    assert rel_l2(final.h.cpu().numpy(), z["state100"][0]) < 1e-5
    assert t_end == pytest.approx(float(z["time100"]), rel=1e-5)
    r = s.run(init, z["output_times"])
    assert rel_l2(r.states.h[-1].cpu().numpy(), z["out_final"][0]) < 1e-3
    assert abs(r.steps_used - int(z["steps_used"])) <= max(2, int(0.01 * int(z["steps_used"])))
    from hybrid_flood_b200.solver import ledger_error

    assert ledger_error(r.ledger) < 1e-6


@pytest.mark.parametrize("mode", MODES)
def test_open_outflow_edge_matches_oracle(cuda_device, mode):
    """256x256 tilted plane with the transmissive east edge (the reference NumPy
    solver has no open edge; the oracle's open edge follows boundary_conditions.py)."""
    from hybrid_flood_b200.solver import B200ShallowWaterSolver, ledger_error
    from hybrid_flood_b200.workloads import tilted_bumps

    w = tilted_bumps(256, 256)
    p = O.make_params(w.bed, w.manning_n, w.domain_mask, **w.solver_kwargs())
    d = cport.Domain(p)
    init = O.initial_state(p, depth_m=0.02)
    s = B200ShallowWaterSolver(w.bed, w.manning_n, w.domain_mask, **w.solver_kwargs(), arithmetic=mode)
    times = np.asarray([0.0, 150.0, 300.0], np.float32)
    want, ft, steps, written, led = d.run(init, times)
    r = s.run(list(init), times)
    assert rel_l2(r.states.h[-1].cpu().numpy(), want[-1, 0]) < 1e-3
    assert led["outflow"] > 0
    assert r.ledger["outflow"] == pytest.approx(led["outflow"], rel=1e-3)
    assert ledger_error(r.ledger) < 1e-6
    # 100 steps
    st_o, t = init, 0.0
    for _ in range(100):
        dt = d.cfl_dt(st_o)
        st_o = d.step(st_o, dt, t)
        t += dt
    got, t_end, n, _ = s.advance(list(init), 100, 0.0)
    assert rel_l2(got.h.cpu().numpy(), st_o.h) < 1e-5
    assert t_end == pytest.approx(t, rel=1e-5)


EDGE_SHAPES = [(1, 1), (1, 7), (9, 1), (3, 5), (37, 70), (65, 129), (40, 257)]


@pytest.mark.parametrize("shape", EDGE_SHAPES)
@pytest.mark.parametrize("bnd", [(0, 0, 0, 0), (1, 1, 1, 1), (1, 0, 0, 1)])
def test_ragged_shapes_masks_and_boundaries(cuda_device, shape, bnd):
    from hybrid_flood_b200.solver import B200ShallowWaterSolver

    rng = np.random.default_rng(hash((shape, bnd)) % 2**32)
    rows, cols = shape
    bed = rng.uniform(0, 0.5, shape).astype(np.float32)
    mask = rng.uniform(size=shape) > 0.2
    mask.flat[0] = True
    n = rng.uniform(0.0, 0.06, shape).astype(np.float32)
    kw = dict(resolution_m=2.0, rainfall_times_s=np.asarray([0.0, 5.0, 30.0], np.float32),
              rainfall_rates_m_s=np.asarray([1e-5, 4e-5, 0.0], np.float32), default_rainfall_m_s=1e-6,
              boundary=bnd, cfl=0.8, dry_tolerance_m=1e-3, max_dt_s=3.0)
    p = O.make_params(bed, n, mask, **kw)
    init = O.initial_state(p, depth_m=np.where(rng.uniform(size=shape) > 0.3, 0.3, 0.0),
                           x_velocity_m_s=rng.normal(0, 0.2, shape), y_velocity_m_s=rng.normal(0, 0.2, shape))
    s = B200ShallowWaterSolver(bed, n, mask, **kw, arithmetic="exact")
    st_o, st_g, t = init, [torch.from_numpy(a).to(cuda_device) for a in init], 0.0
    for _ in range(6):
        dt = O.compute_cfl_dt(st_o, p)
        assert s.cfl_dt(st_g) == dt
        st_o = O.finite_volume_step(st_o, p, dt, t)
        st_g = s.step(st_g, dt, t)
        t += dt
    for g, w in zip(_np(st_g), st_o):
        np.testing.assert_allclose(g, w, rtol=1e-5, atol=1e-7)


def test_vector_widths_agree_bitwise(cuda_device):
    """float4, float2 and scalar load paths give identical results."""
    from hybrid_flood_b200.solver import B200ShallowWaterSolver
    from hybrid_flood_b200.workloads import tilted_bumps

    w = tilted_bumps(64, 96, seed=11)
    s = B200ShallowWaterSolver(w.bed, w.manning_n, w.domain_mask, **w.solver_kwargs())
    init = s.initial_state(depth_m=0.1, x_velocity_m_s=0.3)
    ref = _np(s.step(init, 0.5, 1.0))
    for pad, off in ((4, 0), (2, 2), (1, 1), (3, 1)):
        big = [torch.zeros((64, 96 + pad), device=cuda_device) for _ in range(3)]
        views = []
        for b, a in zip(big, init):
            v = b[:, off:off + 96]
            v.copy_(a)
            views.append(v)
        got = _np(s.step(views, 0.5, 1.0))
        for g, r in zip(got, ref):
            np.testing.assert_array_equal(g, r)


def test_run_validation_and_step_cap(cuda_device):
    z = golden("flat_basin_20")
    s = _solver(z, "exact")
    with pytest.raises(ValueError, match="Output times"):
        s.run(list(z["state0"]), np.asarray([1.0, 2.0], np.float32))
    with pytest.raises(ValueError, match="Output times"):
        s.run(list(z["state0"]), np.asarray([0.0, 2.0, 2.0], np.float32))
    with pytest.raises(RuntimeError, match="max_steps"):
        s.run(list(z["state0"]), z["output_times"], max_steps=3)
    from hybrid_flood_b200.solver import B200ShallowWaterSolver

    with pytest.raises(ValueError, match="identical shapes"):
        B200ShallowWaterSolver(np.zeros((3, 3)), np.zeros((3, 4)), np.ones((3, 3), bool),
                               resolution_m=1.0, rainfall_times_s=[0.0], rainfall_rates_m_s=[0.0])


def test_run_is_deterministic_and_rain_rate_matches(cuda_device):
    z = golden("wetdry_mask_33x47")
    s = _solver(z, "exact")
    times = np.asarray([0.0, 10.0, 25.0], np.float32)
    a = s.run(list(z["state0"]), times)
    b = s.run(list(z["state0"]), times)
    for x, y in zip(a.states, b.states):
        assert torch.equal(x, y)
    assert a.ledger == b.ledger
    p = golden_params(z)
    for t in [-1.0, 0.0, 5.0, 7.5, 20.0, 33.3, 55.0, 60.0]:
        assert s.rainfall_rate(t) == O.rainfall_rate(p, t)
    # the run agrees with the oracle's run
    r = O.run(O.State(*z["state0"]), p, times)
    assert a.steps_used == r.steps_used
    assert rel_l2(a.states.h[-1].cpu().numpy(), r.states.h[-1]) < 1e-5


def test_urban_2048_parity_and_invariants(cuda_device):
    """Full-size (2048x2048 urban) checks against the C oracle: a lake at rest over
    the block DEM (wet/dry block walls, depths up to ~5 m) and 5 steps of the real
    workload (rain, friction, open outflow edge); FP64 ledger closure."""
    from hybrid_flood_b200.solver import B200ShallowWaterSolver, ledger_error
    from hybrid_flood_b200.workloads import urban

    w = urban(2048, 2048)
    kw = w.solver_kwargs()
    kw.update(boundary=(0, 0, 0, 0), rainfall_rates_m_s=np.zeros_like(w.rainfall_rates_m_s))
    p = O.make_params(w.bed, w.manning_n, w.domain_mask, **kw)
    d = cport.Domain(p)
    eta = np.float32(float(np.median(w.bed)) + 0.3)
    depth = np.maximum(eta - w.bed, 0).astype(np.float32)
    init = O.initial_state(p, depth_m=depth)
    s = B200ShallowWaterSolver(w.bed, w.manning_n, w.domain_mask, **kw)
    st, t_end, n, led = s.advance(list(init), 20)
    st_o, t = init, 0.0
    for _ in range(20):
        dt = d.cfl_dt(st_o)
        st_o = d.step(st_o, dt, t)
        t += dt
    got = _np(st)
    # The scheme keeps the lake at rest up to float32 rounding of h + z (|q| ~ 1e-5 at 5 m).
    assert np.abs(got[1]).max() < 1e-4 and np.abs(got[2]).max() < 1e-4
    np.testing.assert_allclose(got[0], st_o.h, atol=1e-6)
    np.testing.assert_allclose(got[1], st_o.hu, atol=1e-6)
    np.testing.assert_allclose(got[2], st_o.hv, atol=1e-6)
    assert ledger_error(led) < 1e-7
    # parity with the C oracle on the real workload (rain, friction, open edge)
    p = O.make_params(w.bed, w.manning_n, w.domain_mask, **w.solver_kwargs())
    d = cport.Domain(p)
    init = O.initial_state(p, depth_m=np.where(w.bed < np.median(w.bed) + 0.1, 0.05, 0.0))
    s = B200ShallowWaterSolver(w.bed, w.manning_n, w.domain_mask, **w.solver_kwargs())
    st_o, t = init, 0.0
    for _ in range(5):
        dt = d.cfl_dt(st_o)
        st_o = d.step(st_o, dt, t)
        t += dt
    got, t_end, n, led = s.advance(list(init), 5, 0.0)
    assert t_end == pytest.approx(t, rel=1e-6)
    assert rel_l2(got.h.cpu().numpy(), st_o.h) < 1e-6
    assert ledger_error(led) < 1e-6


def test_benchmark_compiled_steps_report(cuda_device, tmp_path):
    """Fixed-dt timing helper with the fields of jax_solver/benchmarking.py:17-97."""
    from hybrid_flood_b200.solver import B200ShallowWaterSolver, benchmark_compiled_steps

    z = golden("lake_gauss_20")
    s = _solver(z, "fast")
    with pytest.raises(ValueError):
        benchmark_compiled_steps(s, list(z["state0"]), iterations=0)
    rep = benchmark_compiled_steps(s, list(z["state0"]), iterations=20, dt_s=0.05, output_directory=tmp_path)
    gpu = [r for r in rep["benchmarks"] if r["platform"] == "gpu"][0]
    assert gpu["available"] and gpu["iterations"] == 20 and gpu["seconds_per_step"] > 0
    assert gpu["grid_shape"] == list(z["state0"][0].shape)
    assert rep["gpu_benchmark_available"] and pathlib.Path(rep["output_path"]).exists()
    assert isinstance(s, B200ShallowWaterSolver)
