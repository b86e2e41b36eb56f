"""Generate the golden fixtures in this directory from the UNMODIFIED reference solver.

Run in a container where the reference project is mounted (it is not needed,
and not read, anywhere else):

    python tests/golden/make_golden.py --reference /root/reference

It imports ``hybrid_flood.numpy_solver.shallow_water_2d`` from the reference's
``src/`` (the V1 NumPy solver; NumPy is its only dependency) and runs it on the
cases below, saving inputs and outputs as compressed ``.npz`` files.  The tests
then pin the oracle (and, on a GPU, the CUDA path) against these files without
needing the reference at run time.

Cases (reference test each restates, paths inside the reference project):

* ``one_step_7x9``      one step, ``tests/test_v1_v2_architecture.py:85-104``
* ``lake_sin2_12``      lake at rest to 20 s, ``tests/test_v1_v2_architecture.py:107-117``
* ``flat_basin_20``     reflective basin mass, ``tests/test_jax_solver_conservation.py:240-251``
* ``lake_gauss_20``     lake at rest over a bump, ``tests/test_jax_solver_conservation.py:254-270``
* ``mask_walls_12``     lake at rest at inactive cells, ``tests/test_jax_solver_conservation.py:273-289``
  (the last three are JAX tests there; here the NumPy reference runs them, which
  ``test_v1_v2_architecture.py:85-104`` pins as step-equivalent to JAX)
* ``wetdry_mask_33x47`` irregular mask, wet/dry fronts, varying n, multi-entry
  rain table with a default outside it; 40 CFL steps, states every 10 steps
* ``tilted_bumps_256``  the 256x256 tilted-plane case with all-reflective walls
  (the reference NumPy solver has no open boundary): state after 100 CFL steps
  and the run to 600 s
"""

from __future__ import annotations

import argparse
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
REPO = HERE.parents[1]


def _load_reference(reference: pathlib.Path):
    sys.path.insert(0, str(reference / "src"))
    from hybrid_flood.numpy_solver import shallow_water_2d as ref  # noqa: PLC0415

    return ref


def _solver(ref, bed, manning, mask, *, dx, rain_times, rain_rates, default=0.0, **kw):
    return ref.NumpyShallowWaterSolver(
        bed, manning, mask, resolution_m=dx, rainfall_times_s=rain_times,
        rainfall_rates_m_s=rain_rates, default_rainfall_m_s=default, **kw,
    )


def _controls(solver) -> dict:
    p = solver.params
    return dict(dx=p.dx, dy=p.dy, gravity=p.gravity, cfl=p.cfl, dry=p.dry_tolerance,
                max_dt=p.max_dt, default_rain=p.default_rainfall_m_s)


def _save(name: str, solver, **arrays) -> None:
    p = solver.params
    payload = dict(
        bed=p.bed, manning_n=p.manning_n, domain_mask=p.domain_mask,
        rain_times=p.rainfall_times_s, rain_rates=p.rainfall_rates_m_s,
        boundary=np.zeros(4, dtype=np.int32),
        **{f"ctl_{k}": np.float64(v) for k, v in _controls(solver).items()},
        **arrays,
    )
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **payload)
    print(f"wrote {path.name}: {path.stat().st_size / 1024:.1f} KiB")


def _steps(ref, solver, state, n, t0=0.0, every=None):
    t = float(t0)
    snaps, dts = [], []
    for k in range(n):
        dt = ref.compute_cfl_dt(state, solver.params)
        state = ref.finite_volume_step(state, solver.params, dt, t)
        t += dt
        dts.append(dt)
        if every and (k + 1) % every == 0:
            snaps.append(np.stack(state))
    return state, t, np.asarray(dts), snaps


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=pathlib.Path, default=pathlib.Path("/root/reference"))
    args = ap.parse_args()
    ref = _load_reference(args.reference)

    # one_step_7x9 -------------------------------------------------------------
    rng = np.random.default_rng(7)
    bed = rng.uniform(0.0, 0.2, size=(7, 9)).astype(np.float32)
    rt = np.asarray([0.0, 1000.0], dtype=np.float32)
    rr = np.asarray([1.2e-6, 1.2e-6], dtype=np.float32)
    s = _solver(ref, bed, np.full(bed.shape, 0.03, np.float32), np.ones(bed.shape, bool),
                dx=20.0, rain_times=rt, rain_rates=rr, max_dt_s=2.0)
    h0 = np.full(bed.shape, 0.1, dtype=np.float32)
    hu0 = rng.normal(0.0, 1.0e-3, bed.shape).astype(np.float32)
    hv0 = rng.normal(0.0, 1.0e-3, bed.shape).astype(np.float32)
    out = ref.finite_volume_step(ref.NumpyState(h0, hu0, hv0), s.params, 0.75, 20.0)
    cfl_dt = ref.compute_cfl_dt(ref.NumpyState(h0, hu0, hv0), s.params)
    _save("one_step_7x9", s, state0=np.stack([h0, hu0, hv0]), dt=np.float64(0.75),
          time_s=np.float64(20.0), state1=np.stack(out), cfl_dt0=np.float64(cfl_dt))

    # lake_sin2_12 -------------------------------------------------------------
    x = np.linspace(0.0, 1.0, 12, dtype=np.float32)
    bed = 0.2 * np.outer(np.sin(np.pi * x) ** 2, np.sin(np.pi * x) ** 2)
    rt = np.asarray([0.0, 1000.0], dtype=np.float32)
    rr = np.zeros(2, dtype=np.float32)
    s = _solver(ref, bed, np.full(bed.shape, 0.03, np.float32), np.ones(bed.shape, bool),
                dx=20.0, rain_times=rt, rain_rates=rr, max_dt_s=2.0)
    init = ref.NumpyState(np.float32(0.35) - s.params.bed, np.zeros_like(s.params.bed),
                          np.zeros_like(s.params.bed))
    times = np.asarray([0.0, 20.0], np.float32)
    res = s.run(init, times, max_steps=100)
    _save("lake_sin2_12", s, state0=np.stack(init), output_times=times,
          out_h=res.states.h, out_hu=res.states.hu, out_hv=res.states.hv,
          final_time_s=np.float64(res.final_time_s), steps_used=np.int64(res.steps_used))

    # JAX-test geometries run on the NumPy reference -----------------------------
    def basin_solver(bed, mask=None):
        mask = np.ones(bed.shape, bool) if mask is None else mask
        return _solver(ref, bed.astype(np.float32), np.zeros(bed.shape, np.float32), mask,
                       dx=1.0, rain_times=np.asarray([0.0, 100.0], np.float32),
                       rain_rates=np.zeros(2, np.float32), cfl=0.4, dry_tolerance_m=1.0e-6,
                       max_dt_s=0.1)

    def run_case(name, solver, depth, times):
        init = solver.initial_state(depth_m=depth)
        res = solver.run(init, times, max_steps=1000)
        _save(name, solver, state0=np.stack(init), output_times=times,
              out_h=res.states.h, out_hu=res.states.hu, out_hv=res.states.hv,
              final_time_s=np.float64(res.final_time_s), steps_used=np.int64(res.steps_used))

    bed = np.zeros((20, 20), np.float32)
    depth = np.full_like(bed, 0.1)
    depth[8:12, 8:12] = 0.2
    run_case("flat_basin_20", basin_solver(bed), depth, np.asarray([0.0, 1.0, 2.0], np.float32))

    c = np.linspace(-1.0, 1.0, 20)
    xx, yy = np.meshgrid(c, c)
    bed = (0.03 * np.exp(-5.0 * (xx**2 + yy**2))).astype(np.float32)
    run_case("lake_gauss_20", basin_solver(bed), 0.2 - bed, np.asarray([0.0, 1.0, 2.0], np.float32))

    bed = np.zeros((12, 12), np.float32)
    mask = np.ones_like(bed, dtype=bool)
    mask[4:8, 5:7] = False
    run_case("mask_walls_12", basin_solver(bed, mask), 0.1, np.asarray([0.0, 0.5], np.float32))

    # wetdry_mask_33x47 ---------------------------------------------------------
    rng = np.random.default_rng(2024)
    rows, cols = 33, 47
    yy, xx = np.mgrid[0:rows, 0:cols].astype(np.float64)
    bed = 0.02 * xx + 0.3 * np.sin(xx / 5.0) * np.cos(yy / 7.0) + rng.uniform(0, 0.05, (rows, cols))
    mask = ((xx - 23) ** 2 / 500.0 + (yy - 16) ** 2 / 200.0) < 1.0
    mask[10:14, 20:25] = False
    manning = rng.uniform(0.01, 0.08, (rows, cols))
    rt = np.asarray([5.0, 20.0, 40.0, 55.0], np.float32)
    rr = np.asarray([3e-5, 8e-5, 1e-5, 0.0], np.float32)
    s = _solver(ref, bed, manning, mask, dx=3.0, rain_times=rt, rain_rates=rr, default=2e-6,
                cfl=0.9, dry_tolerance_m=1e-3, max_dt_s=5.0)
    depth = np.where(bed < 0.25, 0.4 - bed, 0.0).clip(0.0, None).astype(np.float32)
    u0 = rng.normal(0.0, 0.05, (rows, cols)).astype(np.float32)
    init = s.initial_state(depth_m=depth, x_velocity_m_s=u0, y_velocity_m_s=-0.5 * u0)
    state, t, dts, snaps = _steps(ref, s, init, 40, every=10)
    _save("wetdry_mask_33x47", s, state0=np.stack(init), snaps=np.stack(snaps), dts=dts,
          final_time_s=np.float64(t))

    # tilted_bumps_256 (all reflective) ---------------------------------------------
    sys.path.insert(0, str(REPO / "gpu-hybrid-flood-forecasting_b200"))
    from hybrid_flood_b200.workloads import tilted_bumps  # noqa: PLC0415

    w = tilted_bumps(256, 256)
    s = _solver(ref, w.bed, w.manning_n, w.domain_mask, dx=w.resolution_m,
                rain_times=w.rainfall_times_s, rain_rates=w.rainfall_rates_m_s,
                cfl=w.cfl, dry_tolerance_m=w.dry_tolerance_m, max_dt_s=w.max_dt_s)
    init = s.initial_state()
    state100, t100, dts, _ = _steps(ref, s, init, 100)
    times = np.asarray([0.0, 300.0, 600.0], np.float32)
    res = s.run(init, times)
    _save("tilted_bumps_256", s, state100=np.stack(state100), time100=np.float64(t100),
          dts100=dts, output_times=times, out_final=np.stack(
              [res.states.h[-1], res.states.hu[-1], res.states.hv[-1]]),
          final_time_s=np.float64(res.final_time_s), steps_used=np.int64(res.steps_used))


if __name__ == "__main__":
    main()
