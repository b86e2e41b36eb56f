"""Output schema on the GPU against the oracle (structured_io.py:160-230).

The fields kernel uses IEEE division and a double-evaluated hypot, so it equals
the reference's NumPy arrays bit for bit (NaN at the same places).  The
streamed run writes the same states as ``run`` (same steps, same clock) into a
NetCDF-3 file with the reference's variables, dimensions and attributes.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import output_numpy as ON

pytestmark = pytest.mark.gpu


def _solver(arith="exact"):
    from hybrid_flood_b200.solver import B200ShallowWaterSolver
    from hybrid_flood_b200.workloads import urban

    w = urban(40, 70, seed=9, duration_s=3600.0)
    mask = np.ones(w.shape, bool)
    mask[10:14, 20:31] = False
    kw = w.solver_kwargs()
    kw["cfl"] = 0.9
    return B200ShallowWaterSolver(w.bed, w.manning_n, mask, **kw, arithmetic=arith), w, mask


def test_output_fields_match_oracle(cuda_device):
    from hybrid_flood_b200.output import FIELDS, output_fields

    s, w, mask = _solver()
    rng = np.random.default_rng(0)
    h = np.where(rng.uniform(size=w.shape) > 0.3, rng.uniform(0, 0.2, w.shape), rng.uniform(0, 2e-4, w.shape))
    state = [h.astype(np.float32), rng.normal(0, 0.01, w.shape).astype(np.float32),
             rng.normal(0, 0.01, w.shape).astype(np.float32)]
    got = output_fields(s, [torch.tensor(a, device=cuda_device) for a in state])
    want = ON.conserved_fields(*state, mask, s.params.dry_tolerance)
    for name, ref in zip(FIELDS, want):
        np.testing.assert_array_equal(got[name].cpu().numpy(), ref)


@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_streamed_run_matches_run_and_schema(cuda_device, tmp_path, arith):
    from hybrid_flood_b200.output import read_netcdf, run_to_netcdf

    s, w, mask = _solver(arith)
    init = s.initial_state(depth_m=np.where(mask, 0.05, 0.0).astype(np.float32))
    times = np.array([0.0, 20.0, 45.0, 90.0], np.float32)
    ref = s.run(init, times)
    res = run_to_netcdf(s, init, times, tmp_path / "f.nc", title="test", crs="EPSG:32643")
    assert res.steps_used == ref.steps_used and res.outputs_written == len(times)
    assert res.final_time_s == pytest.approx(ref.final_time_s, abs=1e-9)
    f = read_netcdf(res.path)
    assert f["depth"].shape == (len(times), *w.shape) and f["elevation"].shape == w.shape
    np.testing.assert_array_equal(f["time"], times.astype(np.float64))
    fields = ON.conserved_fields(ref.states.h.cpu().numpy(), ref.states.hu.cpu().numpy(),
                                 ref.states.hv.cpu().numpy(), mask, s.params.dry_tolerance)
    for name, want in zip(("depth", "x_velocity", "y_velocity", "velocity"), fields):
        np.testing.assert_array_equal(f[name], want)
    np.testing.assert_array_equal(f["elevation"], ON.elevation(w.bed, mask))
    a = f["attrs"]
    assert a["title"] == "test" and a["crs"] == "EPSG:32643" and a["steps_used"] == ref.steps_used
    assert a["numerical_flux"] == "HLL with hydrostatic reconstruction"
    with pytest.raises(RuntimeError):
        run_to_netcdf(s, init, times, tmp_path / "g.nc", max_steps=3)
