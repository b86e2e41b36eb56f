"""Parity on the measured configurations, in the arithmetic each is measured in,
and the float32-vs-float64 error of every configuration (GPU, through the C ABI).

Bars (the north-star bars of this path, written per test):
* relative L2 depth error <= 1e-5 against the float32 oracle after 100 CFL steps;
* relative L2 depth error <= 1e-3 against the float32 oracle at the end of a run;
* against a float64 run of the restated reference solver (``oracle/swe_oracle.c``
  built in double, the same operation order as
  ``src/hybrid_flood/numpy_solver/shallow_water_2d.py:60-327`` without its hard
  float32 casts at ``:324-326``): the GPU's error is stated per configuration and
  must stay within 3x the float32 oracle's own error plus 1e-6 -- the GPU run is as
  close to the float64 solution as the reference's float32 arithmetic is.

Set ``SWE_PARITY_REPORT=<path>`` to have the measured errors written there as JSON.
"""

from __future__ import annotations

import json
import os

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import cport
from oracle import swe_numpy as O

pytestmark = pytest.mark.gpu

_REPORT: dict = {}


def _record(name: str, **values) -> None:
    _REPORT[name] = values
    path = os.environ.get("SWE_PARITY_REPORT")
    if path:
        with open(path, "w") as f:
            json.dump(_REPORT, f, indent=1, sort_keys=True)


def _oracle(w, dtype=np.float32, **over):
    kw = w.solver_kwargs()
    kw.update(over)
    return O.make_params(w.bed, w.manning_n, w.domain_mask, dtype=dtype, **kw)


def _oracle_steps(p, init, n, t0=0.0):
    d = cport.Domain(p)
    st, t = O.State(*(np.asarray(a, p.dtype) for a in init)), t0
    for _ in range(n):
        dt = d.cfl_dt(st)
        st = d.step(st, dt, t)
        t += dt
    return st, t


def _solver(w, arith, **over):
    from hybrid_flood_b200.solver import B200ShallowWaterSolver

    kw = w.solver_kwargs()
    kw.update(over)
    return B200ShallowWaterSolver(w.bed, w.manning_n, w.domain_mask, **kw, arithmetic=arith)


def _h(state) -> np.ndarray:
    return state[0].detach().cpu().numpy() if isinstance(state[0], torch.Tensor) else np.asarray(state[0])


def _fp64_bar(gpu64: float, f32_64: float) -> bool:
    return gpu64 <= 3.0 * f32_64 + 1e-6


def _bench_workload(rows, cols):
    """The measured plain-step workload: urban DEM, streets ponded 5 cm, open east edge."""
    from hybrid_flood_b200.workloads import street_depth, urban

    w = urban(rows, cols)
    return w, street_depth(w)


@pytest.mark.parametrize("arith", ["fast", "exact"])
def test_urban_2048_bench_workload_100_steps(cuda_device, arith):
    """The headline workload (2048x2048 urban, open east edge) in the arithmetic
    it is measured in: 100 CFL steps against the float32 oracle (<= 1e-5), and
    the error against the float64 solution at the same simulated time."""
    w, depth = _bench_workload(2048, 2048)
    p32 = _oracle(w)
    init = O.initial_state(p32, depth_m=depth)
    s = _solver(w, arith)
    got, t_gpu, n, _ = s.advance(list(init), 100, 0.0)
    want, t_or = _oracle_steps(p32, init, 100)
    e32 = rel_l2(_h(got), want.h)
    assert t_gpu == pytest.approx(t_or, rel=1e-5)
    assert e32 <= 1e-5, e32
    # float64 solution at the GPU's simulated time (run to that output time)
    times = np.asarray([0.0, t_gpu], np.float32)
    r64 = cport.Domain(_oracle(w, np.float64)).run(init, times)
    r32 = cport.Domain(p32).run(init, times)
    g = s.run(list(init), times)
    gpu64 = rel_l2(g.states.h[-1].cpu().numpy(), r64[0][-1, 0])
    f32_64 = rel_l2(r32[0][-1, 0], r64[0][-1, 0])
    _record(f"config1_urban2048_{arith}", steps=100, rel_l2_vs_f32_oracle=e32, rel_l2_vs_f64=gpu64,
            f32_oracle_vs_f64=f32_64, simulated_s=float(t_gpu))
    assert _fp64_bar(gpu64, f32_64), (gpu64, f32_64)


def test_urban_512_fast_long_window(cuda_device):
    """Urban 512x512 in fast arithmetic over 600 s of simulated time (about two
    thousand steps of moving water through the street grid): <= 1e-5 after 100
    steps and <= 1e-3 at the end against the float32 oracle."""
    w, depth = _bench_workload(512, 512)
    p32 = _oracle(w)
    init = O.initial_state(p32, depth_m=depth)
    s = _solver(w, "fast")
    got100, _, _, _ = s.advance(list(init), 100, 0.0)
    want100, _ = _oracle_steps(p32, init, 100)
    e100 = rel_l2(_h(got100), want100.h)
    assert e100 <= 1e-5, e100
    times = np.asarray([0.0, 300.0, 600.0], np.float32)
    g = s.run(list(init), times)
    r32 = cport.Domain(p32).run(init, times)
    r64 = cport.Domain(_oracle(w, np.float64)).run(init, times)
    e_end = rel_l2(g.states.h[-1].cpu().numpy(), r32[0][-1, 0])
    gpu64 = rel_l2(g.states.h[-1].cpu().numpy(), r64[0][-1, 0])
    f32_64 = rel_l2(r32[0][-1, 0], r64[0][-1, 0])
    _record("config1_urban512_fast_600s", steps=int(g.steps_used), rel_l2_100_steps=e100,
            rel_l2_end_vs_f32_oracle=e_end, rel_l2_end_vs_f64=gpu64, f32_oracle_vs_f64=f32_64)
    assert g.steps_used == r32[2]
    assert e_end <= 1e-3, e_end
    assert _fp64_bar(gpu64, f32_64), (gpu64, f32_64)


@pytest.mark.parametrize("arith", ["fast", "exact"])
def test_tilted_bumps_256_open_edge(cuda_device, arith):
    """The 256x256 plain-forward case as specified: dry start, 20 mm/h for
    600 s, reflective walls with an open (transmissive) east edge, CFL 0.9,
    dry threshold 1e-3: <= 1e-5 after 100 steps, <= 1e-3 at 600 s."""
    from hybrid_flood_b200.workloads import tilted_bumps

    w = tilted_bumps(256, 256, seed=0)
    assert w.boundary == (0, 1, 0, 0)
    p32 = _oracle(w)
    init = O.initial_state(p32, depth_m=0.0)
    s = _solver(w, arith)
    got100, _, _, _ = s.advance(list(init), 100, 0.0)
    want100, _ = _oracle_steps(p32, init, 100)
    e100 = rel_l2(_h(got100), want100.h)
    assert e100 <= 1e-5, e100
    times = np.asarray([0.0, 300.0, 600.0], np.float32)
    g = s.run(list(init), times)
    r32 = cport.Domain(p32).run(init, times)
    r64 = cport.Domain(_oracle(w, np.float64)).run(init, times)
    e_end = rel_l2(g.states.h[-1].cpu().numpy(), r32[0][-1, 0])
    gpu64 = rel_l2(g.states.h[-1].cpu().numpy(), r64[0][-1, 0])
    f32_64 = rel_l2(r32[0][-1, 0], r64[0][-1, 0])
    _record(f"config0_tilted256_open_{arith}", steps=int(g.steps_used), rel_l2_100_steps=e100,
            rel_l2_end_vs_f32_oracle=e_end, rel_l2_end_vs_f64=gpu64, f32_oracle_vs_f64=f32_64)
    assert e_end <= 1e-3, e_end
    assert _fp64_bar(gpu64, f32_64), (gpu64, f32_64)


def test_adjoint_rollout_forward_512_fixed_dt(cuda_device):
    """The adjoint configuration's forward: 512x512 dx = 2 m, log-normal n,
    2000 fixed steps of 0.2 s from a ponded start (exact arithmetic, as the
    adjoint rollout runs it): the final depth against the float32 oracle and the
    float64 solution."""
    from hybrid_flood_b200.solver import B200ShallowWaterSolver, _ptr, _stream
    from hybrid_flood_b200.workloads import adjoint_case

    w, _, n_est, _ = adjoint_case(512, 512)
    depth = np.maximum(1.0 - w.bed, 0.2).astype(np.float32)
    s = B200ShallowWaterSolver(w.bed, n_est, w.domain_mask, **w.solver_kwargs(), arithmetic="exact")
    st = s.initial_state(depth_m=depth)
    steps, dt = 2000, 0.2
    rc = s._lib.swe_rollout_forward(s._handle, _ptr(st.h), _ptr(st.hu), _ptr(st.hv), st.h.stride(0), steps, dt,
                                    0.0, None, None, 0, 1, None, None, 1, _stream(s.device))
    assert rc == 0
    torch.cuda.synchronize()
    out = {}
    for name, dtype in (("f32", np.float32), ("f64", np.float64)):
        p = _oracle(w, dtype)
        d = cport.Domain(p)
        o = O.initial_state(p, depth_m=depth)
        t = 0.0
        for _ in range(steps):
            o = d.step(o, dt, t)
            t += dt
        out[name] = o.h
    e32 = rel_l2(_h(st), out["f32"])
    gpu64 = rel_l2(_h(st), out["f64"])
    f32_64 = rel_l2(out["f32"], out["f64"])
    _record("config2_adjoint512_forward_exact", steps=steps, rel_l2_end_vs_f32_oracle=e32, rel_l2_end_vs_f64=gpu64,
            f32_oracle_vs_f64=f32_64)
    assert e32 <= 1e-3, e32
    assert _fp64_bar(gpu64, f32_64), (gpu64, f32_64)


def test_ensemble_config_sized_members_fast(cuda_device):
    """Ensemble members of the batched configuration's sizes (768x1536, 1024x1024,
    256x256) through B200Ensemble in fast arithmetic: each member after 100 of
    its own CFL steps against the float32 oracle (<= 1e-5), the 768x1536 member
    also against the float64 solution."""
    from hybrid_flood_b200.ensemble import B200Ensemble
    from hybrid_flood_b200.workloads import as_member, street_depth, urban

    ws = [urban(768, 1536, seed=1003, rain_scale=1.3, n_scale=0.9), urban(1024, 1024, seed=1004),
          urban(256, 256, seed=1005, rain_scale=0.7, n_scale=1.15)]
    ens = B200Ensemble([as_member(w) for w in ws], arithmetic="fast")
    depths = [street_depth(w) for w in ws]
    states = ens.initial_states(depths)
    res = ens.advance_(states, 100)
    for m, (w, st) in enumerate(zip(ws, states)):
        p32 = _oracle(w)
        init = O.initial_state(p32, depth_m=depths[m])
        want, t_or = _oracle_steps(p32, init, 100)
        e = rel_l2(_h(st), want.h)
        assert res[m][0] == pytest.approx(t_or, rel=1e-5)
        assert e <= 1e-5, (m, e)
        if m == 0:
            t_end = res[m][0]
            times = np.asarray([0.0, t_end], np.float32)
            r64 = cport.Domain(_oracle(w, np.float64)).run(init, times)
            r32 = cport.Domain(p32).run(init, times)
            gpu64 = rel_l2(_h(st), r64[0][-1, 0])
            f32_64 = rel_l2(r32[0][-1, 0], r64[0][-1, 0])
            _record("config3_member768x1536_fast", steps=100, rel_l2_vs_f32_oracle=e, rel_l2_vs_f64=gpu64,
                    f32_oracle_vs_f64=f32_64)
            assert _fp64_bar(gpu64, f32_64), (gpu64, f32_64)


def test_hybrid_member_1024_interval_fast(cuda_device):
    """One 1024x1024 urban member of the hybrid configuration over one 60 s
    correction interval (advance_to, float64 target) in fast arithmetic, against
    the float32 oracle (<= 1e-3 at the interval end) and the float64 solution."""
    from hybrid_flood_b200.workloads import street_depth, urban

    w = urban(1024, 1024, seed=2000)
    depth = street_depth(w)
    p32 = _oracle(w)
    init = O.initial_state(p32, depth_m=depth)
    s = _solver(w, "fast")
    st = s.initial_state(depth_m=depth)
    t_end, n, _ = s.advance_to_(st, 0.0, 60.0, 5000)
    assert t_end == pytest.approx(60.0, abs=1e-6)
    times = np.asarray([0.0, 60.0], np.float32)
    r32 = cport.Domain(p32).run(init, times)
    r64 = cport.Domain(_oracle(w, np.float64)).run(init, times)
    e32 = rel_l2(_h(st), r32[0][-1, 0])
    gpu64 = rel_l2(_h(st), r64[0][-1, 0])
    f32_64 = rel_l2(r32[0][-1, 0], r64[0][-1, 0])
    _record("config4_member1024_fast_60s", steps=int(n), rel_l2_vs_f32_oracle=e32, rel_l2_vs_f64=gpu64,
            f32_oracle_vs_f64=f32_64)
    assert e32 <= 1e-3, e32
    assert _fp64_bar(gpu64, f32_64), (gpu64, f32_64)
