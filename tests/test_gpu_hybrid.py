"""Physics-AI coupling on the GPU against the oracle (hybrid/coupled_forecast.py).

* features: bit-exact in float32 (same operations, same order) and in
  bfloat16 (round-to-nearest-even of the float32 value);
* correction: the volume sums are float64 on both sides but summed in a
  different order, so the projection scale may differ by one float32 ulp:
  depth and momenta within 2 ulp;
* advance to a correction time: exact arithmetic, so the step count equals
  the float64-clock C oracle's; the friction power (CUDA ``powf`` against the
  C library's ``powf``) may differ by an ulp, so the state is compared at
  1e-6 relative L2 (depth) and 1e-5 (momenta);
* coupled rollouts: the corrector runs through cuDNN (TF32 off) on the GPU and
  on the CPU for the oracle, so the residuals differ in the last bits; the
  trajectories are compared at 1e-5 relative L2.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import max_ulp, rel_l2
from oracle import cport
from oracle import hybrid_numpy as HN
from oracle import swe_numpy as O

pytestmark = pytest.mark.gpu


def _case(rows=48, cols=64, seed=3, arith="exact"):
    from hybrid_flood_b200.solver import B200ShallowWaterSolver
    from hybrid_flood_b200.workloads import urban

    w = urban(rows, cols, seed=seed, duration_s=3600.0)
    mask = np.ones(w.shape, bool)
    mask[rows // 3: rows // 3 + 5, cols // 2: cols // 2 + 7] = False
    kw = w.solver_kwargs()
    kw["cfl"] = 0.9
    solver = B200ShallowWaterSolver(w.bed, w.manning_n, mask, **kw, arithmetic=arith)
    params = O.make_params(w.bed, w.manning_n, mask, **kw)
    rng = np.random.default_rng(seed)
    h = np.where(rng.uniform(size=w.shape) > 0.2, rng.uniform(0.0, 0.3, w.shape), 0.0).astype(np.float32)
    h = np.where(mask, h, 0.0).astype(np.float32)
    hu = np.where(h > 1e-3, rng.normal(0, 0.02, w.shape), 0.0).astype(np.float32)
    hv = np.where(h > 1e-3, rng.normal(0, 0.02, w.shape), 0.0).astype(np.float32)
    return solver, params, w, mask, (h, hu, hv)


def _dev(state, device):
    from hybrid_flood_b200.solver import SWEState

    return SWEState(*(torch.tensor(a, dtype=torch.float32, device=device) for a in state))


def _inputs(w, rng, layout="reference6", nres=3):
    from hybrid_flood_b200.hybrid import HybridInputs

    if layout == "reference6":
        return HybridInputs(rng.normal(0, 1, w.shape).astype(np.float32), rng.normal(0, 1, w.shape).astype(np.float32),
                            np.array([0.1, 0.01, -0.02], np.float32), np.array([0.2, 0.3, 0.4], np.float32),
                            25.0, np.array([0.01, 0.02, 0.03][:nres], np.float32))
    return HybridInputs(None, None, np.array([0.1, 0.002, -0.001, 1.5, 3.0], np.float32),
                        np.array([0.2, 0.05, 0.04, 3.0, 4.0], np.float32), 25.0,
                        np.array([0.01, 0.02, 0.03][:nres], np.float32))


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
def test_reference6_features_match_oracle(cuda_device, dtype):
    from hybrid_flood_b200.hybrid import network_features

    solver, params, w, mask, state = _case()
    hi = _inputs(w, np.random.default_rng(1))
    t = 1234.5
    got = network_features(solver, _dev(state, cuda_device), hi, t, dtype=dtype)
    want = HN.network_features(*state, mask, params.dry_tolerance, O.rainfall_rate(params, t), hi.terrain_standardized,
                               hi.roughness_standardized, hi.state_mean, hi.state_std, hi.rainfall_scale_mm_hr)
    assert tuple(got.shape) == want.shape == (1, *w.shape, 6)
    want_t = torch.from_numpy(want).to(dtype)
    assert torch.equal(got.cpu(), want_t)


def test_state5_features_match_oracle(cuda_device):
    from hybrid_flood_b200.hybrid import network_features

    solver, params, w, mask, state = _case(seed=4)
    hi = _inputs(w, np.random.default_rng(2), "state5")
    t = 600.0
    got = network_features(solver, _dev(state, cuda_device), hi, t, layout="state5")
    rain_mm = np.float32(O.rainfall_rate(params, t) * HN.M_S_TO_MM_HR)
    want = HN.state5_features(*state, w.bed, mask, rain_mm, hi.state_mean, hi.state_std)
    assert torch.equal(got.cpu(), torch.from_numpy(want))


@pytest.mark.parametrize("nres,bf16,clip", [(3, False, True), (3, False, False), (1, True, True)])
def test_correction_matches_oracle(cuda_device, nres, bf16, clip):
    from hybrid_flood_b200.hybrid import apply_residual_correction

    solver, params, w, mask, state = _case(seed=5)
    rng = np.random.default_rng(9)
    res = rng.normal(0, 0.05, (*w.shape, nres)).astype(np.float32)
    lim = np.array([0.06, 0.03, 0.02][:nres], np.float32) if clip else None
    dt = torch.bfloat16 if bf16 else torch.float32
    # NCHW channels_last, as the corrector returns it
    r_dev = torch.tensor(res, device=cuda_device).to(dt).permute(2, 0, 1)[None]
    res_used = r_dev[0].permute(1, 2, 0).float().cpu().numpy()
    got = apply_residual_correction(solver, _dev(state, cuda_device), r_dev, correction_relaxation=0.5,
                                    clip_limits=lim)
    want = HN.apply_residual_correction(*state, res_used, mask, params.dry_tolerance, 0.5, clip_limits=lim)
    for g, w_ in zip(got, want):
        assert max_ulp(g.cpu().numpy(), w_) <= 2
    # the physics volume is kept
    assert float(got.h.double().sum()) == pytest.approx(float(np.where(mask, state[0], 0).astype(np.float64).sum()),
                                                        rel=2e-6)


def test_correction_preserves_volume_and_runs_in_place(cuda_device):
    """Restates tests/test_hybrid_rollout.py:37-64 on a synthetic grid, in place."""
    from hybrid_flood_b200.hybrid import apply_residual_correction
    from hybrid_flood_b200.solver import SWEState

    solver, params, w, mask, _ = _case(seed=6)
    depth = np.where(mask, 0.02, 0.0).astype(np.float32)
    res = np.zeros((*w.shape, 3), np.float32)
    res[..., 0] = np.where(mask, -0.01, 0.0)
    pred = _dev((depth, np.zeros_like(depth), np.zeros_like(depth)), cuda_device)
    out = apply_residual_correction(solver, pred, torch.tensor(res, device=cuda_device), correction_relaxation=1.0)
    assert float(out.h.sum()) == pytest.approx(float(depth.sum()), rel=2e-6)
    same = SWEState(*(t.clone() for t in pred))
    apply_residual_correction(solver, same, torch.tensor(res, device=cuda_device), correction_relaxation=1.0,
                              out=same)
    for a, b in zip(same, out):
        assert torch.equal(a, b)


def test_advance_to_matches_oracle_and_fills_nan_when_short(cuda_device):
    from hybrid_flood_b200.hybrid import advance_physics_to_time

    solver, params, w, mask, state = _case(seed=7)
    dom = cport.Domain(params)
    got, steps = advance_physics_to_time(solver, _dev(state, cuda_device), 120.0, 180.0, max_substeps=500)
    want, wsteps = HN.advance_physics_to_time(dom, O.State(*state), 120.0, 180.0, 500)
    assert steps == wsteps > 1
    assert rel_l2(got.h.cpu().numpy(), want[0]) < 1e-6
    for g, w_ in zip(got[1:], want[1:]):
        assert rel_l2(g.cpu().numpy(), w_) < 1e-5
    short, s2 = advance_physics_to_time(solver, _dev(state, cuda_device), 120.0, 180.0, max_substeps=2)
    assert s2 == 2
    assert all(bool(torch.isnan(t).all()) for t in short)
    with pytest.raises(ValueError):
        advance_physics_to_time(solver, _dev(state, cuda_device), 0.0, 60.0, max_substeps=0)


def _small_net(cin, cout, seed=0, scale=0.05):
    from hybrid_flood_b200.unet import ResidualUNet

    torch.manual_seed(seed)
    net = ResidualUNet(input_channels=cin, depth=2, channels=(8, 16), output_channels=cout)
    with torch.no_grad():
        net.residual_head.weight.normal_(0, scale)
        net.residual_head.bias.normal_(0, scale)
    return net.eval()


def _oracle_rollout(params, state, net, hi, times, max_sub, relax, sigma, layout="reference6"):
    dom = cport.Domain(params)
    st = O.State(*state)
    out = [st]
    total = 0
    lim = np.float32(sigma) * np.asarray(hi.residual_std, np.float32)
    for k in range(1, len(times)):
        t0 = times[k - 1]
        if layout == "reference6":
            f = HN.network_features(*st, params.domain_mask, params.dry_tolerance, O.rainfall_rate(params, t0),
                                    hi.terrain_standardized, hi.roughness_standardized, hi.state_mean, hi.state_std,
                                    hi.rainfall_scale_mm_hr)
        else:
            f = HN.state5_features(*st, params.bed, params.domain_mask,
                                   np.float32(O.rainfall_rate(params, t0) * HN.M_S_TO_MM_HR), hi.state_mean,
                                   hi.state_std)
        adv, n = HN.advance_physics_to_time(dom, st, t0, times[k], max_sub)
        total += n
        with torch.no_grad():
            r = net(torch.from_numpy(f).permute(0, 3, 1, 2))[0].permute(1, 2, 0).numpy()
        st = O.State(*HN.apply_residual_correction(*adv, r, params.domain_mask, params.dry_tolerance, relax, clip_limits=lim))
        out.append(st)
    return out, total


def test_coupled_forecast_matches_oracle(cuda_device):
    from hybrid_flood_b200.hybrid import run_coupled_forecast

    torch.backends.cudnn.allow_tf32 = False
    torch.backends.cuda.matmul.allow_tf32 = False
    solver, params, w, mask, state = _case(seed=8)
    hi = _inputs(w, np.random.default_rng(3))
    net = _small_net(6, 3)
    times = np.array([0.0, 60.0, 120.0, 180.0])
    want, wsteps = _oracle_rollout(params, state, net, hi, times, 400, 0.05, 5.0)
    res = run_coupled_forecast(solver, _dev(state, cuda_device), net.to(cuda_device), hi, times,
                               max_substeps_per_interval=400, correction_relaxation=0.05)
    assert res.physics_steps_used == wsteps
    for k in range(len(times)):
        for q in range(3):
            assert rel_l2(res.states[q][k].cpu().numpy(), want[k][q]) < 1e-5
    with pytest.raises(ValueError):
        run_coupled_forecast(solver, _dev(state, cuda_device), net, hi, times, max_substeps_per_interval=0)
    with pytest.raises(ValueError):
        run_coupled_forecast(solver, _dev(state, cuda_device), net, hi, times[:1], max_substeps_per_interval=10)


def test_bf16_channels_last_corrector_tracks_float32(cuda_device):
    from hybrid_flood_b200.hybrid import run_coupled_forecast
    from hybrid_flood_b200.unet import corrector_4level

    solver, params, w, mask, state = _case(64, 64, seed=9, arith="fast")
    hi = _inputs(w, np.random.default_rng(4), "state5", nres=1)
    torch.manual_seed(1)
    net = corrector_4level()
    with torch.no_grad():
        net.residual_head.weight.normal_(0, 0.02)
    times = np.array([0.0, 60.0, 120.0])
    f32 = run_coupled_forecast(solver, _dev(state, cuda_device), net.to(cuda_device).eval(), hi, times,
                               max_substeps_per_interval=400, correction_relaxation=0.5, feature_layout="state5")
    bf = net.to(dtype=torch.bfloat16, memory_format=torch.channels_last)
    b16 = run_coupled_forecast(solver, _dev(state, cuda_device), bf, hi, times, max_substeps_per_interval=400,
                               correction_relaxation=0.5, feature_layout="state5")
    assert bool(torch.isfinite(b16.states.h).all())
    assert rel_l2(b16.states.h[-1].cpu().numpy(), f32.states.h[-1].cpu().numpy()) < 1e-2
    # each correction keeps the physics volume, so the corrector never adds water:
    # total depth stays that of the float32 run to float32 rounding of the step
    assert float(b16.states.h[-1].double().sum()) == pytest.approx(float(f32.states.h[-1].double().sum()), rel=1e-3)


def test_ensemble_advance_to_and_coupled_ensemble_match_single_domains(cuda_device):
    from hybrid_flood_b200.ensemble import B200Ensemble
    from hybrid_flood_b200.hybrid import run_coupled_ensemble, run_coupled_forecast
    from hybrid_flood_b200.solver import B200ShallowWaterSolver
    from hybrid_flood_b200.workloads import urban

    torch.backends.cudnn.allow_tf32 = False
    members, states = [], []
    for m in range(3):
        w = urban(40, 56, seed=20 + m, rain_scale=1.0 + 0.5 * m, duration_s=3600.0)
        kw = w.solver_kwargs()
        members.append(dict(bed=w.bed, manning_n=w.manning_n, domain_mask=w.domain_mask, **kw))
        rng = np.random.default_rng(m)
        h = np.where(w.domain_mask, rng.uniform(0.0, 0.2, w.shape), 0.0).astype(np.float32)
        states.append((h, np.zeros_like(h), np.zeros_like(h)))
    ens = B200Ensemble(members, arithmetic="exact")
    # advance_to: members bit-equal to single-domain advance_to
    cur = [_dev(s, cuda_device) for s in states]
    res = ens.advance_to_(cur, [0.0, 10.0, 30.0], 90.0, 1000)
    for m, (t, n, _) in enumerate(res):
        kw = {k: v for k, v in members[m].items() if k not in ("bed", "manning_n", "domain_mask")}
        s = B200ShallowWaterSolver(members[m]["bed"], members[m]["manning_n"], members[m]["domain_mask"], **kw,
                                   arithmetic="exact")
        one = _dev(states[m], cuda_device)
        t1, n1, _ = s.advance_to_(one, [0.0, 10.0, 30.0][m], 90.0, 1000)
        assert (t, n) == (t1, n1)
        assert abs(t - 90.0) < 1e-7
        for a, b in zip(cur[m], one):
            assert torch.equal(a, b)
    # coupled ensemble vs per-member coupled rollouts
    hi = _inputs(w, np.random.default_rng(5), "state5", nres=1)
    net = _small_net(5, 1, seed=3).to(cuda_device)
    times = np.array([0.0, 60.0, 120.0])
    traj, steps = run_coupled_ensemble(ens, states, net, hi, times, max_substeps_per_interval=500,
                                       correction_relaxation=0.5)
    for m in range(3):
        kw = {k: v for k, v in members[m].items() if k not in ("bed", "manning_n", "domain_mask")}
        s = B200ShallowWaterSolver(members[m]["bed"], members[m]["manning_n"], members[m]["domain_mask"], **kw,
                                   arithmetic="exact")
        one = run_coupled_forecast(s, _dev(states[m], cuda_device), net, hi, times, max_substeps_per_interval=500,
                                   correction_relaxation=0.5, feature_layout="state5")
        assert one.physics_steps_used == steps[m]
        for q in range(3):
            assert rel_l2(traj[m][q].cpu().numpy(), one.states[q].cpu().numpy()) < 1e-5


def test_overlapped_corrector_gives_the_same_rollout(cuda_device):
    """The corrector on a side stream (overlapping the physics) changes nothing."""
    from hybrid_flood_b200.hybrid import run_coupled_forecast

    torch.backends.cudnn.benchmark = False
    solver, params, w, mask, state = _case(seed=12)
    hi = _inputs(w, np.random.default_rng(6))
    net = _small_net(6, 3, seed=4).to(cuda_device)
    times = np.array([0.0, 30.0, 60.0])
    a = run_coupled_forecast(solver, _dev(state, cuda_device), net, hi, times, max_substeps_per_interval=400,
                             overlap=True)
    b = run_coupled_forecast(solver, _dev(state, cuda_device), net, hi, times, max_substeps_per_interval=400,
                             overlap=False)
    assert a.physics_steps_used == b.physics_steps_used
    for x, y in zip(a.states, b.states):
        assert torch.equal(x, y)


@pytest.mark.parametrize("layout,dtype", [("reference6", torch.float32), ("state5", torch.bfloat16)])
def test_ensemble_coupling_calls_equal_per_member_calls(cuda_device, layout, dtype):
    """One batched features call and one batched correction call over an
    ensemble give every member exactly what the per-member calls give."""
    from hybrid_flood_b200.ensemble import B200Ensemble
    from hybrid_flood_b200.hybrid import (LAYOUTS, apply_residual_correction, ensemble_apply_correction,
                                          ensemble_domains, ensemble_network_features, network_features)
    from hybrid_flood_b200.workloads import urban

    members, states, his = [], [], []
    for m in range(3):
        w = urban(40, 56, seed=40 + m, rain_scale=1.0 + 0.5 * m, duration_s=3600.0)
        members.append(dict(bed=w.bed, manning_n=w.manning_n, domain_mask=w.domain_mask, **w.solver_kwargs()))
        rng = np.random.default_rng(70 + m)
        h = np.where(w.domain_mask, rng.uniform(0.0, 0.2, w.shape), 0.0).astype(np.float32)
        hu = np.where(h > 1e-3, rng.normal(0, 0.02, w.shape), 0.0).astype(np.float32)
        states.append(_dev((h, hu, np.zeros_like(h) + 0.001), cuda_device))
        his.append(_inputs(w, np.random.default_rng(80 + m), layout, nres=3))
    ens = B200Ensemble(members, arithmetic="exact")
    doms = ensemble_domains(ens)
    C = LAYOUTS[layout][1]
    batch = torch.full((3, 40, 56, C), 7.0, dtype=dtype, device=cuda_device)
    ensemble_network_features(ens, states, his, 1234.5, layout=layout, out=batch)
    for m in range(3):
        one = network_features(doms[m], states[m], his[m], 1234.5, layout=layout, dtype=dtype)
        assert torch.equal(batch[m], one[0])
    # residual as a corrector returns it: NCHW logical, channels-last memory, bfloat16
    g = torch.Generator(device="cpu").manual_seed(9)
    res = (0.05 * torch.randn((3, 3, 40, 56), generator=g)).to(cuda_device, torch.bfloat16)
    res = res.contiguous(memory_format=torch.channels_last)
    lims = [np.array([0.02, 0.03, 0.04], np.float32), None, np.array([0.5, 0.5, 0.5], np.float32)]
    got = ensemble_apply_correction(ens, states, res, correction_relaxation=0.7, clip_limits=lims)
    for m in range(3):
        want = apply_residual_correction(doms[m], states[m], res[m:m + 1], correction_relaxation=0.7,
                                         clip_limits=lims[m])
        for a, b in zip(got[m], want):
            assert torch.equal(a, b)


def test_coupling_matches_the_reference_coupling_code(cuda_device):
    """The CUDA coupling against ``tests/golden/coupling_ref6.npz``: outputs of the
    reference's own ``coupled_forecast.py`` run with a NumPy stand-in for jax
    (make_coupling_golden.py).  Features bit for bit; correction within 4 ulp
    (float64 volume sums here, float32 there); the forecast with the same
    linear corrector as a 1x1 convolution: the same step count, 1e-5 relative L2."""
    from conftest import golden
    from hybrid_flood_b200.boundary import BoundaryConfig
    from hybrid_flood_b200.hybrid import (HybridInputs, apply_residual_correction, network_features,
                                          run_coupled_forecast)
    from hybrid_flood_b200.solver import B200ShallowWaterSolver

    torch.backends.cudnn.allow_tf32 = False
    z = golden("coupling_ref6")
    bnd = BoundaryConfig(tuple(int(b) for b in z["boundary"]))
    solver = B200ShallowWaterSolver(z["bed"], z["manning_n"], z["domain_mask"], resolution_m=float(z["dx"]),
                                    rainfall_times_s=z["rain_times"], rainfall_rates_m_s=z["rain_rates"],
                                    default_rainfall_m_s=float(z["default_rain"]), boundaries=bnd,
                                    arithmetic="exact")
    hi = HybridInputs(z["terrain_std"], z["roughness_std"], z["state_mean"], z["state_std"], float(z["rain_scale"]),
                      z["residual_std"])
    st = _dev(tuple(z["state"]), cuda_device)
    for tag in ("break", "past"):
        f = network_features(solver, st, hi, float(z[f"features_{tag}_time"]), layout="reference6")
        np.testing.assert_array_equal(f.cpu().numpy(), z[f"features_{tag}"])
    lim = z["clip_sigma"] * z["residual_std"]
    res = torch.tensor(z["residual"], device=cuda_device)
    got = apply_residual_correction(solver, st, res, correction_relaxation=float(z["relaxation"]), clip_limits=lim)
    for a, q in zip(got, ("h", "hu", "hv")):
        assert max_ulp(a.cpu().numpy(), z[f"corrected_{q}"]) <= 4, q

    fs = B200ShallowWaterSolver(z["forecast_bed"], z["forecast_manning_n"], z["forecast_mask"],
                                resolution_m=float(z["dx"]), rainfall_times_s=[0.0, 1000.0],
                                rainfall_rates_m_s=[2.0e-5, 2.0e-5], boundaries=bnd, arithmetic="exact")
    fhi = HybridInputs(z["forecast_terrain_std"], z["forecast_roughness_std"], z["forecast_state_mean"],
                       z["forecast_state_std"], 25.0, z["forecast_residual_std"])
    net = torch.nn.Conv2d(6, 3, 1)
    with torch.no_grad():
        net.weight.copy_(torch.from_numpy(z["forecast_W"].T.copy())[:, :, None, None])
        net.bias.copy_(torch.from_numpy(z["forecast_b"]))
    out = run_coupled_forecast(fs, _dev(tuple(z["forecast_state"]), cuda_device), net.to(cuda_device).eval(), fhi,
                               z["forecast_times"].astype(np.float64), max_substeps_per_interval=400,
                               correction_relaxation=0.5, correction_clip_sigma=2.0)
    assert out.physics_steps_used == int(z["forecast_steps"])
    for q, name in enumerate(("h", "hu", "hv")):
        for k in range(len(z["forecast_times"])):
            assert rel_l2(out.states[q][k].cpu().numpy(), z[f"forecast_{name}"][k]) < 1e-5, (k, name)
