"""CPU checks of the coupling's host pieces: the U-Net against the reference's
own network (golden fixture), relaxation selection, and the hybrid oracle."""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from conftest import golden
from oracle import hybrid_numpy as HN
from oracle import swe_numpy as O


def test_unet_matches_reference_network():
    """``tests/golden/unet_d3_odd.npz`` holds the reference ``TorchResidualUNet``'s
    parameters, an odd-sized input and its output (make_unet_golden.py)."""
    from hybrid_flood_b200.unet import ResidualUNet, count_parameters

    z = golden("unet_d3_odd")
    net = ResidualUNet(input_channels=6, depth=3, channels=(4, 8, 16), output_channels=3)
    sd = {k[len("param/"):]: torch.from_numpy(z[k]) for k in z.files if k.startswith("param/")}
    net.load_state_dict(sd, strict=True)
    assert count_parameters(net) == int(z["n_params"])
    with torch.no_grad():
        y = net(torch.from_numpy(z["x"]))
    np.testing.assert_allclose(y.numpy(), z["y"], rtol=1e-5, atol=1e-4)
    full = ResidualUNet(input_channels=6, depth=3, channels=(16, 32, 64), output_channels=3)
    assert count_parameters(full) == int(z["n_params_16_32_64"]) == 150_883


def test_unet_head_is_zero_initialised_and_validates_arguments():
    from hybrid_flood_b200.unet import ResidualUNet, corrector_4level

    net = corrector_4level()
    with torch.no_grad():
        y = net(torch.randn(1, 5, 32, 32))
    assert tuple(y.shape) == (1, 1, 32, 32)
    assert float(y.abs().max()) == 0.0
    for bad in (dict(depth=0, channels=(4,)), dict(depth=3, channels=(4, 8)),
                dict(depth=2, channels=(4, 8), kernel_size=2)):
        with pytest.raises(ValueError):
            ResidualUNet(input_channels=3, **bad)
    with pytest.raises(ValueError):
        ResidualUNet(input_channels=3, depth=1, channels=(4,), activation="swish")


def test_relaxation_selection():
    """Restates tests/test_hybrid_rollout.py:28-34 plus the error branches of rollout.py:58-66."""
    from hybrid_flood_b200.hybrid import select_relaxation_by_validation as sel

    assert sel({0.1: 0.02, 0.05: 0.01, 0.025: 0.01, 0.0: 0.03}) == (0.025, 0.01)
    assert sel({0.1: math.nan, 0.05: 0.2, -0.1: 0.0}) == (0.05, 0.2)
    with pytest.raises(ValueError):
        sel({})
    with pytest.raises(ValueError):
        sel({0.1: math.inf, -1.0: 0.1})


def _grid(seed=0, shape=(20, 24)):
    rng = np.random.default_rng(seed)
    mask = np.ones(shape, bool)
    mask[5:9, 6:10] = False
    h = np.where(mask & (rng.uniform(size=shape) > 0.3), rng.uniform(0, 0.3, shape), 0).astype(np.float32)
    hu = np.where(h > 1e-3, rng.normal(0, 0.05, shape), 0).astype(np.float32)
    hv = np.where(h > 1e-3, rng.normal(0, 0.05, shape), 0).astype(np.float32)
    return rng, mask, h, hu, hv


def test_oracle_correction_preserves_volume():
    """tests/test_hybrid_rollout.py:37-64 on a synthetic grid: uniform depth, -0.01 residual."""
    _, mask, _, _, _ = _grid()
    depth = np.where(mask, 0.02, 0.0).astype(np.float32)
    res = np.zeros((*mask.shape, 3), np.float32)
    res[..., 0] = np.where(mask, -0.01, 0.0)
    h, hu, hv = HN.apply_residual_correction(depth, np.zeros_like(depth), np.zeros_like(depth), res, mask, 1e-4, 1.0)
    np.testing.assert_allclose(h.sum(), depth.sum(), rtol=2e-6)
    assert not hu.any() and not hv.any()


def test_oracle_correction_clip_and_depth_only():
    rng, mask, h, hu, hv = _grid(1)
    res = rng.normal(0, 0.2, (*mask.shape, 3)).astype(np.float32)
    lim = np.array([0.05, 0.01, 0.01], np.float32)
    ch, chu, chv = HN.apply_residual_correction(h, hu, hv, res, mask, 1e-4, 0.5, clip_limits=lim)
    ch2, _, _ = HN.apply_residual_correction(h, hu, hv, np.clip(res, -lim, lim), mask, 1e-4, 0.5)
    np.testing.assert_array_equal(ch, ch2)
    assert (ch >= 0).all() and not ch[~mask].any()
    np.testing.assert_allclose(ch.astype(np.float64).sum(), np.where(mask, h, 0).astype(np.float64).sum(), rtol=1e-6)
    # depth-only residual keeps the velocities
    d1, dhu, dhv = HN.apply_residual_correction(h, hu, hv, res[..., :1], mask, 1e-4, 0.5)
    u = HN._velocity(hu, h, 1e-4)
    wet = mask & (d1 > 1e-4)
    np.testing.assert_array_equal(dhu, np.where(wet, d1 * u, 0).astype(np.float32))
    # no water at all: the prediction comes back unchanged
    z = np.zeros_like(h)
    zh, _, _ = HN.apply_residual_correction(z, z, z, res, mask, 1e-4, 0.5)
    np.testing.assert_array_equal(zh, z)


def test_oracle_advance_matches_run_loop_and_nan_fills():
    from oracle import cport

    rng, mask, h, hu, hv = _grid(2)
    bed = rng.uniform(0, 0.2, mask.shape).astype(np.float32)
    p = O.make_params(bed, np.full(mask.shape, 0.03, np.float32), mask, resolution_m=2.0,
                      rainfall_times_s=[0.0, 100.0], rainfall_rates_m_s=[1e-5, 2e-5], cfl=0.9)
    dom = cport.Domain(p)
    st = O.State(h, hu, hv)
    adv, steps = HN.advance_physics_to_time(dom, st, 0.0, 30.0, 10_000)
    out, _, ref_steps, _, _ = dom.run(st, [0.0, 30.0], max_steps=10_000)
    assert steps == ref_steps
    for q in range(3):
        np.testing.assert_array_equal(adv[q], out[-1, q])
    short, n = HN.advance_physics_to_time(dom, st, 0.0, 30.0, 1)
    assert n == 1 and all(np.isnan(a).all() for a in short)


def test_oracle_features_layouts():
    rng, mask, h, hu, hv = _grid(3)
    t = rng.normal(0, 1, mask.shape).astype(np.float32)
    f = HN.network_features(h, hu, hv, mask, 1e-4, 5.5556e-6, t, t, [0, 0, 0], [1, 1, 1], 20.0)
    assert f.shape == (1, *mask.shape, 6) and f.dtype == np.float32
    np.testing.assert_array_equal(f[0, ..., 0], np.where(mask, h, 0))
    np.testing.assert_allclose(f[0, 0, 0, 3], 5.5556e-6 * 3.6e6 / 20.0, rtol=1e-6)
    g = HN.state5_features(h, hu, hv, t, mask, 20.0, [0] * 5, [2] * 5)
    assert g.shape == (1, *mask.shape, 5)
    np.testing.assert_array_equal(g[0, ..., 4], np.where(mask, np.float32(10.0), 0))


def test_output_oracle_schema_fields():
    """structured_io.py:160-209: velocities only where depth > dry, NaN off the mask."""
    from oracle import output_numpy as ON

    _, mask, h, hu, hv = _grid(4)
    d, u, v, s = ON.conserved_fields(h, hu, hv, mask, 1e-4)
    assert np.isnan(d[~mask]).all() and np.isnan(s[~mask]).all()
    wet = mask & (h > 1e-4)
    np.testing.assert_array_equal(u[wet], (hu[wet] / h[wet]).astype(np.float32))
    assert not u[mask & ~wet].any()
    np.testing.assert_array_equal(s[mask], np.hypot(u[mask], v[mask]).astype(np.float32))
    stack = ON.conserved_fields(np.stack([h, h]), np.stack([hu, hu]), np.stack([hv, hv]), mask, 1e-4)
    np.testing.assert_array_equal(stack[0][1], d)
