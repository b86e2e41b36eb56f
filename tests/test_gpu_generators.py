"""Device generators of the synthetic inputs (GPU, through the C ABI).

Deterministic parts are checked bit for bit against the host generators of
``hybrid_flood_b200.workloads`` (the plane, the block mask from the same
rectangles, the bed and Manning arrays); the smoothing of a given noise field
to within one float32 ulp (its float64 sums may be added in another order);
the generators' own random draws by their distributions.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,seed", [((96, 160), 3), ((512, 384), 11), ((2048, 2048), 1)])
def test_urban_from_numpy_rectangles_is_bit_exact(cuda_device, shape, seed):
    from hybrid_flood_b200.generators import urban_device
    from hybrid_flood_b200.workloads import urban, urban_rects

    rows, cols = shape
    w = urban(rows, cols, seed=seed, n_scale=1.1, rain_scale=0.8)
    rects = urban_rects(rows, cols, seed=seed)
    m = urban_device(rows, cols, seed=seed, n_scale=1.1, rain_scale=0.8, rects=rects)
    assert m["blocks_used"] == len(rects)
    np.testing.assert_array_equal(m["bed"].cpu().numpy(), w.bed)
    np.testing.assert_array_equal(m["manning_n"].cpu().numpy(), w.manning_n)
    assert m["block_mask"].cpu().numpy().mean() == pytest.approx(w.meta["block_fraction"], abs=0)
    # the device generator's own hyetograph has the host one's shape and time axis
    np.testing.assert_array_equal(m["rainfall_times_s"], w.rainfall_times_s)
    assert m["rainfall_rates_m_s"].shape == w.rainfall_rates_m_s.shape


def test_urban_own_draws_distribution_and_determinism(cuda_device):
    from hybrid_flood_b200.generators import urban_device

    rows, cols = 1024, 1536
    a = urban_device(rows, cols, seed=1234)
    b = urban_device(rows, cols, seed=1234)
    c = urban_device(rows, cols, seed=1235)
    assert torch.equal(a["bed"], b["bed"]) and torch.equal(a["manning_n"], b["manning_n"])
    assert not torch.equal(a["bed"], c["bed"])
    frac = a["block_mask"].float().mean().item()
    # the rectangle that crosses the target adds at most 20 x 20 cells
    assert 0.30 <= frac <= 0.30 + 400 / (rows * cols)
    x = (np.arange(cols) + 0.5) * 1.0
    plane = 0.003 * (cols - x)[None, :]
    blk = a["block_mask"].cpu().numpy()
    bed = a["bed"].cpu().numpy()
    np.testing.assert_array_equal(bed, np.where(blk, plane + 10.0, plane - 0.2).astype(np.float32))
    man = a["manning_n"].cpu().numpy()
    assert set(np.unique(man).tolist()) == {np.float32(0.015), np.float32(0.05)}
    # expected number of rectangles: coverage 1 - exp(-n E[area] / cells) = 0.3, E[area] = 12.5^2
    expect = -np.log(0.7) * rows * cols / 12.5 ** 2
    assert 0.8 * expect < a["blocks_used"] < 1.25 * expect


def test_gamma_hyetograph_distribution(cuda_device):
    from scipy import stats

    from hybrid_flood_b200.generators import gamma_hyetograph_device
    from hybrid_flood_b200.workloads import MM_HR_TO_M_S

    n = 20000
    t, r = gamma_hyetograph_device(77, values=n, step_s=60.0, shape_k=0.8, scale_mm_hr=6.0)
    t2, r2 = gamma_hyetograph_device(77, values=n)
    assert torch.equal(r, r2)
    np.testing.assert_array_equal(t.cpu().numpy(), (np.arange(n) * 60.0).astype(np.float32))
    mm = r.cpu().numpy().astype(np.float64) / MM_HR_TO_M_S
    assert mm.min() > 0
    assert mm.mean() == pytest.approx(0.8 * 6.0, rel=0.03)
    assert mm.var() == pytest.approx(0.8 * 36.0, rel=0.08)
    ks = stats.kstest(mm, stats.gamma(a=0.8, scale=6.0).cdf)
    assert ks.pvalue > 1e-3, ks
    # and for a shape above one (Marsaglia-Tsang without the boost)
    _, r3 = gamma_hyetograph_device(5, values=n, shape_k=2.5, scale_mm_hr=1.0)
    ks3 = stats.kstest(r3.cpu().numpy().astype(np.float64) / MM_HR_TO_M_S, stats.gamma(a=2.5, scale=1.0).cdf)
    assert ks3.pvalue > 1e-3, ks3


def test_lognormal_field_from_numpy_noise_matches_host(cuda_device):
    from hybrid_flood_b200.generators import lognormal_field_device
    from hybrid_flood_b200.workloads import smoothed_lognormal_field

    shape, seed = (300, 257), 2
    want = smoothed_lognormal_field(shape, median=0.03, sigma_log=0.3, seed=seed)
    noise = torch.from_numpy(np.random.default_rng(seed).normal(0.0, 1.0, shape)).to(cuda_device)
    got = lognormal_field_device(shape, median=0.03, sigma_log=0.3, seed=0, noise=noise).cpu().numpy()
    # same float64 operations up to the order of the smoothing and moment sums: at most one float32 ulp
    np.testing.assert_allclose(got, want, rtol=1.2e-7, atol=0)


def test_lognormal_field_own_draws(cuda_device):
    from hybrid_flood_b200.generators import lognormal_field_device

    f = lognormal_field_device((1024, 768), median=0.03, sigma_log=0.3, seed=9).cpu().numpy().astype(np.float64)
    g = lognormal_field_device((1024, 768), median=0.03, sigma_log=0.3, seed=9).cpu().numpy().astype(np.float64)
    np.testing.assert_array_equal(f, g)
    z = np.log(f / 0.03) / 0.3
    assert z.std() == pytest.approx(1.0, abs=1e-5)  # normalised to unit standard deviation
    assert abs(z.mean()) < 0.05 and np.median(f) == pytest.approx(0.03, rel=0.05)
    # smoothing correlates neighbours (a 9-cell Gaussian, sigma 1.5 cells)
    assert np.corrcoef(z[:, :-1].ravel(), z[:, 1:].ravel())[0, 1] > 0.8


def test_solver_from_device_fields_matches_host_fields(cuda_device):
    """A domain packed from device memory runs the same steps as one packed from the host."""
    from hybrid_flood_b200.generators import street_depth_device, urban_device
    from hybrid_flood_b200.solver import B200ShallowWaterSolver
    from hybrid_flood_b200.workloads import street_depth, urban, urban_rects

    rows, cols = 256, 320
    rects = urban_rects(rows, cols, seed=4)
    m = urban_device(rows, cols, seed=4, rects=rects)
    w = urban(rows, cols, seed=4)
    kw = {k: v for k, v in m.items() if k not in ("bed", "manning_n", "domain_mask", "block_mask", "blocks_used")}
    kw["rainfall_rates_m_s"] = w.rainfall_rates_m_s  # the host hyetograph, so the runs compare
    kw["rainfall_times_s"] = w.rainfall_times_s
    sd = B200ShallowWaterSolver(m["bed"], m["manning_n"], m["domain_mask"], **kw, arithmetic="fast")
    sh = B200ShallowWaterSolver(w.bed, w.manning_n, w.domain_mask, **kw, arithmetic="fast")
    d_dev = street_depth_device(m)
    np.testing.assert_array_equal(d_dev.cpu().numpy(), street_depth(w))
    a, ta, _, _ = sd.advance(sd.initial_state(depth_m=street_depth(w)), 40)
    b, tb, _, _ = sh.advance(sh.initial_state(depth_m=street_depth(w)), 40)
    assert ta == tb
    for x, y in zip(a, b):
        assert torch.equal(x, y)
