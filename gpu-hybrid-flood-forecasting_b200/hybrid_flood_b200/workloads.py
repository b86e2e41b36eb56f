"""Seeded synthetic inputs: DEMs, Manning fields and hyetographs.

The reference's own production inputs (a 517x551 Gurugram grid built from
GeoTIFF/GeoPackage files, ``src/hybrid_flood/jax_solver/shallow_water_2d.py:72-181``)
are not available, so every workload here is generated from a seed.  Layout
follows the reference grid convention (``structured_io.py:118-120``): arrays are
``[rows, cols]`` = ``[y, x]``, row index increasing northward, column index
increasing eastward.

Workloads
---------
``tilted_bumps``   plane of slope 0.005 falling toward +x (east) plus 8 Gaussian
                   bumps/depressions (amplitude U(-0.5, 0.5) m, sigma U(10, 30) m,
                   centres uniform over the domain); uniform n = 0.03; 20 mm/h
                   of rain for 600 s; reflective walls except an open (transmissive)
                   east edge; CFL 0.9; dry threshold 1e-3 m.  256x256 at dx = 2 m.
``urban``          plane of slope 0.003 falling toward +x, 30 % covered by seeded
                   rectangular blocks 5-20 cells a side raised 10 m, streets
                   (every non-block cell) 0.2 m lower; n = 0.015 on streets and
                   0.05 on blocks; 181 one-minute Gamma(k=0.8, theta=6 mm/h)
                   rain values over 10,800 s.  2048x2048 at dx = 1 m.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

MM_HR_TO_M_S = 1.0e-3 / 3600.0

REFLECTIVE = 0
OPEN = 1


@dataclass
class Workload:
    """Inputs for one solver run (all arrays ``[rows, cols]`` float32 / bool)."""

    name: str
    bed: np.ndarray
    manning_n: np.ndarray
    domain_mask: np.ndarray
    resolution_m: float
    rainfall_times_s: np.ndarray
    rainfall_rates_m_s: np.ndarray
    default_rainfall_m_s: float = 0.0
    rainfall_multiplier: np.ndarray | None = None
    boundary: tuple = (REFLECTIVE, OPEN, REFLECTIVE, REFLECTIVE)
    gravity_m_s2: float = 9.81
    cfl: float = 0.45
    dry_tolerance_m: float = 1.0e-4
    max_dt_s: float = 10.0
    duration_s: float = 600.0
    initial_depth_m: float | np.ndarray = 0.0
    meta: dict = field(default_factory=dict)

    @property
    def shape(self) -> tuple[int, int]:
        return tuple(self.bed.shape)

    def solver_kwargs(self) -> dict:
        """Keyword arguments shared by the oracle and the device solver."""
        return dict(
            resolution_m=self.resolution_m,
            rainfall_times_s=self.rainfall_times_s,
            rainfall_rates_m_s=self.rainfall_rates_m_s,
            default_rainfall_m_s=self.default_rainfall_m_s,
            rainfall_multiplier=self.rainfall_multiplier,
            boundary=self.boundary,
            gravity_m_s2=self.gravity_m_s2,
            cfl=self.cfl,
            dry_tolerance_m=self.dry_tolerance_m,
            max_dt_s=self.max_dt_s,
        )


def _gaussian_bumps(rows: int, cols: int, dx: float, count: int, rng) -> np.ndarray:
    y = (np.arange(rows, dtype=np.float64) + 0.5) * dx
    x = (np.arange(cols, dtype=np.float64) + 0.5) * dx
    amp = rng.uniform(-0.5, 0.5, count)
    sigma = rng.uniform(10.0, 30.0, count)
    cx = rng.uniform(0.0, cols * dx, count)
    cy = rng.uniform(0.0, rows * dx, count)
    out = np.zeros((rows, cols), dtype=np.float64)
    for a, s, px, py in zip(amp, sigma, cx, cy):
        gy = np.exp(-((y - py) ** 2) / (2.0 * s * s))
        gx = np.exp(-((x - px) ** 2) / (2.0 * s * s))
        out += a * np.outer(gy, gx)
    return out


def tilted_bumps(rows: int = 256, cols: int = 256, *, dx: float = 2.0, seed: int = 0,
                 slope: float = 0.005, bumps: int = 8) -> Workload:
    """Tilted plane + Gaussian bumps (the 256x256, dx = 2 m plain-forward case)."""
    rng = np.random.default_rng(seed)
    x = (np.arange(cols, dtype=np.float64) + 0.5) * dx
    plane = slope * (cols * dx - x)[None, :] * np.ones((rows, 1))
    bed = (plane + _gaussian_bumps(rows, cols, dx, bumps, rng)).astype(np.float32)
    rain = 20.0 * MM_HR_TO_M_S
    return Workload(
        name=f"tilted_bumps_{rows}x{cols}",
        bed=bed,
        manning_n=np.full((rows, cols), 0.03, dtype=np.float32),
        domain_mask=np.ones((rows, cols), dtype=bool),
        resolution_m=dx,
        rainfall_times_s=np.asarray([0.0, 600.0], dtype=np.float32),
        rainfall_rates_m_s=np.asarray([rain, rain], dtype=np.float32),
        boundary=(REFLECTIVE, OPEN, REFLECTIVE, REFLECTIVE),
        cfl=0.9,
        dry_tolerance_m=1.0e-3,
        max_dt_s=10.0,
        duration_s=600.0,
        meta={"seed": seed, "slope": slope, "bumps": bumps, "downslope": "+x (east)"},
    )


def gamma_hyetograph(seed: int, *, values: int = 181, step_s: float = 60.0,
                     shape_k: float = 0.8, scale_mm_hr: float = 6.0):
    """``values`` rain intensities drawn from Gamma(k, theta) mm/h, one per ``step_s``."""
    rng = np.random.default_rng(seed)
    rates = rng.gamma(shape_k, scale_mm_hr, values) * MM_HR_TO_M_S
    times = np.arange(values, dtype=np.float64) * step_s
    return times.astype(np.float32), rates.astype(np.float32)


def urban_blocks(rows: int, cols: int, rng, *, coverage: float = 0.30,
                 min_side: int = 5, max_side: int = 20, rects: list | None = None) -> np.ndarray:
    """Boolean block mask: seeded rectangles until ``coverage`` of the cells is covered.

    ``rects``, when given, receives the rectangles drawn, in order, as
    ``(row0, col0, height, width)``."""
    blocks = np.zeros((rows, cols), dtype=bool)
    target = coverage * rows * cols
    covered = 0
    while covered < target:
        h = int(rng.integers(min_side, max_side + 1))
        w = int(rng.integers(min_side, max_side + 1))
        r0 = int(rng.integers(0, max(rows - h, 0) + 1))
        c0 = int(rng.integers(0, max(cols - w, 0) + 1))
        if rects is not None:
            rects.append((r0, c0, h, w))
        patch = blocks[r0:r0 + h, c0:c0 + w]
        covered += int(patch.size - patch.sum())
        patch[...] = True
    return blocks


def urban_rects(rows: int, cols: int, *, seed: int = 1, **kw) -> list:
    """The rectangles ``urban(rows, cols, seed=seed)`` draws, in order."""
    rects: list = []
    urban_blocks(rows, cols, np.random.default_rng(seed), rects=rects, **kw)
    return rects


def urban(rows: int = 2048, cols: int = 2048, *, dx: float = 1.0, seed: int = 1,
          slope: float = 0.003, rain_scale: float = 1.0, n_scale: float = 1.0,
          duration_s: float = 10_800.0) -> Workload:
    """Synthetic urban DEM (the 2048x2048, dx = 1 m plain-forward-at-scale case)."""
    rng = np.random.default_rng(seed)
    x = (np.arange(cols, dtype=np.float64) + 0.5) * dx
    plane = slope * (cols * dx - x)[None, :] * np.ones((rows, 1))
    blocks = urban_blocks(rows, cols, rng)
    bed = plane + np.where(blocks, 10.0, -0.2)
    manning = np.where(blocks, 0.05, 0.015) * n_scale
    times, rates = gamma_hyetograph(seed + 7919)
    return Workload(
        name=f"urban_{rows}x{cols}",
        bed=bed.astype(np.float32),
        manning_n=manning.astype(np.float32),
        domain_mask=np.ones((rows, cols), dtype=bool),
        resolution_m=dx,
        rainfall_times_s=times,
        rainfall_rates_m_s=(rates * np.float32(rain_scale)).astype(np.float32),
        boundary=(REFLECTIVE, OPEN, REFLECTIVE, REFLECTIVE),
        cfl=0.9,
        dry_tolerance_m=1.0e-3,
        max_dt_s=10.0,
        duration_s=duration_s,
        meta={"seed": seed, "slope": slope, "block_fraction": float(blocks.mean()),
              "downslope": "+x (east)", "rain_scale": rain_scale, "n_scale": n_scale},
    )


ENSEMBLE_SHAPES = ((256, 256), (512, 512), (1024, 1024), (768, 1536))


def ensemble_members(n: int = 64, *, seed: int = 2024, shapes=ENSEMBLE_SHAPES,
                     rain_sigma_log: float = 0.4, n_range=(0.8, 1.2)) -> list[Workload]:
    """The batched-ensemble case: ``n`` urban members of uneven size.

    Member m uses DEM seed 1000 + m; its size is drawn uniformly from ``shapes``;
    its rain is scaled by a LogNormal(0, sigma_log) factor and its Manning n by
    U(n_range).  Expected total for 64 members: 64 x 638,976 = 40.9 M cells.
    """
    rng = np.random.default_rng(seed)
    picks = rng.integers(0, len(shapes), n)
    rain_f = rng.lognormal(0.0, rain_sigma_log, n)
    n_f = rng.uniform(n_range[0], n_range[1], n)
    out = []
    for m in range(n):
        rows, cols = shapes[int(picks[m])]
        w = urban(rows, cols, seed=1000 + m, rain_scale=float(rain_f[m]), n_scale=float(n_f[m]))
        w.name = f"member{m:02d}_{rows}x{cols}"
        out.append(w)
    return out


def as_member(w: Workload) -> dict:
    """Keyword arguments of one ensemble member (the B200ShallowWaterSolver constructor's)."""
    return dict(bed=w.bed, manning_n=w.manning_n, domain_mask=w.domain_mask, **w.solver_kwargs())


def street_depth(w: Workload, depth_m: float = 0.05) -> np.ndarray:
    """Initial ponding of ``depth_m`` on the street cells of an urban workload
    (cells within 1 m of the sloping plane; block tops stay dry)."""
    rows, cols = w.shape
    slope = float(w.meta.get("slope", 0.003))
    x = (np.arange(cols, dtype=np.float64) + 0.5) * w.resolution_m
    plane = slope * (cols * w.resolution_m - x)[None, :]
    return np.where((w.bed - plane) < 1.0, depth_m, 0.0).astype(np.float32)


def smoothed_lognormal_field(shape, *, median: float, sigma_log: float, seed: int,
                             smooth_cells: int = 9) -> np.ndarray:
    """Log-normal field (median, sigma of log) smoothed by a ``smooth_cells``-wide Gaussian."""
    rng = np.random.default_rng(seed)
    g = rng.normal(0.0, 1.0, shape)
    radius = smooth_cells // 2
    x = np.arange(-radius, radius + 1, dtype=np.float64)
    sig = smooth_cells / 6.0
    k = np.exp(-0.5 * (x / sig) ** 2)
    k /= k.sum()
    pad = np.pad(g, radius, mode="reflect")
    sm = np.apply_along_axis(lambda v: np.convolve(v, k, mode="valid"), 1, pad)
    sm = np.apply_along_axis(lambda v: np.convolve(v, k, mode="valid"), 0, sm)
    sm /= sm.std() if sm.std() > 0 else 1.0
    return (median * np.exp(sigma_log * sm)).astype(np.float32)


def adjoint_case(rows: int = 512, cols: int = 512, *, dx: float = 2.0, truth_seed: int = 1,
                 estimate_seed: int = 2, gauges: int = 16, gauge_seed: int = 7):
    """The adjoint case: tilted-plane DEM as the 256x256 case (on a 512x512, dx = 2 m grid),
    log-normal Manning n (median 0.03, sigma_log 0.3, 9-cell smoothing); the truth
    uses ``truth_seed`` and the estimate ``estimate_seed``; ``gauges`` random gauge cells.
    Returns (workload, n_truth, n_estimate, gauge_index)."""
    w = tilted_bumps(rows, cols, dx=dx, seed=0)
    n_truth = smoothed_lognormal_field((rows, cols), median=0.03, sigma_log=0.3, seed=truth_seed)
    n_est = smoothed_lognormal_field((rows, cols), median=0.03, sigma_log=0.3, seed=estimate_seed)
    rng = np.random.default_rng(gauge_seed)
    idx = rng.choice(rows * cols, size=gauges, replace=False).astype(np.int64)
    w.manning_n = n_est
    w.name = f"adjoint_{rows}x{cols}"
    return w, n_truth, n_est, idx
