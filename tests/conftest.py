"""Test configuration: markers, import paths and golden-fixture helpers."""

from __future__ import annotations

import pathlib
import sys

import numpy as np
import pytest

REPO = pathlib.Path(__file__).resolve().parents[1]
PKG_ROOT = REPO / "gpu-hybrid-flood-forecasting_b200"
GOLDEN = REPO / "tests" / "golden"
for p in (str(REPO), str(PKG_ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a) device")


def golden(name: str):
    """Load ``tests/golden/<name>.npz`` (generated from the reference by make_golden.py)."""
    return np.load(GOLDEN / f"{name}.npz")


def golden_params(z, **overrides):
    """Oracle parameters rebuilt from a golden fixture's inputs and controls."""
    from oracle import swe_numpy as O

    kw = dict(
        resolution_m=float(z["ctl_dx"]), rainfall_times_s=z["rain_times"],
        rainfall_rates_m_s=z["rain_rates"], default_rainfall_m_s=float(z["ctl_default_rain"]),
        gravity_m_s2=float(z["ctl_gravity"]), cfl=float(z["ctl_cfl"]),
        dry_tolerance_m=float(z["ctl_dry"]), max_dt_s=float(z["ctl_max_dt"]),
    )
    kw.update(overrides)
    return O.make_params(z["bed"], z["manning_n"], z["domain_mask"], **kw)


def golden_solver_kwargs(z, **overrides):
    """Keyword arguments for B200ShallowWaterSolver from a golden fixture."""
    kw = dict(
        resolution_m=float(z["ctl_dx"]), rainfall_times_s=z["rain_times"],
        rainfall_rates_m_s=z["rain_rates"], default_rainfall_m_s=float(z["ctl_default_rain"]),
        gravity_m_s2=float(z["ctl_gravity"]), cfl=float(z["ctl_cfl"]),
        dry_tolerance_m=float(z["ctl_dry"]), max_dt_s=float(z["ctl_max_dt"]),
    )
    kw.update(overrides)
    return kw


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


def max_ulp(a, b) -> int:
    """Largest distance in float32 units in the last place."""
    ai = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    bi = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    ai = np.where(ai < 0, -(ai & 0x7FFFFFFF), ai)
    bi = np.where(bi < 0, -(bi & 0x7FFFFFFF), bi)
    return int(np.abs(ai - bi).max()) if ai.size else 0


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)
