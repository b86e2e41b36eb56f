"""Synthetic inputs generated in device memory (the C ABI's ``swe_generate_*``).

The reference conditions its terrain on the host from GIS inputs
(``src/hybrid_flood/dem/synthetic_terrain.py:114`` ``generate_base_terrain``,
``src/hybrid_flood/dem/urban_conditioning.py:128`` ``condition_urban_terrain``).
The measurement workloads are seeded synthetic fields of the same kind
(:mod:`hybrid_flood_b200.workloads` builds them on the host with NumPy); these
functions build the same kinds of field on the GPU, so that ensembles of many
members and refined targets need no host generation or upload:

* :func:`urban_device` -- the urban DEM (plane, seeded blocks raised 10 m,
  streets 0.2 m lower), its Manning field and a Gamma hyetograph;
* :func:`gamma_hyetograph_device` -- one-minute Gamma(k, theta) rain values;
* :func:`lognormal_field_device` -- a smoothed log-normal field (Manning n).

Given the rectangles NumPy drew (``workloads.urban_rects``), :func:`urban_device`
reproduces ``workloads.urban``'s bed and Manning arrays bit for bit; with its
own counter-based draws it produces fields of the same distribution.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .workloads import MM_HR_TO_M_S, OPEN, REFLECTIVE


def _stream(device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _device(device) -> torch.device:
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    return dev if dev.index is not None else torch.device("cuda", torch.cuda.current_device())


def gamma_hyetograph_device(seed: int, *, values: int = 181, step_s: float = 60.0, shape_k: float = 0.8,
                            scale_mm_hr: float = 6.0, device=None) -> tuple[torch.Tensor, torch.Tensor]:
    """``values`` rain rates (m/s) drawn from Gamma(k, theta) mm/h, one per ``step_s``; device float32."""
    dev = _device(device)
    lib = _lib.load()
    times = torch.empty(values, dtype=torch.float32, device=dev)
    rates = torch.empty(values, dtype=torch.float32, device=dev)
    with torch.cuda.device(dev):
        rc = lib.swe_generate_gamma_hyetograph(int(values), float(step_s), float(shape_k), float(scale_mm_hr),
                                               MM_HR_TO_M_S, int(seed) & 0xFFFFFFFFFFFFFFFF,
                                               ctypes.c_void_p(times.data_ptr()), ctypes.c_void_p(rates.data_ptr()),
                                               _stream(dev))
    _lib.check(rc, "swe_generate_gamma_hyetograph")
    return times, rates


def lognormal_field_device(shape, *, median: float, sigma_log: float, seed: int, smooth_cells: int = 9,
                           noise: torch.Tensor | None = None, device=None) -> torch.Tensor:
    """Log-normal field (median, sigma of log) smoothed by a ``smooth_cells``-wide
    Gaussian, as ``workloads.smoothed_lognormal_field``; ``noise`` (device
    float64, the field's shape) replaces the generator's own normal draws."""
    dev = _device(device)
    rows, cols = (int(x) for x in shape)
    lib = _lib.load()
    out = torch.empty((rows, cols), dtype=torch.float32, device=dev)
    nptr = None
    if noise is not None:
        if not (noise.device == dev and noise.dtype == torch.float64 and tuple(noise.shape) == (rows, cols)):
            raise ValueError("noise must be a device float64 tensor of the field's shape")
        noise = noise.contiguous()
        nptr = ctypes.c_void_p(noise.data_ptr())
    with torch.cuda.device(dev):
        rc = lib.swe_generate_lognormal_field(rows, cols, float(median), float(sigma_log), int(smooth_cells),
                                              int(seed) & 0xFFFFFFFFFFFFFFFF, nptr, ctypes.c_void_p(out.data_ptr()),
                                              _stream(dev))
    _lib.check(rc, "swe_generate_lognormal_field")
    return out


def urban_device(rows: int = 2048, cols: int = 2048, *, dx: float = 1.0, seed: int = 1, slope: float = 0.003,
                 rain_scale: float = 1.0, n_scale: float = 1.0, coverage: float = 0.30, min_side: int = 5,
                 max_side: int = 20, rects=None, device=None) -> dict:
    """The urban workload built on the device.

    Returns the keyword arguments of :class:`B200ShallowWaterSolver` (and of an
    ensemble member): ``bed``, ``manning_n`` and ``domain_mask`` as device
    tensors, the hyetograph as host arrays, and the controls of
    ``workloads.urban``; plus ``block_mask`` (device bool) and ``blocks_used``.
    ``rects`` (a sequence of ``(row0, col0, height, width)``) replaces the
    generator's own rectangle draws.
    """
    dev = _device(device)
    lib = _lib.load()
    bed = torch.empty((rows, cols), dtype=torch.float32, device=dev)
    man = torch.empty((rows, cols), dtype=torch.float32, device=dev)
    blocks = torch.empty((rows, cols), dtype=torch.uint8, device=dev)
    q = _lib.UrbanDesc()
    q.rows, q.cols, q.dx, q.slope, q.coverage = int(rows), int(cols), float(dx), float(slope), float(coverage)
    q.min_side, q.max_side = int(min_side), int(max_side)
    q.block_raise_m, q.street_offset_m = 10.0, -0.2
    q.n_block, q.n_street, q.n_scale = 0.05, 0.015, float(n_scale)
    q.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    keep = None
    if rects is not None:
        keep = np.ascontiguousarray(np.asarray(rects, dtype=np.int32).reshape(-1, 4))
        q.n_rects, q.rects = int(keep.shape[0]), keep.ctypes.data
    used = ctypes.c_int32()
    with torch.cuda.device(dev):
        rc = lib.swe_generate_urban(ctypes.byref(q), ctypes.c_void_p(bed.data_ptr()), ctypes.c_void_p(man.data_ptr()),
                                    ctypes.c_void_p(blocks.data_ptr()), ctypes.byref(used), _stream(dev))
    _lib.check(rc, "swe_generate_urban")
    del keep
    times, rates = gamma_hyetograph_device(seed + 7919, device=dev)
    rates_h = (rates.cpu().numpy() * np.float32(rain_scale)).astype(np.float32)
    return dict(
        bed=bed, manning_n=man, domain_mask=torch.ones((rows, cols), dtype=torch.bool, device=dev),
        resolution_m=float(dx), rainfall_times_s=times.cpu().numpy(), rainfall_rates_m_s=rates_h,
        default_rainfall_m_s=0.0, boundary=(REFLECTIVE, OPEN, REFLECTIVE, REFLECTIVE), gravity_m_s2=9.81,
        cfl=0.9, dry_tolerance_m=1.0e-3, max_dt_s=10.0, block_mask=blocks.bool(), blocks_used=int(used.value),
    )


def street_depth_device(member: dict, depth_m: float = 0.05, slope: float = 0.003) -> torch.Tensor:
    """Initial ponding of ``depth_m`` on the street cells of a device urban member
    (cells within 1 m of the sloping plane), as ``workloads.street_depth``."""
    bed = member["bed"]
    rows, cols = bed.shape
    dx = float(member["resolution_m"])
    x = (torch.arange(cols, dtype=torch.float64, device=bed.device) + 0.5) * dx
    plane = slope * (cols * dx - x)[None, :]
    return torch.where((bed.double() - plane) < 1.0, depth_m, 0.0).to(torch.float32)


def member_fields(member: dict) -> dict:
    """The solver keyword arguments of a device member (drops the generator's extras)."""
    return {k: v for k, v in member.items() if k not in ("block_mask", "blocks_used")}
