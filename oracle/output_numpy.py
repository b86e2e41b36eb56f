"""NumPy restatement of the reference's output schema fields (test oracle).

TEST INFRASTRUCTURE ONLY.  Restates ``conserved_to_xarray``
(``src/hybrid_flood/structured_io.py:160-209``) without xarray: depth, x/y
velocity (``np.divide`` where depth > dry, else 0), speed (``np.hypot`` in
float32) and elevation, each NaN off the domain mask.
"""

from __future__ import annotations

import numpy as np


def conserved_fields(h, hu, hv, mask, dry_tolerance_m):
    """(depth, x_velocity, y_velocity, velocity) of one state or a stack of states."""
    depth = np.asarray(h, dtype=np.float32).copy()
    momentum_x = np.asarray(hu, dtype=np.float32)
    momentum_y = np.asarray(hv, dtype=np.float32)
    wet = depth > np.float32(dry_tolerance_m)
    velocity_x = np.zeros_like(depth)
    velocity_y = np.zeros_like(depth)
    np.divide(momentum_x, depth, out=velocity_x, where=wet)
    np.divide(momentum_y, depth, out=velocity_y, where=wet)
    speed = np.hypot(velocity_x, velocity_y).astype(np.float32)
    off = ~np.asarray(mask, dtype=bool)
    for values in (depth, velocity_x, velocity_y, speed):
        values[..., off] = np.nan
    return depth, velocity_x, velocity_y, speed


def elevation(bed, mask):
    z = np.asarray(bed, dtype=np.float32).copy()
    z[~np.asarray(mask, dtype=bool)] = np.nan
    return z
