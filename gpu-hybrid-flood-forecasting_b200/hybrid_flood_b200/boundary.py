"""Boundary codes, ordered left, right, bottom, top.

Same codes and helpers as ``src/hybrid_flood/jax_solver/boundary_conditions.py:9-52``
of the reference: 0 = reflective wall (normal momentum negated in the ghost
ring), 1 = open / transmissive (zero-gradient copy).  The CUDA kernels apply
the ghost ring on the fly while loading edge cells; :func:`apply_ghost_cells`
materialises it with torch for inspection and tests.
"""

from __future__ import annotations

from typing import NamedTuple, Sequence

import torch

REFLECTIVE = 0
OPEN = 1


class BoundaryConfig(NamedTuple):
    """Boundary codes ordered as left, right, bottom, top."""

    types: tuple


def all_reflective() -> BoundaryConfig:
    return BoundaryConfig((REFLECTIVE, REFLECTIVE, REFLECTIVE, REFLECTIVE))


def all_open() -> BoundaryConfig:
    return BoundaryConfig((OPEN, OPEN, OPEN, OPEN))


def codes(boundaries: BoundaryConfig | Sequence[int] | None) -> tuple[int, int, int, int]:
    """Normalise a boundary argument (``None`` = all reflective, the reference default)."""
    if boundaries is None:
        return all_reflective().types
    raw = boundaries.types if isinstance(boundaries, BoundaryConfig) else boundaries
    if hasattr(raw, "tolist"):
        raw = raw.tolist()
    out = tuple(int(v) for v in raw)
    if len(out) != 4 or any(v not in (REFLECTIVE, OPEN) for v in out):
        raise ValueError("Boundary codes must be four values (left, right, bottom, top) in {0, 1}.")
    return out


def apply_ghost_cells(h: torch.Tensor, hu: torch.Tensor, hv: torch.Tensor, boundary_types):
    """Pad one ghost layer and reflect only the normal momentum component."""
    left, right, bottom, top = codes(boundary_types)
    pad = lambda a: torch.nn.functional.pad(a[None, None], (1, 1, 1, 1), mode="replicate")[0, 0]  # noqa: E731
    hg, hug, hvg = pad(h), pad(hu), pad(hv)
    if left == REFLECTIVE:
        hug[:, 0] = -hug[:, 1]
    if right == REFLECTIVE:
        hug[:, -1] = -hug[:, -2]
    if bottom == REFLECTIVE:
        hvg[0, :] = -hvg[1, :]
    if top == REFLECTIVE:
        hvg[-1, :] = -hvg[-2, :]
    return hg, hug, hvg
