"""Allocation-free CFL reduction, checked against the allocating entry point (GPU).

``swe_max_inverse_dt_noalloc`` is for callers that cannot call cudaMalloc when
they need a CFL time step: code running under a framework's caching allocator
(where a direct cudaMalloc can fail even though the framework's pool has room)
and time-stepping loops that forbid allocation once running.  It keeps its
scratch in a fixed device array inside the library, so two calls in a row must
each give the same answer as ``swe_max_inverse_dt`` (which uses a domain and
allocates) -- the second call must not see leftovers of the first.

The file name makes pytest collect it last, after every other test.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _noalloc(lib, state, mask_dev, rows, cols, out, *, g, dry, dx):
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    return lib.swe_max_inverse_dt_noalloc(
        ptr(state[0]), ptr(state[1]), ptr(state[2]), state[0].stride(0), ptr(mask_dev),
        rows, cols, g, dry, dx, dx, ptr(out), stream)


def test_noalloc_matches_allocating_entry_point_on_two_calls(cuda_device):
    from hybrid_flood_b200 import _lib
    from hybrid_flood_b200.solver import B200ShallowWaterSolver
    from hybrid_flood_b200.workloads import urban

    rows, cols = 384, 512
    w = urban(rows, cols, seed=3)
    mask = np.ones((rows, cols), dtype=bool)
    mask[100:140, 200:260] = False
    kw = w.solver_kwargs()
    s = B200ShallowWaterSolver(w.bed, w.manning_n, mask, **kw, arithmetic="exact")
    rng = np.random.default_rng(9)
    states = []
    for depth, speed in ((0.05, 0.2), (0.4, 1.5)):
        st = s.initial_state(depth_m=rng.uniform(0.0, depth, (rows, cols)).astype(np.float32),
                             x_velocity_m_s=rng.normal(0.0, speed, (rows, cols)).astype(np.float32),
                             y_velocity_m_s=rng.normal(0.0, speed, (rows, cols)).astype(np.float32))
        states.append(st)
    lib = _lib.load()
    mask_dev = torch.from_numpy(mask.astype(np.uint8)).to(cuda_device)
    out = torch.full((1,), -1.0, dtype=torch.float32, device=cuda_device)
    got = []
    for st in states:  # two calls in a row through the same static scratch
        rc = _noalloc(lib, st, mask_dev, rows, cols, out, g=kw["gravity_m_s2"],
                      dry=kw["dry_tolerance_m"], dx=kw["resolution_m"])
        _lib.check(rc, "swe_max_inverse_dt_noalloc")
        torch.cuda.synchronize()
        got.append(float(out.item()))
    want = [s.max_inverse_dt(st) for st in states]
    # Both reductions evaluate the same float32 operations and take a maximum,
    # which is order independent: the results must be identical.
    assert got == want
    assert want[0] != want[1]


def test_noalloc_padded_pitch_matches_allocating_entry_point(cuda_device):
    """State planes whose row pitch exceeds the column count (views into wider
    buffers): the kernel reads the state at the pitch and the mask densely, and
    the result equals the allocating entry point's on the same views, twice."""
    from hybrid_flood_b200 import _lib
    from hybrid_flood_b200.solver import B200ShallowWaterSolver, SWEState
    from hybrid_flood_b200.workloads import urban

    rows, cols, pad = 200, 300, 37
    w = urban(rows, cols, seed=4)
    mask = np.ones((rows, cols), dtype=bool)
    mask[20:90, 5:40] = False
    kw = w.solver_kwargs()
    s = B200ShallowWaterSolver(w.bed, w.manning_n, mask, **kw, arithmetic="exact")
    rng = np.random.default_rng(17)
    lib = _lib.load()
    mask_dev = torch.from_numpy(mask.astype(np.uint8)).to(cuda_device)
    out = torch.full((1,), -1.0, dtype=torch.float32, device=cuda_device)
    got, want = [], []
    for depth, speed in ((0.3, 2.0), (0.02, 0.1)):
        dense = s.initial_state(depth_m=rng.uniform(0.0, depth, (rows, cols)).astype(np.float32),
                                x_velocity_m_s=rng.normal(0.0, speed, (rows, cols)).astype(np.float32),
                                y_velocity_m_s=rng.normal(0.0, speed, (rows, cols)).astype(np.float32))
        # padding filled with values that would dominate the maximum if read
        wide = [torch.full((rows, cols + pad), 50.0, device=cuda_device) for _ in range(3)]
        views = []
        for big, a in zip(wide, dense):
            v = big[:, :cols]
            v.copy_(a)
            views.append(v)
        st = SWEState(*views)
        assert st.h.stride(0) == cols + pad
        rc = _noalloc(lib, st, mask_dev, rows, cols, out, g=kw["gravity_m_s2"],
                      dry=kw["dry_tolerance_m"], dx=kw["resolution_m"])
        _lib.check(rc, "swe_max_inverse_dt_noalloc")
        torch.cuda.synchronize()
        got.append(float(out.item()))
        want.append(s.max_inverse_dt(st))
    assert got == want
    assert want[0] != want[1]


def test_noalloc_rejects_grids_above_its_limit(cuda_device):
    from hybrid_flood_b200 import _lib

    lib = _lib.load()
    t = torch.zeros((1, 4096), device=cuda_device)
    mask = torch.ones((1, 4096), dtype=torch.uint8, device=cuda_device)
    out = torch.zeros(1, device=cuda_device)
    rows = _lib.SWE_NOALLOC_MAX_CELLS // 4096 + 1
    rc = _noalloc(lib, (t, t, t), mask, rows, 4096, out, g=9.81, dry=1e-3, dx=1.0)
    assert rc == _lib.SWE_ERR_INVALID
    assert "allocation-free limit" in _lib.last_error()
