"""Device-resident stepping and the captured step graphs (GPU, through the C ABI).

The resident run is the reference's step loop (``numpy_solver/shallow_water_2d.py:402-412``)
on a state that stays in the solver's buffers: advancing it in pieces of any
length must give the same state, clock, step count and ledger, bit for bit, as
one ``swe_advance`` over the whole count, whether the pieces are replayed from a
32-step CUDA graph or launched one step at a time.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _case(arith):
    from hybrid_flood_b200.solver import B200ShallowWaterSolver
    from hybrid_flood_b200.workloads import street_depth, urban

    w = urban(192, 320, seed=5)
    s = B200ShallowWaterSolver(w.bed, w.manning_n, w.domain_mask, **w.solver_kwargs(), arithmetic=arith)
    return s, s.initial_state(depth_m=street_depth(w))


@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_resident_pieces_equal_one_advance(cuda_device, arith):
    s, init = _case(arith)
    pieces = (7, 32, 33, 1, 64, 3)  # odd starts, whole graphs, graph + remainder
    total = sum(pieces)
    ref, t_ref, n_ref, led_ref = s.advance(init, total, 2.5)
    s.resident_load(init, 2.5)
    for k in pieces:
        s.resident_steps(k)
    out = type(init)(*(torch.empty_like(t) for t in init))
    t, n, led = s.resident_store(out)
    assert n == n_ref == total
    assert t == t_ref
    assert led == led_ref
    for a, b in zip(out, ref):
        assert torch.equal(a, b)
    # the store does not end the resident run: more steps continue from it
    s.resident_steps(5)
    t2, n2, _ = s.resident_store(out)
    assert n2 == total + 5 and t2 > t


def test_prepared_graphs_give_the_same_steps(cuda_device):
    """resident_prepare only captures: the prepared pieces run exactly as unprepared ones."""
    s, init = _case("fast")
    ref, t_ref, n_ref, led_ref = s.advance(init, 5 + 20 + 45, 0.0)
    s.resident_load(init, 0.0)
    s.resident_steps(5)
    s.resident_prepare(20)  # an odd start: graphs of 20 steps from buffer 1
    s.resident_prepare(0)
    s.resident_steps(20)
    s.resident_prepare(45)
    s.resident_steps(45)
    out = type(init)(*(torch.empty_like(t) for t in init))
    t, n, led = s.resident_store(out)
    assert (t, n) == (t_ref, n_ref) and led == led_ref
    for a, b in zip(out, ref):
        assert torch.equal(a, b)
    with pytest.raises(ValueError):
        s.resident_prepare(-1)


def test_resident_run_is_ended_by_other_runs(cuda_device):
    s, init = _case("fast")
    out = type(init)(*(torch.empty_like(t) for t in init))
    with pytest.raises(ValueError, match="resident"):
        s.resident_steps(1)
    s.resident_load(init)
    s.resident_steps(2)
    s.advance(init, 3)  # any other run replaces the resident state
    with pytest.raises(ValueError, match="resident"):
        s.resident_store(out)


def test_run_with_graph_chunks_matches_the_oracle_step_count(cuda_device):
    """swe_run replays 32-step graphs between its completion polls: a run of a
    few hundred steps still stops exactly at its output times."""
    from conftest import rel_l2
    from oracle import cport
    from oracle import swe_numpy as O
    from hybrid_flood_b200.workloads import street_depth, urban

    w = urban(96, 160, seed=8)
    p = O.make_params(w.bed, w.manning_n, w.domain_mask, **w.solver_kwargs())
    init = O.initial_state(p, depth_m=street_depth(w))
    times = np.asarray([0.0, 20.0, 45.0, 90.0], np.float32)
    want = cport.Domain(p).run(init, times)
    from hybrid_flood_b200.solver import B200ShallowWaterSolver

    s = B200ShallowWaterSolver(w.bed, w.manning_n, w.domain_mask, **w.solver_kwargs(), arithmetic="exact")
    got = s.run(list(init), times)
    assert got.steps_used == want[2] and got.steps_used > 64
    for k in range(len(times)):
        assert rel_l2(got.states.h[k].cpu().numpy(), want[0][k, 0]) < 1e-5


def test_run_to_host_equals_run(cuda_device):
    """The host-memory run (outputs copied back while the run continues) gives
    the same outputs, clock, step count and ledger as the device run."""
    import numpy as np

    s, init = _case("fast")
    host = [t.cpu().numpy() for t in init]
    times = np.asarray([0.0, 5.0, 11.0, 30.0, 31.5], np.float32)
    a = s.run(init, times)
    b = s.run_to_host(host, times)
    assert (a.steps_used, a.outputs_written, a.final_time_s, a.ledger) == (
        b.steps_used, b.outputs_written, b.final_time_s, b.ledger)
    for x, y in zip(a.states, b.states):
        np.testing.assert_array_equal(x.cpu().numpy(), y)
    out = [torch.zeros((len(times), *s.shape)) for _ in range(3)]  # pageable buffers work too
    c = s.run_to_host(host, times, out=out)
    for x, y in zip(a.states, c.states):
        np.testing.assert_array_equal(x.cpu().numpy(), y)
    with pytest.raises(RuntimeError, match="max_steps"):
        s.run_to_host(host, times, max_steps=3)


@pytest.mark.parametrize("arith", ["exact", "fast"])
def test_runs_follow_a_manning_change(cuda_device, arith):
    """After set_manning on a domain that has already run (its step graphs
    captured), a run equals one on a domain created with the new n (ragged
    last strip, masked cells)."""
    from hybrid_flood_b200.adjoint import set_manning
    from hybrid_flood_b200.solver import B200ShallowWaterSolver
    from hybrid_flood_b200.workloads import street_depth, urban

    w = urban(96, 200, seed=9)
    mask = w.domain_mask.copy()
    mask[40:47, 60:70] = False
    kw = w.solver_kwargs()
    s = B200ShallowWaterSolver(w.bed, w.manning_n, mask, **kw, arithmetic=arith)
    init = s.initial_state(depth_m=street_depth(w))
    s.advance(init, 20, 0.0)
    n2 = (w.manning_n * np.where(np.arange(w.shape[1]) % 64 < 2, 3.0, 0.5)[None, :]).astype(np.float32)
    set_manning(s, torch.tensor(n2, device=cuda_device))
    fresh = B200ShallowWaterSolver(w.bed, n2, mask, **kw, arithmetic=arith)
    a, ta, na, la = s.advance(init, 60, 0.0)
    b, tb, nb, lb = fresh.advance(init, 60, 0.0)
    assert (ta, na) == (tb, nb)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
