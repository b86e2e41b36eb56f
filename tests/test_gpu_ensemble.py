"""Batched ensemble (one launch per step over members of uneven size) on the GPU.

Every member must evolve exactly as if it ran alone: in exact arithmetic the
ensemble's states and clocks are bit-identical to single-domain runs of the
same members; in fast arithmetic each member stays within the headline bar
(relative L2 depth <= 1e-5 after 100 steps) of the C oracle.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import cport
from oracle import swe_numpy as O

pytestmark = pytest.mark.gpu


def _members():
    from hybrid_flood_b200.workloads import tilted_bumps, urban

    rng = np.random.default_rng(5)
    out = []
    w = tilted_bumps(37, 70, seed=1)
    mask = np.ones(w.shape, bool)
    mask[10:20, 30:40] = False
    out.append(dict(bed=w.bed, manning_n=w.manning_n, domain_mask=mask, **w.solver_kwargs()))
    w = urban(64, 64, seed=2)
    out.append(dict(bed=w.bed, manning_n=w.manning_n, domain_mask=w.domain_mask,
                    **{**w.solver_kwargs(), "boundary": (1, 1, 1, 1)}))
    w = tilted_bumps(130, 200, seed=3)
    out.append(dict(bed=w.bed, manning_n=w.manning_n, domain_mask=w.domain_mask, **w.solver_kwargs()))
    w = urban(5, 300, seed=4)
    out.append(dict(bed=w.bed, manning_n=w.manning_n, domain_mask=w.domain_mask, **w.solver_kwargs()))
    w = urban(256, 129, seed=6)
    kw = w.solver_kwargs()
    kw["rainfall_multiplier"] = rng.uniform(0.5, 1.5, w.shape).astype(np.float32)
    out.append(dict(bed=w.bed, manning_n=w.manning_n, domain_mask=w.domain_mask, **kw))
    depths = [0.05, 0.3, 0.02, 0.1, np.where(rng.uniform(size=(256, 129)) > 0.5, 0.08, 0.0)]
    return out, depths


def _solver(m, arith):
    from hybrid_flood_b200.solver import B200ShallowWaterSolver

    kw = {k: v for k, v in m.items() if k not in ("bed", "manning_n", "domain_mask")}
    return B200ShallowWaterSolver(m["bed"], m["manning_n"], m["domain_mask"], **kw, arithmetic=arith)


def test_exact_ensemble_members_match_single_domain_runs(cuda_device):
    from hybrid_flood_b200.ensemble import B200Ensemble
    from hybrid_flood_b200.solver import ledger_error

    members, depths = _members()
    ens = B200Ensemble(members, arithmetic="exact")
    states = ens.initial_states(depths)
    starts = [0.0, 5.0, 10.0, 0.0, 2.5]
    res = ens.advance_(states, 30, start_times=starts)
    times = set()
    for m, st, (t, n, led), depth, t0 in zip(members, states, res, depths, starts):
        s = _solver(m, "exact")
        single, t1, n1, led1 = s.advance(s.initial_state(depth_m=depth), 30, t0)
        assert n == n1 == 30
        assert t == t1
        for a, b in zip(st, single):
            assert torch.equal(a, b)
        # Same states bit for bit; the volumes are summed in a different order
        # (float partials per 32-row batch in the paired kernel), so they agree
        # to float64 rounding of float partial sums.
        assert led["volume"] == pytest.approx(led1["volume"], rel=1e-7)
        assert ledger_error(led) < 1e-6
        times.add(round(t - t0, 6))
    assert len(times) > 1  # members advanced with their own CFL dt


def test_fast_ensemble_tracks_oracle(cuda_device):
    from hybrid_flood_b200.ensemble import B200Ensemble

    members, depths = _members()
    ens = B200Ensemble(members, arithmetic="fast")
    states = ens.initial_states(depths)
    res = ens.advance_(states, 100)
    for i in (0, 2, 4):
        m = members[i]
        kw = {k: v for k, v in m.items() if k not in ("bed", "manning_n", "domain_mask")}
        p = O.make_params(m["bed"], m["manning_n"], m["domain_mask"], **kw)
        d = cport.Domain(p)
        st = O.initial_state(p, depth_m=depths[i])
        t = 0.0
        for _ in range(100):
            dt = d.cfl_dt(st)
            st = d.step(st, dt, t)
            t += dt
        assert rel_l2(states[i].h.cpu().numpy(), st.h) < 1e-5
        assert res[i][0] == pytest.approx(t, rel=1e-5)
    from hybrid_flood_b200.solver import ledger_error

    assert max(ledger_error(r[2]) for r in res) < 1e-6


def test_ensemble_rows_per_warp_does_not_change_results(cuda_device, tmp_path):
    from hybrid_flood_b200.ensemble import B200Ensemble

    members, depths = _members()
    ens = B200Ensemble(members, arithmetic="exact")
    ref = ens.initial_states(depths)
    ens.advance_(ref, 12)
    for rows in (4, 8, 64):
        ens.set_rows_per_warp(rows)
        st = ens.initial_states(depths)
        ens.advance_(st, 12)
        for a, b in zip(st, ref):
            for x, y in zip(a, b):
                assert torch.equal(x, y)
    best = ens.autotune(ens.initial_states(depths), candidates=(8, 16), steps=4, cache=tmp_path / "tune.json")
    assert best in (8, 16)
    assert (tmp_path / "tune.json").exists()
    assert ens.autotune(ens.initial_states(depths), candidates=(8, 16), steps=4,
                        cache=tmp_path / "tune.json") == best


def test_ensemble_ledger_drift_is_the_float32_schemes(cuda_device):
    """The batched configuration (64 urban members, 200 fast steps): the worst
    member's mass-ledger closing error is the float32 state's rounding drift,
    not an accounting error -- the float32 C oracle run over the same member
    and the same simulated time drifts by the same order, and the float64 run
    closes its ledger to rounding of float64 sums."""
    from hybrid_flood_b200.ensemble import B200Ensemble
    from hybrid_flood_b200.solver import ledger_error
    from hybrid_flood_b200.workloads import as_member, ensemble_members, street_depth

    ws = ensemble_members(64)
    ens = B200Ensemble([as_member(w) for w in ws], arithmetic="fast")
    depths = [street_depth(w) for w in ws]
    res = ens.advance_(ens.initial_states(depths), 200)
    errs = [ledger_error(r[2]) for r in res]
    m = int(np.argmax(errs))
    w = ws[m]
    times = np.asarray([0.0, res[m][0]], np.float32)
    drift = {}
    for name, dtype in (("f32", np.float32), ("f64", np.float64)):
        p = O.make_params(w.bed, w.manning_n, w.domain_mask, dtype=dtype, **w.solver_kwargs())
        out = cport.Domain(p).run(O.initial_state(p, depth_m=depths[m]), times)
        drift[name] = O.ledger_error(out[4])
    print(f"worst member {m} {w.shape}: GPU {errs[m]:.3g}, float32 oracle {drift['f32']:.3g}, "
          f"float64 oracle {drift['f64']:.3g}")
    assert drift["f64"] < 1e-10
    assert errs[m] <= 1e-6 or errs[m] <= 3.0 * drift["f32"], (errs[m], drift)


def test_default_rows_per_warp_fits_one_round(cuda_device, monkeypatch):
    """Without tuning an ensemble marches the fewest rows (at least 32) whose work
    items fit the persistent grid (4 CTAs of 4 warps per SM) in one round."""
    from hybrid_flood_b200.ensemble import B200Ensemble
    from hybrid_flood_b200.workloads import as_member, urban

    monkeypatch.delenv("SWE_ENSEMBLE_ROWS", raising=False)
    sms = torch.cuda.get_device_properties(cuda_device).multi_processor_count
    slots = 4 * sms

    def items(shapes, R):
        return sum(-(-(-(-r // R) * -(-c // 64)) // 4) for r, c in shapes)

    w = urban(1024, 1024, seed=3)
    shapes = [w.shape] * 16
    ens = B200Ensemble([as_member(w)] * 16, arithmetic="fast")
    R = ens.rows_per_warp
    assert R >= 32 and items(shapes, R) <= slots
    assert R == 32 or items(shapes, R - 1) > slots
    small = urban(96, 128, seed=4)
    assert B200Ensemble([as_member(small)] * 3, arithmetic="fast").rows_per_warp == 32
