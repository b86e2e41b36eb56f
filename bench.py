"""Benchmark of the B200 shallow-water step (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--arith exact|fast] [--rows 2048 --cols 2048]

Workload: the 2048x2048 plain-forward-at-scale case -- synthetic urban DEM
at dx = 1 m (plane of slope 0.003, 30 % seeded building blocks raised 10 m,
streets 0.2 m lower), Manning n 0.015 on streets / 0.05 on blocks, a
181-value Gamma hyetograph over 10,800 s, open east edge, CFL 0.9, dry
threshold 1e-3 m.  The state starts ponded (5 cm on streets) and is spun up
for 200 steps before warm-up, so the timed steps see moving water.

A "step" is one finite-volume time step over the whole grid: CFL dt from the
previous state's reduction, fluxes, update, friction, masks, and the next CFL
reduction plus FP64 ledger, all inside the fused kernel.  The state is loaded
into the solver's resident buffers before timing; the timed region is exactly
K step launches (whole 32-step CUDA graphs where K allows), bracketed by a
barrier and a device synchronisation, timed with CUDA events on the launching
stream.  ``value`` is cell-updates/s over those K steps.  The per-step working
set is 134 MB (five input planes and three output planes of 16.8 MB), above the
126 MB L2, so no flush is inserted.  ``e2e`` times ``B200ShallowWaterSolver.run_to_host``
called once with HOST (pinned NumPy-backed) state over the workload's 10,800 s
forecast window with an output every 600 s, the host->device copy of the state
and the device->host copy of every recorded snapshot inside the timed region.  The line
also carries the same resident timing in exact arithmetic (``exact_arithmetic``).

Multi-GPU: one process per GPU, each advancing its own replica of the domain
(weak scaling, no collective in the timed region); ``value`` is the sum over
ranks divided by the slowest rank's time.  ``--decompose`` also times the one
domain split into row strips across the ranks (halo exchange over NCCL, strong
scaling) in a sub-object.

``--impl reference`` times the CPU implementation of the same path: the C
restatement of the reference step (oracle/swe_oracle.c, OpenMP over all host
threads) on the same workload and the same config, whole-grid steps.
"""

from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import sys
import threading
import time

import numpy as np

REPO = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "gpu-hybrid-flood-forecasting_b200"))
sys.path.insert(0, str(REPO))

METRIC = "cell-updates/s (plain single-domain step, 2048x2048 urban)"
BYTES_PER_CELL = 32  # h, hu, hv, bed, n^2 read (20 B) + h, hu, hv written (12 B)
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one fast-arithmetic
# step_kernel_pair launch on the default 2048x2048 workload, per cell-update, from an
# ncu capture of that launch: reported as roofline.traffic for that configuration only.
NCU_TRAFFIC_PER_CELL = (92.77184e6 + 17.041664e6) / 4194304
REFERENCE_MAX_STEPS = 200  # whole-grid steps the CPU reference arm times at most


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--arith", choices=["exact", "fast"], default="fast")
    ap.add_argument("--rows", type=int, default=2048)
    ap.add_argument("--cols", type=int, default=2048)
    ap.add_argument("--spinup", type=int, default=200)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-window-s", type=float, default=10800.0,
                    help="simulated window of the e2e forecast (the workload's hyetograph window)")
    ap.add_argument("--e2e-every-s", type=float, default=600.0, help="output interval of the e2e forecast")
    ap.add_argument("--e2e-max-steps", type=int, default=200_000, help="step cap of the e2e forecast")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--ensemble-members", type=int, default=64)
    ap.add_argument("--ensemble-steps", type=int, default=200)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--adjoint-steps", type=int, default=2000)
    ap.add_argument("--no-hybrid", action="store_true")
    ap.add_argument("--hybrid-members", type=int, default=16)
    ap.add_argument("--hybrid-size", type=int, default=1024)
    ap.add_argument("--hybrid-intervals", type=int, default=10)
    ap.add_argument("--no-training", action="store_true")
    ap.add_argument("--training-members", type=int, default=16)
    ap.add_argument("--training-size", type=int, default=1024)
    ap.add_argument("--no-aux", action="store_true", help="skip the timing of the kernels around the step")
    ap.add_argument("--exact-steps", type=int, default=200, help="steps of the exact-arithmetic leg (0: skip)")
    ap.add_argument("--aux-size", type=int, default=4096)
    ap.add_argument("--decompose", action="store_true",
                    help="also time the single domain split into row strips, one per GPU over NCCL (strong scaling)")
    return ap.parse_args()


def _workload(rows, cols):
    from hybrid_flood_b200.workloads import street_depth, urban

    w = urban(rows, cols)
    return w, street_depth(w)


def _config(args, world: int) -> dict:
    """The workload description both arms print (the driver compares them)."""
    return {"workload": f"urban {args.rows}x{args.cols} dx=1m (plain forward at scale)",
            "cells_per_gpu": args.rows * args.cols, "parallelism": f"replicas{world}",
            "l2": "per-step working set 134 MB > 126 MB L2; no flush", "spinup_steps": args.spinup}


def _peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _tensor_peak():
    """Dense bf16 TFLOP/s: the sustained cuBLAS figure of MEASURED_PEAKS.json, else the fallback."""
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        for key in ("bf16_tflops_sustained", "bf16_tflops"):
            if key in d:
                return float(d[key]), f"measured ({key})"
    return 1400.0, "fallback (sustained)"


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled through NVML in a
    background thread every ~0.5 ms; :meth:`summary` keeps the samples taken
    between :meth:`mark_start` and :meth:`mark_end` (the timed region)."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, device):
        self.device = device
        self.samples: list[tuple[float, float, int]] = []
        self.window = (None, None)
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        self._nv = None
        self._h = None

    def __enter__(self):
        try:
            import pynvml as nv
            import torch

            nv.nvmlInit()
            self._nv = nv
            props = torch.cuda.get_device_properties(self.device)
            try:
                bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
                self._h = nv.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:  # noqa: BLE001 - fall back to the ordinal
                self._h = nv.nvmlDeviceGetHandleByIndex(self.device.index or 0)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self._h, nv.NVML_CLOCK_SM))
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        except Exception:  # noqa: BLE001 - no NVML: report no samples
            self._nv = None
        return self

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self._h))
                self.samples.append((time.perf_counter(), mhz, rs))
            except Exception:  # noqa: BLE001
                return
            time.sleep(0.0005)

    def mark_start(self):
        self.window = (time.perf_counter(), None)

    def sample_until(self, event, min_samples: int = 3):
        """Sample on this thread while `event` (the end of the timed region) has
        not completed: a short region (a few launches) still gets samples taken
        while its kernels run."""
        if self._nv is None:
            return
        nv = self._nv
        taken = 0
        while taken < 1000 and not event.query():  # each sample starts while the region runs
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self._h))
            except Exception:  # noqa: BLE001
                return
            self.samples.append((time.perf_counter(), mhz, rs))
            taken += 1

    def mark_end(self):
        self.window = (self.window[0], time.perf_counter())

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=2)
        if self._nv is not None:
            try:
                self._nv.nvmlShutdown()
            except Exception:  # noqa: BLE001
                pass

    def summary(self) -> dict:
        t0, t1 = self.window
        inside = [s for s in self.samples if t0 is not None and t1 is not None and t0 <= s[0] <= t1]
        reasons = set()
        nv = self._nv
        for _, _, rs in inside:
            for name, attr in self.REASONS:
                bit = getattr(nv, attr, 0) if nv is not None else 0
                if bit and rs & bit:
                    reasons.add(name)
        return {"sm_mhz": statistics.median([s[1] for s in inside]) if inside else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(reasons), "samples": len(inside),
                "source": "NVML, every ~0.5 ms during the timed region"}


def _cpu_port_time(w, depth, steps: int, threads: int):
    """Time the C restatement of the reference step on the host: (s/step, cells).

    Each step is the reference loop's CFL reduction plus the step
    (``numpy_solver/shallow_water_2d.py:402-412``)."""
    from oracle import cport
    from oracle import swe_numpy as O

    p = O.make_params(w.bed, w.manning_n, w.domain_mask, **w.solver_kwargs())
    d = cport.Domain(p)
    cport.set_threads(threads)
    st = O.initial_state(p, depth_m=depth)
    t = 0.0
    dt = d.cfl_dt(st)
    st = d.step(st, dt, t)  # warm-up (first touch of the buffers)
    t += dt
    t0 = time.perf_counter()
    for _ in range(steps):
        dt = d.cfl_dt(st)
        st = d.step(st, dt, t)
        t += dt
    el = time.perf_counter() - t0
    return el / steps, w.bed.size


def _numpy_reference_time(w, depth, steps: int) -> dict:
    """The reference NumPy solver's loop (restated bit for bit in
    ``oracle/swe_numpy.py``, pinned to the reference's own outputs): NumPy's
    elementwise operations use one core."""
    from oracle import swe_numpy as O

    p = O.make_params(w.bed, w.manning_n, w.domain_mask, **w.solver_kwargs())
    st = O.initial_state(p, depth_m=depth)
    t = 0.0
    st = O.finite_volume_step(st, p, O.compute_cfl_dt(st, p), t)  # warm-up
    t0 = time.perf_counter()
    for _ in range(steps):
        dt = O.compute_cfl_dt(st, p)
        st = O.finite_volume_step(st, p, dt, t)
        t += dt
    el = time.perf_counter() - t0
    return {"value": w.bed.size * steps / el, "unit": "cell-updates/s", "cores": 1, "steps": steps,
            "s_per_step": el / steps, "grid": list(w.shape)}


def _cpu_legs(w, depth) -> dict:
    """Host-core baselines of the same path: the C port on every host thread,
    the reference NumPy loop on one core (the 256x256 and 2048x2048 cases), and
    JAX-CPU when JAX is importable."""
    from hybrid_flood_b200.workloads import tilted_bumps
    from oracle import cport

    threads = cport.default_threads()
    per_step, cells = _cpu_port_time(w, depth, 3, threads)
    out = {"value": cells / per_step, "unit": "cell-updates/s", "cores": threads, "kind": "port",
           "sample": "3 whole-grid steps of the same workload (C restatement, every host thread)",
           "host_cores": os.cpu_count()}
    small = tilted_bumps(256, 256)
    out["numpy"] = {"config0_256x256": _numpy_reference_time(small, np.full(small.shape, 0.01, np.float32), 20),
                    "config1_2048x2048": _numpy_reference_time(w, depth, 3),
                    "kind": "reference NumPy loop (oracle/swe_numpy.py, bit-identical to the reference)"}
    try:
        import jax  # noqa: F401

        out["jax_cpu"] = "importable but not timed by this bench"
    except ImportError:
        out["jax_cpu"] = "unavailable on this box (jax is not installed)"
    return out


def _parity(args, w, depth, dev) -> dict:
    """100 CFL steps of the measured workload on the GPU against the float32 and
    float64 C restatements (relative L2 of the depth)."""
    from hybrid_flood_b200.solver import B200ShallowWaterSolver
    from oracle import cport
    from oracle import swe_numpy as O

    n = 100
    s = B200ShallowWaterSolver(w.bed, w.manning_n, w.domain_mask, **w.solver_kwargs(), arithmetic=args.arith,
                               device=dev)
    init = O.initial_state(O.make_params(w.bed, w.manning_n, w.domain_mask, **w.solver_kwargs()), depth_m=depth)
    got, t_gpu, _, _ = s.advance(list(init), n, 0.0)
    h = got.h.cpu().numpy().astype(np.float64)
    out = {"steps": n, "simulated_s": t_gpu}
    for name, dtype in (("f32", np.float32), ("f64", np.float64)):
        p = O.make_params(w.bed, w.manning_n, w.domain_mask, dtype=dtype, **w.solver_kwargs())
        d = cport.Domain(p)
        st, t = O.State(*(np.asarray(a, dtype) for a in init)), 0.0
        for _ in range(n):
            dt = d.cfl_dt(st)
            st = d.step(st, dt, t)
            t += dt
        ref = np.asarray(st.h, np.float64)
        out[f"rel_l2_vs_{name}"] = float(np.linalg.norm(h - ref) / np.linalg.norm(ref))
        if name == "f64":
            out["f32_oracle_vs_f64"] = float(np.linalg.norm(np.asarray(f32_h, np.float64) - ref) / np.linalg.norm(ref))
        else:
            f32_h = st.h
    out["bar"] = "rel L2 depth <= 1e-5 after 100 steps (vs the float32 restatement)"
    return out


def _device_setup(ws, arith: str, dev) -> dict:
    """Time generating the same members' fields on the device (their own seeded
    draws, hybrid_flood_b200.generators) and creating the ensemble from them."""
    import torch

    from hybrid_flood_b200.ensemble import B200Ensemble
    from hybrid_flood_b200.generators import member_fields, urban_device

    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    mems = [member_fields(urban_device(w.shape[0], w.shape[1], seed=int(w.meta["seed"]),
                                       rain_scale=float(w.meta["rain_scale"]), n_scale=float(w.meta["n_scale"]),
                                       device=dev)) for w in ws]
    torch.cuda.synchronize(dev)
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    ens = B200Ensemble(mems, arithmetic=arith, device=dev)
    torch.cuda.synchronize(dev)
    create_s = time.perf_counter() - t0
    del ens, mems
    return {"device_generate_s": gen_s, "device_fields_ensemble_create_s": create_s,
            "members": len(ws), "cells": int(sum(w.bed.size for w in ws))}


def _ensemble(args, dev, rank: int, world: int):
    """Batched 64-member ensemble vs the same members run one by one (plain path).

    Both are timed the same way: the members' states are loaded first, and the
    CUDA events bracket only the step launches (the ensemble's 50-step graphs;
    the plain solvers' resident steps, member after member, on one stream).
    With N ranks the members are partitioned across GPUs (cell-balanced bin
    pack, no per-step collective): the value is all members' cell-updates over
    the slowest rank's time (strong scaling of a fixed ensemble)."""
    import torch

    from hybrid_flood_b200.ensemble import B200Ensemble
    from hybrid_flood_b200.sharding import max_over_ranks, shard_members
    from hybrid_flood_b200.solver import B200ShallowWaterSolver, ledger_error
    from hybrid_flood_b200.workloads import as_member, ensemble_members, street_depth

    t0 = time.perf_counter()
    ws_all = ensemble_members(args.ensemble_members)
    host_gen_s = time.perf_counter() - t0
    cells_all = [w.shape[0] * w.shape[1] for w in ws_all]
    mine = shard_members(cells_all, world)[rank]
    ws = [ws_all[i] for i in mine]
    members = [as_member(w) for w in ws]
    depths = [street_depth(w) for w in ws]
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    ens = B200Ensemble(members, arithmetic=args.arith, device=dev)
    torch.cuda.synchronize(dev)
    host_create_s = time.perf_counter() - t0
    setup = _device_setup(ws, args.arith, dev)
    setup.update({"host_numpy_generate_s": host_gen_s, "host_fields_ensemble_create_s": host_create_s})
    states = ens.initial_states(depths)
    ens.advance_(states, 50)  # spin-up
    tune_states = [type(s)(*(t.clone() for t in s)) for s in states]
    best = ens.autotune(tune_states, candidates=(48, 64, 96, 128, 160, 192, 256, 320), steps=50, cache=None)
    del tune_states
    ens.advance_(states, 50)  # warm-up (graph capture)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    ens.set_timing(True)
    res = ens.advance_(states, args.ensemble_steps)
    ms, n = ens.last_step_time()
    ms = max_over_ranks(ms)
    cells = sum(cells_all)
    value = cells * n / (ms / 1e3)
    errs = [ledger_error(r[2]) for r in res]
    worst_ledger = max_over_ranks(max(errs))
    worst_member = {"index": int(mine[int(np.argmax(errs))]), "steps": int(res[int(np.argmax(errs))][1]),
                    "shape": list(ws[int(np.argmax(errs))].shape)}
    # Plain path, member after member, same steps (each member its own solver, resident state).
    solvers = [B200ShallowWaterSolver(m["bed"], m["manning_n"], m["domain_mask"],
                                      **{k: v for k, v in m.items() if k not in ("bed", "manning_n", "domain_mask")},
                                      arithmetic=args.arith, device=dev) for m in members]
    for s, d in zip(solvers, depths):
        s.resident_load(s.initial_state(depth_m=d))
        s.resident_steps(100)  # spin-up and warm-up
        s.resident_prepare(args.ensemble_steps)  # the timed steps' graphs, captured now
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for s in solvers:
        s.resident_steps(args.ensemble_steps)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    plain_ms = max_over_ranks(e0.elapsed_time(e1))
    plain_value = cells * args.ensemble_steps / (plain_ms / 1e3)
    peak, kind = _peaks()
    return {
        "value": value, "unit": "cell-updates/s", "members": len(ws_all), "cells": cells,
        "members_per_rank_max": int(max_over_ranks(len(mine))), "scaling": "strong" if world > 1 else "n/a",
        "steps": n, "ms_per_step": ms / n, "rows_per_warp": best,
        "roofline_frac": BYTES_PER_CELL * value / world / 1e9 / peak, "peak_kind": kind,
        "plain_sequential_value": plain_value, "speedup_vs_plain_sequential": value / plain_value,
        "timing": "both arms: CUDA events around the step launches only (states loaded beforehand)",
        "ledger_rel_error_max": worst_ledger, "ledger_worst_member": worst_member,
        "gpu_launches": ens.last_launch_count(), "setup": setup,
        "workload": f"{len(ws_all)} urban members from {{256^2, 512^2, 1024^2, 768x1536}}, dx=1m, "
                    "rain x LogNormal(0.4), n x U(0.8,1.2), seeds 1000+m",
    }


def _adjoint(args, dev):
    """Forward vs forward+adjoint time of the differentiable gauge rollout
    (512x512, dx = 2 m, 2000 fixed-dt steps, gauges every 10 steps, checkpoint every 50)."""
    import torch

    from hybrid_flood_b200.adjoint import gauge_rollout
    from hybrid_flood_b200.solver import B200ShallowWaterSolver
    from hybrid_flood_b200.workloads import adjoint_case

    w, n_truth, n_est, gauges = adjoint_case(512, 512)
    solver = B200ShallowWaterSolver(w.bed, n_est, w.domain_mask, **w.solver_kwargs(), arithmetic="exact",
                                    device=dev)
    depth = np.maximum(1.0 - w.bed, 0.2).astype(np.float32)
    h0 = torch.tensor(depth, device=dev)
    steps, dt = args.adjoint_steps, 0.2
    kw = dict(n_steps=steps, dt=dt, gauge_index=gauges, obs_every=10, checkpoint_every=50)
    with torch.no_grad():
        obs = gauge_rollout(solver, torch.tensor(n_truth, device=dev), h0, 1.0, **kw)
    n_t = torch.tensor(n_est, device=dev, requires_grad=True)
    h_t = h0.clone().requires_grad_(True)
    s_t = torch.tensor(1.0, device=dev, requires_grad=True)
    stream = torch.cuda.current_stream(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    with torch.no_grad():
        gauge_rollout(solver, n_t, h_t, s_t, **kw)  # warm-up of the forward
    warm = gauge_rollout(solver, n_t, h_t, s_t, **kw)  # and of the backward (scratch, plans)
    torch.mean((warm - obs) ** 2).backward()
    n_t.grad = h_t.grad = s_t.grad = None
    torch.cuda.synchronize(dev)
    ev[0].record(stream)
    with torch.no_grad():
        gauge_rollout(solver, n_t, h_t, s_t, **kw)
    ev[1].record(stream)
    ev[2].record(stream)
    pred = gauge_rollout(solver, n_t, h_t, s_t, **kw)
    loss = torch.mean((pred - obs) ** 2)
    loss.backward()
    ev[3].record(stream)
    torch.cuda.synchronize(dev)
    f_ms = ev[0].elapsed_time(ev[1])
    fb_ms = ev[2].elapsed_time(ev[3])
    return {"workload": "512x512 dx=2m tilted plane + bumps, log-normal n (median 0.03, sigma_log 0.3, "
                        f"9-cell smoothing), 16 gauges every 10 steps, {steps} fixed-dt steps, checkpoint/50",
            "steps": steps, "forward_ms": f_ms, "forward_adjoint_ms": fb_ms, "ratio": fb_ms / f_ms,
            "loss": float(loss.detach()), "grad_n_norm": float(n_t.grad.norm()), "grad_rain_scale": float(s_t.grad)}


def _aux(args, dev):
    """Device time and achieved bandwidth of the kernels around the step, each on an
    aux_size x aux_size urban field (default 4096^2, inputs larger than the L2): the
    run-start CFL/volume reduction, the allocation-free CFL reduction, the output
    schema fields, the network features (5 channels, bf16), the volume-preserving
    correction, the smoothed log-normal field and the urban DEM generator.  Each is
    timed with CUDA events around `reps` back-to-back calls through the public API;
    bytes are the kernels' algorithmic traffic per cell (reads + writes)."""
    import ctypes

    import torch

    from hybrid_flood_b200 import _lib
    from hybrid_flood_b200.generators import lognormal_field_device, member_fields, street_depth_device, urban_device
    from hybrid_flood_b200.hybrid import HybridInputs, apply_residual_correction, network_features
    from hybrid_flood_b200.output import output_fields
    from hybrid_flood_b200.solver import B200ShallowWaterSolver

    n = args.aux_size
    cells = n * n
    peak, kind = _peaks()
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps

    out = {}

    def entry(name, ms, bytes_per_cell, note):
        gbs = bytes_per_cell * cells / (ms / 1e3) / 1e9
        out[name] = {"ms": ms, "bytes_per_cell": bytes_per_cell, "achieved_gbs": gbs, "frac": gbs / peak,
                     "note": note}

    member = urban_device(n, n, device=dev)
    ms = timed(lambda: urban_device(n, n, device=dev), 3)
    entry("urban_dem", ms, 9, "rectangle draws, first cover per cell, bed + Manning n + block mask written "
                              "(9 B/cell); includes the hyetograph's copy to the host")
    ms = timed(lambda: lognormal_field_device((n, n), median=0.03, sigma_log=0.4, seed=5, device=dev), 5)
    entry("lognormal_field", ms, 44, "normal draws (8 B), two smoothing passes (2 x 16 B), moments and the "
                                     "log-normal map (12 B), float64 intermediates")
    solver = B200ShallowWaterSolver(**member_fields(member), arithmetic=args.arith, device=dev)
    state = solver.initial_state(depth_m=street_depth_device(member))
    solver.advance_(state, 20, 0.0)
    ms = timed(lambda: solver.max_inverse_dt(state), 10)
    entry("reduce_kernel", ms, 16, "run-start CFL maximum and volume: h, hu, hv and n^2 read; "
                                   "the call returns the value to the host")
    lib = _lib.load()
    mask = torch.ones((n, n), dtype=torch.uint8, device=dev)
    res = torch.empty(1, dtype=torch.float32, device=dev)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    sp = ctypes.c_void_p(stream.cuda_stream)

    def noalloc():
        _lib.check(lib.swe_max_inverse_dt_noalloc(ptr(state.h), ptr(state.hu), ptr(state.hv), n, ptr(mask), n, n,
                                                   9.81, 1.0e-3, 1.0, 1.0, ptr(res), sp), "noalloc")

    if cells <= 16_777_216:
        entry("max_inverse_dt_noalloc_kernel", timed(noalloc, 10), 13, "h, hu, hv and the mask byte read")
    fields = torch.empty((4, n, n), dtype=torch.float32, device=dev)
    entry("schema_kernel", timed(lambda: output_fields(solver, state, fields), 10), 32,
          "h, hu, hv and n^2 (mask) read (16 B), depth, u, v, speed written (16 B)")
    hi = HybridInputs(None, None, np.zeros(5, np.float32), np.ones(5, np.float32), 1.0, np.ones(3, np.float32))
    feats = torch.empty((1, n, n, 5), dtype=torch.bfloat16, device=dev)
    entry("features_kernel", timed(lambda: network_features(solver, state, hi, 600.0, layout="state5",
                                                            dtype=torch.bfloat16, out=feats), 10), 30,
          "h, hu, hv, n^2 (mask) and bed read (20 B), 5 bf16 channels written (10 B)")
    resid = torch.zeros((n, n, 3), dtype=torch.bfloat16, device=dev)
    corr = type(state)(*(torch.empty_like(t) for t in state))
    entry("correction", timed(lambda: apply_residual_correction(solver, state, resid, correction_relaxation=0.5,
                                                                out=corr), 10), 56,
          "sums pass: n^2, h and the bf16 residual's sectors read, provisional depth written (18 B); "
          "apply pass: n^2, h, hu, hv, provisional depth and the residual read, new state written (38 B)")
    return {"size": [n, n], "peak_gbs": peak, "peak_kind": kind, "kernels": out,
            "timing": "CUDA events around back-to-back calls of the public API (host work between calls included)"}


def _hybrid(args, dev):
    """Coupled physics + corrector rollout: 16 urban 1024x1024 members, the
    4-level (32/64/128/256) bfloat16 channels_last corrector on (h, hu, hv, z,
    rain), a depth correction every 60 s at relaxation 0.5, 10 intervals."""
    import torch

    from hybrid_flood_b200.ensemble import B200Ensemble
    from hybrid_flood_b200.hybrid import HybridInputs, run_coupled_ensemble
    from hybrid_flood_b200.unet import corrector_4level
    from hybrid_flood_b200.workloads import as_member, street_depth, urban

    torch.backends.cudnn.benchmark = True
    M, S = args.hybrid_members, args.hybrid_size
    ws = [urban(S, S, seed=2000 + m, rain_scale=float(np.exp(0.4 * np.random.default_rng(m).normal())))
          for m in range(M)]
    ens = B200Ensemble([as_member(w) for w in ws], arithmetic=args.arith, device=dev)
    depths = [street_depth(w) for w in ws]
    states = [tuple(t.cpu().numpy() for t in s) for s in ens.initial_states(depths)]
    z = np.stack([w.bed for w in ws])
    h0 = np.stack([s[0] for s in states])
    hi = HybridInputs(None, None,
                      np.array([h0.mean(), 0.0, 0.0, z.mean(), 5.0], np.float32),
                      np.array([max(h0.std(), 1e-3), 0.05, 0.05, max(z.std(), 1e-3), 5.0], np.float32),
                      25.0, np.array([0.01], np.float32))
    torch.manual_seed(0)
    net = corrector_4level()
    with torch.no_grad():
        net.residual_head.weight.normal_(0.0, 0.01)
    net = net.to(device=dev, dtype=torch.bfloat16, memory_format=torch.channels_last).eval()
    kw = dict(max_substeps_per_interval=5000, correction_relaxation=0.5, feature_layout="state5", keep_states=False)
    # the initial states resident on the device before the timed region, like every input of the bench
    states = [tuple(torch.as_tensor(a, device=dev) for a in s) for s in states]
    run_coupled_ensemble(ens, states, net, hi, np.array([0.0, 60.0]), **kw)  # warm-up: graphs, cuDNN plans
    times = 60.0 * np.arange(args.hybrid_intervals + 1)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    tm: dict = {}
    ens.set_timing(True)
    e0.record(stream)
    traj, steps = run_coupled_ensemble(ens, states, net, hi, times, **kw, timings=tm)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    total_ms = e0.elapsed_time(e1)
    # the corrector alone on the same batch, for the time split
    feats = torch.zeros((M, S, S, 5), dtype=torch.bfloat16, device=dev).permute(0, 3, 1, 2)
    with torch.no_grad():
        net(feats)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(3):
            net(feats)
        e1.record(stream)
    torch.cuda.synchronize(dev)
    net_ms = e0.elapsed_time(e1) / 3
    # FLOPs of one corrector forward (convolutions and transposed convolutions, 2 per MAC)
    from torch.utils.flop_counter import FlopCounterMode

    from hybrid_flood_b200 import unet as unet_mod

    fused_on = unet_mod._FUSED["on"]
    unet_mod._FUSED["on"] = False  # the counter sees torch convolutions, not cuDNN's fused calls (same math)
    with torch.no_grad(), FlopCounterMode(display=False) as fc:
        net(feats)
    unet_mod._FUSED["on"] = fused_on
    net_flops = float(fc.get_total_flops())
    tf_peak, tf_kind = _tensor_peak()
    cells = M * S * S
    phys_updates = float(S * S * steps.sum())
    finite = all(bool(torch.isfinite(t).all()) for tr in traj for t in tr)
    return {"workload": f"{M} urban {S}x{S} members dx=1m, correction every 60 s, relaxation 0.5, "
                        f"{args.hybrid_intervals} intervals, 4-level bf16 channels_last corrector (5 in, 1 out)",
            "members": M, "cells": cells, "intervals": args.hybrid_intervals, "total_ms": total_ms,
            "ms_per_interval": total_ms / args.hybrid_intervals, "physics_steps_mean": float(steps.mean()),
            "physics_steps_max": int(steps.max()), "corrector_ms_per_interval": net_ms,
            "corrector_share": net_ms * args.hybrid_intervals / total_ms,
            "corrector_tflop_per_forward": net_flops / 1e12,
            "corrector_tflops": net_flops / (net_ms / 1e3) / 1e12,
            "corrector_frac_of_bf16_peak": net_flops / (net_ms / 1e3) / 1e12 / tf_peak,
            "bf16_peak_tflops": tf_peak, "bf16_peak_kind": tf_kind,
            "physics_ms_per_interval": tm.get("physics_ms", 0.0) / args.hybrid_intervals,
            "physics_cell_updates_per_s": phys_updates / (tm["physics_ms"] / 1e3) if tm.get("physics_ms") else None,
            "cell_updates_per_s": phys_updates / (total_ms / 1e3), "finite": finite}


def _training(args, dev):
    """One optimiser step of the corrector trained THROUGH the solver: 16 urban
    1024x1024 members, 10 correction intervals of 60 s, targets from 2x refined
    (2048x2048, dx = 0.5 m) runs block-averaged back; bf16 4-level corrector."""
    import torch

    from hybrid_flood_b200.ensemble import B200Ensemble
    from hybrid_flood_b200.hybrid import HybridInputs
    from hybrid_flood_b200.training import refined_targets, train_step
    from hybrid_flood_b200.unet import corrector_4level
    from hybrid_flood_b200.workloads import as_member, street_depth, urban

    torch.backends.cudnn.benchmark = True
    M, S, K = args.training_members, args.training_size, args.hybrid_intervals
    times = 60.0 * np.arange(K + 1)
    ws = [urban(S, S, seed=3000 + m) for m in range(M)]
    members = [as_member(w) for w in ws]
    depths = [street_depth(w) for w in ws]
    stream = torch.cuda.current_stream(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize(dev)
    ev[0].record(stream)
    targets = [refined_targets(mem, d0, times, device=dev) for mem, d0 in zip(members, depths)]
    ev[1].record(stream)
    ens = B200Ensemble(members, arithmetic=args.arith, device=dev)
    states = [tuple(torch.as_tensor(a, device=dev) for a in (d, np.zeros_like(d), np.zeros_like(d))) for d in depths]
    z = np.stack([w.bed for w in ws])
    h0 = np.stack(depths)
    hi = HybridInputs(None, None, np.array([h0.mean(), 0.0, 0.0, z.mean(), 5.0], np.float32),
                      np.array([max(h0.std(), 1e-3), 0.05, 0.05, max(z.std(), 1e-3), 5.0], np.float32),
                      25.0, np.array([0.01], np.float32))
    torch.manual_seed(0)
    net = corrector_4level().to(device=dev, dtype=torch.bfloat16, memory_format=torch.channels_last)
    opt = torch.optim.Adam(net.parameters(), lr=1e-4)
    kw = dict(max_substeps_per_interval=5000, correction_relaxation=0.5, feature_layout="state5")
    loss0, _ = train_step(ens, states, net, opt, hi, times, targets, **kw)  # warm-up: graphs, cuDNN plans
    torch.cuda.synchronize(dev)
    ev[2].record(stream)
    loss1, steps = train_step(ens, states, net, opt, hi, times, targets, **kw)
    ev[3].record(stream)
    torch.cuda.synchronize(dev)
    step_ms = ev[2].elapsed_time(ev[3])
    return {"workload": f"{M} urban {S}x{S} members dx=1m, {K} intervals of 60 s, targets from 2x refined runs, "
                        "bf16 4-level corrector, relaxation 0.5, Adam",
            "members": M, "intervals": K, "train_step_ms": step_ms, "target_runs_ms": ev[0].elapsed_time(ev[1]),
            "physics_steps_mean": float(steps.float().mean()), "loss_first": loss0, "loss_second": loss1,
            "peak_mem_gb": torch.cuda.max_memory_allocated(dev) / 1e9}


def _decomposed(args, dev, rank: int, world: int):
    """The same 2048x2048 domain split into one row strip per rank (halo rows,
    domain-wide dt, NCCL exchange): all ranks' cell-updates over the slowest rank's
    time (strong scaling of a fixed domain)."""
    import torch

    from hybrid_flood_b200.decomposition import NcclStrip
    from hybrid_flood_b200.sharding import max_over_ranks
    from hybrid_flood_b200.workloads import as_member

    w, depth = _workload(args.rows, args.cols)
    strip = NcclStrip(as_member(w), rank=rank, world=world, arithmetic=args.arith, device=dev)
    z = np.zeros_like(depth)
    local = strip.local_state([torch.tensor(a, device=dev) for a in (depth, z, z)])
    t, _, _ = strip.advance_(local, args.spinup + args.warmup, 0.0)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    strip.advance_(local, args.steps, t)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = max_over_ranks(e0.elapsed_time(e1))
    return {"value": w.bed.size * args.steps / (ms / 1e3), "unit": "cell-updates/s", "scaling": "strong",
            "strips": world, "ms_per_step": ms / args.steps,
            "workload": f"urban {args.rows}x{args.cols} split into {world} row strips (NCCL halo exchange)"}


def run_reference(args, rank: int, world: int):
    """The CPU implementation of the same path on the host cores: the C
    restatement of the reference step on every host thread, whole-grid steps of
    the same workload (``min(K, 200)`` timed, after ``min(W, 3)`` warm-up)."""
    if rank != 0:
        return
    from oracle import cport

    w, depth = _workload(args.rows, args.cols)
    threads = cport.default_threads()
    k = max(1, min(args.steps, REFERENCE_MAX_STEPS))
    per_step, cells = _cpu_port_time(w, depth, k, threads)
    value = cells / per_step
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-updates/s",
        "n_gpus": args.gpus, "steps": k, "steps_requested": args.steps, "warmup": args.warmup,
        "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": _config(args, world),
        "arith": "C restatement, IEEE float32, no FMA",
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                         "sample": f"{k} whole-grid steps of the same workload"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _exact_leg(args, w, depth, dev) -> dict:
    """The same resident step timing in exact arithmetic (the mode that is bit-identical
    to the reference's float32 NumPy solver on its golden runs): W warm-up steps, then
    ``--exact-steps`` steps between CUDA events."""
    import torch

    from hybrid_flood_b200.solver import B200ShallowWaterSolver

    solver = B200ShallowWaterSolver(w.bed, w.manning_n, w.domain_mask, **w.solver_kwargs(), arithmetic="exact",
                                    device=dev)
    state = solver.initial_state(depth_m=depth)
    t_sim, _, _ = solver.advance_(state, args.spinup, 0.0)
    solver.resident_load(state, t_sim)
    solver.resident_steps(args.warmup)
    solver.resident_prepare(args.exact_steps)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    torch.cuda._sleep(200_000)
    e0.record(stream)
    solver.resident_steps(args.exact_steps)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    solver.resident_store(state)
    cells = w.bed.size
    value = cells * args.exact_steps / (ms / 1e3)
    peak, kind = _peaks()
    return {"value": value, "unit": "cell-updates/s", "steps": args.exact_steps, "ms_per_step": ms / args.exact_steps,
            "roofline_frac": BYTES_PER_CELL * value / 1e9 / peak, "peak_kind": kind,
            "arith": "exact (IEEE-rounded float32, the reference's operation order)"}


def _e2e(args, solver, state, t_sim, dev, world: int) -> dict:
    """``B200ShallowWaterSolver.run_to_host`` with host state: one forecast over the
    workload's whole hyetograph window (``--e2e-window-s``, 10,800 s) with an
    output every ``--e2e-every-s`` seconds; the state goes in from pinned host
    memory and every recorded snapshot comes back to pinned host memory inside
    the timed region."""
    import torch

    cells = solver.shape[0] * solver.shape[1]
    host = [t.cpu().numpy().copy() for t in state]
    pinned = [torch.from_numpy(a).pin_memory() for a in host]
    window = float(args.e2e_window_s)
    times = np.arange(0.0, window + 0.5 * args.e2e_every_s, args.e2e_every_s).astype(np.float32)
    n_out = len(times)
    outs_host = [torch.empty((n_out, *solver.shape), dtype=torch.float32).pin_memory() for _ in range(3)]
    stream = torch.cuda.current_stream(dev)
    # warm-up of the run path (staging for n_out snapshots, copy stream) on a short window
    solver.run_to_host(pinned, np.arange(n_out, dtype=np.float32), out=outs_host, max_steps=args.e2e_max_steps)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e0.record(stream)
    res = solver.run_to_host(pinned, times, out=outs_host, max_steps=args.e2e_max_steps)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - w0
    ms = e0.elapsed_time(e1)
    steps = res.steps_used
    plane = cells * 4
    return {"value": cells * steps * world / (ms / 1e3), "unit": "cell-updates/s",
            "h2d_bytes_per_step": int(3 * plane / max(steps, 1)),
            "d2h_bytes_per_step": int(3 * plane * n_out / max(steps, 1)),
            "call": f"B200ShallowWaterSolver.run_to_host(pinned host state, {n_out} output times every "
                    f"{args.e2e_every_s:g} s, pinned host outputs)",
            "steps_per_call": steps, "simulated_window_s": window, "wall_s": wall}


def run_b200(args, rank: int, world: int):
    import torch

    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist = dist_mod
        dist.init_process_group("nccl", device_id=dev, timeout=datetime.timedelta(seconds=300))
    from hybrid_flood_b200.solver import B200ShallowWaterSolver, ledger_error

    w, depth = _workload(args.rows, args.cols)
    solver = B200ShallowWaterSolver(w.bed, w.manning_n, w.domain_mask, **w.solver_kwargs(),
                                    arithmetic=args.arith, device=dev)
    state = solver.initial_state(depth_m=depth)
    t_sim, _, _ = solver.advance_(state, args.spinup, 0.0)
    cells = w.bed.size
    stream = torch.cuda.current_stream(dev)
    # Resident state: W untimed warm-up steps, then exactly K timed steps.
    solver.resident_load(state, t_sim)
    # The graphs of the warm-up and timed steps are captured now, outside the timed region.
    solver.resident_prepare(args.warmup)
    solver.resident_prepare(args.steps)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clocks:
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
        clocks.mark_start()
        # A ~0.1 ms sleep kernel and the W warm-up steps run ahead of the start
        # event: the host enqueues the timed steps while they run (the region
        # holds no host latency), and the GPU enters the region under load.
        torch.cuda._sleep(200_000)
        solver.resident_steps(args.warmup)
        start.record(stream)
        solver.resident_steps(args.steps)
        end.record(stream)
        clocks.sample_until(end)
        torch.cuda.synchronize(dev)
        clocks.mark_end()
    if dist:
        dist.barrier()
    ms = start.elapsed_time(end)
    launches = solver.last_launch_count()
    t_before = t_sim
    t_sim, steps_done, ledger = solver.resident_store(state)
    if dist:
        tt = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt[0])
    value = cells * args.steps * world / (ms / 1e3)
    window = t_sim - t_before

    e2e = None if args.no_e2e else _e2e(args, solver, state, t_sim, dev, world)
    exact = _exact_leg(args, w, depth, dev) if (args.arith == "fast" and args.exact_steps > 0 and rank == 0) else None
    dec = _decomposed(args, dev, rank, world) if args.decompose else None
    ens = None
    if not args.no_ensemble:
        ens = _ensemble(args, dev, rank, world)
    adj = None
    if not args.no_adjoint and rank == 0:
        adj = _adjoint(args, dev)
    hyb = None
    if not args.no_hybrid and rank == 0:
        hyb = _hybrid(args, dev)
    trn = None
    if not args.no_training and rank == 0:
        trn = _training(args, dev)
    par = None
    if not args.no_parity and rank == 0:
        par = _parity(args, w, depth, dev)
    aux = None
    if not args.no_aux and rank == 0:
        aux = _aux(args, dev)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    peak, peak_kind = _peaks()
    per_launch_ms = ms / args.steps
    achieved = BYTES_PER_CELL * cells / (per_launch_ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": _config(args, world), "arith": args.arith,
        "simulated_window_s": window,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": (NCU_TRAFFIC_PER_CELL * cells
                                 if (args.rows, args.cols, args.arith) == (2048, 2048, "fast") else None),
                     "traffic_unit": "bytes per launch (ncu capture of the same launch)",
                     "kernel": "step_kernel_pair (fused step + CFL + ledger), the only kernel of the timed region",
                     "bytes_per_cell": BYTES_PER_CELL, "peak_kind": peak_kind,
                     "kernel_ms_per_launch": per_launch_ms,
                     "duration": "timed-region CUDA events / K (back-to-back step launches, gaps included)"},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
        "ledger_rel_error": ledger_error(ledger),
    }
    if e2e:
        line["e2e"] = e2e
    if exact:
        line["exact_arithmetic"] = exact
    if par:
        line["parity"] = par
    if ens:
        line["ensemble"] = ens
    if adj:
        line["adjoint"] = adj
    if hyb:
        line["hybrid"] = hyb
    if dec:
        line["decomposed"] = dec
    if trn:
        line["training"] = trn
    if aux:
        line["aux_kernels"] = aux
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = _cpu_legs(w, depth)
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def main():
    args = _args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.steps < 1 or args.warmup < 0:
        raise SystemExit("--steps must be >= 1 and --warmup >= 0")
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_b200(args, rank, world)


if __name__ == "__main__":
    main()
