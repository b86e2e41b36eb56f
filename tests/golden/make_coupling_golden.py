"""Generate ``coupling_ref6.npz`` from the reference's own coupling code.

Run where the reference project is mounted (nothing else reads it):

    python tests/golden/make_coupling_golden.py --reference /root/reference

The reference couples physics and corrector in JAX
(``src/hybrid_flood/hybrid/coupled_forecast.py``), and jax is not installed in
this image.  This script imports that module UNMODIFIED, together with the JAX
solver it calls (``jax_solver/numerics.py``, ``boundary_conditions.py``), after
putting a small NumPy stand-in for ``jax`` into ``sys.modules``:

* ``jax.numpy`` is NumPy (float32 arrays in, float32 out, as JAX's default
  32-bit mode keeps them; ``interp`` is rounded back to the table's dtype);
* ``jax.jit`` is the identity; ``jax.lax.scan``, ``cond`` and ``while_loop`` are
  Python loops; ``jax.tree.map`` maps over NamedTuple fields;
* ``array.at[idx].set(v)`` / ``.add(v)`` return updated copies.

What the fixture pins is therefore the reference's coupling logic and operation
order under NumPy's float32 arithmetic: the features, the residual clip, the
volume-preserving correction and the outer loop of ``run_coupled_forecast``
(features of the pre-advance state, physics to the next time, residual,
clip, correction).  Two known differences from real JAX stay: float32 sums are
NumPy's pairwise sums (XLA may sum in another order), and the forecast clock is
float32, as JAX's default mode has it (the float64 NumPy run loop is what the
rest of the parity suite follows).

Cases (``coupling_ref6.npz``):

* ``features_*``: ``network_features`` of a 20x28 masked wet/dry state at a
  rain-table breakpoint and past the table (default rain);
* ``corrected_*``: ``apply_residual_correction`` of the same state with a
  three-channel residual clipped at ``clip_sigma * residual_std``
  (``coupled_forecast.py:199-200``);
* ``forecast_*``: ``run_coupled_forecast`` on a 24x32 masked urban-like grid
  with an open east edge, output times 0/20/40/60 s, relaxation 0.5, clip
  sigma 2, and a linear corrector ``residual = features @ W + b`` (W, b saved)
  standing in for the network.
"""

from __future__ import annotations

import argparse
import pathlib
import sys
import types

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent


class _Arr(np.ndarray):
    """ndarray with JAX's functional ``.at[idx].set/add``."""

    @property
    def at(self):
        arr = self

        class _Index:
            def __getitem__(self, idx):
                class _Update:
                    def set(self, v):
                        out = np.array(arr, copy=True).view(_Arr)
                        out[idx] = v
                        return out

                    def add(self, v):
                        out = np.array(arr, copy=True).view(_Arr)
                        out[idx] += v
                        return out

                return _Update()

        return _Index()


def _wrap(x):
    if isinstance(x, np.ndarray) and not isinstance(x, _Arr):
        return x.view(_Arr)
    if isinstance(x, tuple) and not hasattr(x, "_fields"):
        return tuple(_wrap(v) for v in x)
    return x


def _install_numpy_jax() -> None:
    jnp = types.ModuleType("jax.numpy")
    jnp.ndarray = np.ndarray

    def numpy_attr(name):
        f = getattr(np, name)
        if not callable(f) or isinstance(f, type):
            return f
        return lambda *a, **k: _wrap(f(*a, **k))

    jnp.__getattr__ = numpy_attr

    def interp(x, xp, fp, left=None, right=None):
        return _wrap(np.asarray(np.interp(x, xp, fp, left=left, right=right), dtype=np.asarray(fp).dtype))

    jnp.interp = interp

    def scan(f, init, xs=None, length=None):
        carry, ys = init, []
        n = length if xs is None else len(xs)
        for i in range(n):
            carry, y = f(carry, None if xs is None else xs[i])
            ys.append(y)
        if not ys or ys[0] is None:
            return carry, None
        if isinstance(ys[0], tuple):
            return carry, type(ys[0])(*(_wrap(np.stack(c)) for c in zip(*ys)))
        return carry, _wrap(np.stack(ys))

    def while_loop(cond, body, init):
        v = init
        while bool(cond(v)):
            v = body(v)
        return v

    lax = types.ModuleType("jax.lax")
    lax.scan = scan
    lax.while_loop = while_loop
    lax.cond = lambda pred, t, f, *ops: t(*ops) if bool(pred) else f(*ops)

    def tree_map(f, tree):
        if isinstance(tree, tuple) and hasattr(tree, "_fields"):
            return type(tree)(*(f(v) for v in tree))
        return f(tree)

    jax = types.ModuleType("jax")
    jax.numpy = jnp
    jax.lax = lax
    jax.tree = types.SimpleNamespace(map=tree_map)
    jax.Array = np.ndarray
    jax.jit = lambda fn=None, **kw: fn if fn is not None else (lambda g: g)
    sys.modules.update({"jax": jax, "jax.numpy": jnp, "jax.lax": lax})


def _f32(a):
    return np.asarray(a, dtype=np.float32).view(_Arr)


def _params(N, bed, manning, mask, *, dx, rain_t, rain_r, default_rain, boundary):
    return N.SWEParams(
        bed=_f32(bed), manning_n=_f32(manning), domain_mask=np.asarray(mask, bool).view(_Arr),
        rainfall_multiplier=_f32(np.ones_like(bed)), boundary_types=np.asarray(boundary, np.int32).view(_Arr),
        rainfall_times_s=_f32(rain_t), rainfall_rates_m_s=_f32(rain_r), default_rainfall_m_s=_f32(default_rain),
        dx=_f32(dx), dy=_f32(dx), gravity=_f32(9.81), cfl=_f32(0.45), dry_tolerance=_f32(1.0e-4),
        max_dt=_f32(10.0))


def _state(rng, mask, depth=0.3):
    h = np.where(rng.uniform(size=mask.shape) > 0.25, rng.uniform(0.0, depth, mask.shape), 0.0)
    h = np.where(mask, h, 0.0).astype(np.float32)
    hu = np.where(h > 1e-3, rng.normal(0, 0.02, mask.shape), 0.0).astype(np.float32)
    hv = np.where(h > 1e-3, rng.normal(0, 0.02, mask.shape), 0.0).astype(np.float32)
    return h, hu, hv


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=pathlib.Path, default=pathlib.Path("/root/reference"))
    args = ap.parse_args()
    _install_numpy_jax()
    sys.path.insert(0, str(args.reference / "src"))
    from hybrid_flood.hybrid import coupled_forecast as CF  # noqa: PLC0415
    from hybrid_flood.jax_solver import numerics as N  # noqa: PLC0415

    out = {}
    # features and correction on one masked wet/dry state ------------------------
    rng = np.random.default_rng(11)
    H, W = 20, 28
    mask = np.ones((H, W), bool)
    mask[4:9, 10:15] = False
    mask[15:, :3] = False
    bed = rng.uniform(0.0, 0.5, (H, W)).astype(np.float32)
    manning = rng.uniform(0.02, 0.05, (H, W)).astype(np.float32)
    rain_t, rain_r, default_rain = [0.0, 30.0, 90.0], [1.0e-5, 3.0e-5, 2.0e-5], 5.0e-6
    p = _params(N, bed, manning, mask, dx=2.0, rain_t=rain_t, rain_r=rain_r, default_rain=default_rain,
                boundary=[0, 1, 0, 0])
    h, hu, hv = _state(rng, mask)
    hi = CF.HybridInputs(_f32(rng.normal(0, 1, (H, W))), _f32(rng.normal(0, 1, (H, W))),
                         _f32([0.1, 0.01, -0.02]), _f32([0.2, 0.3, 0.4]), _f32(25.0), _f32([0.01, 0.02, 0.03]))
    st = N.SWEState(_f32(h), _f32(hu), _f32(hv))
    for tag, t in (("break", 30.0), ("past", 150.0)):
        out[f"features_{tag}"] = np.asarray(CF.network_features(st, p, hi, np.float32(t)))
        out[f"features_{tag}_time"] = np.float32(t)
    residual = _f32(rng.normal(0, 0.05, (H, W, 3)))
    clip_sigma, relax = np.float32(2.0), np.float32(0.7)
    limits = clip_sigma * hi.residual_std
    clipped = np.clip(residual, -limits, limits)  # coupled_forecast.py:199-200
    corr = CF.apply_residual_correction(st, _wrap(clipped), p, correction_relaxation=relax)
    out.update(corrected_h=np.asarray(corr.h), corrected_hu=np.asarray(corr.hu), corrected_hv=np.asarray(corr.hv))
    out.update(bed=bed, manning_n=manning, domain_mask=mask, rain_times=np.float32(rain_t),
               rain_rates=np.float32(rain_r), default_rain=np.float32(default_rain), boundary=np.int32([0, 1, 0, 0]),
               dx=np.float32(2.0), state=np.stack([h, hu, hv]), terrain_std=np.asarray(hi.terrain_standardized),
               roughness_std=np.asarray(hi.roughness_standardized), state_mean=np.asarray(hi.state_mean),
               state_std=np.asarray(hi.state_std), rain_scale=np.float32(25.0),
               residual_std=np.asarray(hi.residual_std), residual=np.asarray(residual), clip_sigma=clip_sigma,
               relaxation=relax)

    # the coupled forecast loop ------------------------------------------------
    rng = np.random.default_rng(12)
    H, W = 24, 32
    fmask = np.ones((H, W), bool)
    fmask[6:10, 8:14] = False
    fmask[16:20, 20:27] = False
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float32)
    fbed = (0.02 * (W - xx) + 0.01 * yy + np.where(fmask, 0.0, 3.0)).astype(np.float32)
    fman = np.full((H, W), 0.03, np.float32)
    fp = _params(N, fbed, fman, fmask, dx=2.0, rain_t=[0.0, 1000.0], rain_r=[2.0e-5, 2.0e-5], default_rain=0.0,
                 boundary=[0, 1, 0, 0])
    fh, fhu, fhv = _state(rng, fmask, depth=0.2)
    fhi = CF.HybridInputs(_f32(rng.normal(0, 1, (H, W))), _f32(rng.normal(0, 1, (H, W))),
                          _f32([0.05, 0.0, 0.0]), _f32([0.1, 0.2, 0.2]), _f32(25.0), _f32([0.005, 0.01, 0.01]))
    Wm = (0.02 * rng.normal(size=(6, 3))).astype(np.float32)
    bm = (0.01 * rng.normal(size=3)).astype(np.float32)

    def apply_fn(variables, features):
        v = variables["params"]
        return _wrap((np.asarray(features) @ v["W"] + v["b"]).astype(np.float32))

    times = _f32([0.0, 20.0, 40.0, 60.0])
    res = CF.run_coupled_forecast(N.SWEState(_f32(fh), _f32(fhu), _f32(fhv)), fp, {"W": Wm, "b": bm}, apply_fn,
                                  fhi, times, max_substeps_per_interval=400, correction_relaxation=0.5,
                                  correction_clip_sigma=2.0)
    out.update(forecast_bed=fbed, forecast_manning_n=fman, forecast_mask=fmask, forecast_state=np.stack([fh, fhu, fhv]),
               forecast_terrain_std=np.asarray(fhi.terrain_standardized),
               forecast_roughness_std=np.asarray(fhi.roughness_standardized),
               forecast_state_mean=np.asarray(fhi.state_mean), forecast_state_std=np.asarray(fhi.state_std),
               forecast_residual_std=np.asarray(fhi.residual_std), forecast_W=Wm, forecast_b=bm,
               forecast_times=np.asarray(times), forecast_h=np.asarray(res.states.h),
               forecast_hu=np.asarray(res.states.hu), forecast_hv=np.asarray(res.states.hv),
               forecast_steps=np.int64(res.physics_steps_used))
    path = HERE / "coupling_ref6.npz"
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in out.items()})
    print(f"wrote {path.name}: {path.stat().st_size / 1024:.1f} KiB, forecast steps {int(res.physics_steps_used)}")


if __name__ == "__main__":
    with np.errstate(divide="ignore", invalid="ignore"):
        main()
