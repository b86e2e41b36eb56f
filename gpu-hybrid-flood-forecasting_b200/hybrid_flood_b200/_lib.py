"""ctypes binding of ``libswe_b200.so`` (the C ABI in ``include/swe_b200.h``).

This is the only place Python touches the native library.  It loads the
in-tree build and raises if it is missing: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import pathlib

from . import build as _build

SWE_OK = 0
SWE_ERR_INVALID = 1
SWE_ERR_CUDA = 2
SWE_ERR_MAX_STEPS = 3
SWE_ERR_NONFINITE = 4
SWE_ERR_NO_DEVICE = 5

SWE_ARITH_EXACT = 0
SWE_ARITH_FAST = 1

SWE_NOALLOC_MAX_CELLS = 16_777_216
SWE_COMM_ID_BYTES = 128

#: Every entry point ``include/swe_b200.h`` declares.
EXPORTS = (
    "swe_domain_create",
    "swe_domain_destroy",
    "swe_step",
    "swe_max_inverse_dt",
    "swe_cfl_dt",
    "swe_rainfall_rate",
    "swe_run",
    "swe_run_host",
    "swe_advance",
    "swe_last_launch_count",
    "swe_resident_load",
    "swe_resident_steps",
    "swe_resident_prepare",
    "swe_resident_store",
    "swe_set_timing",
    "swe_last_step_time",
    "swe_max_inverse_dt_noalloc",
    "swe_domain_set_rain_scale",
    "swe_domain_set_manning",
    "swe_adjoint_step",
    "swe_rollout_forward",
    "swe_rollout_backward",
    "swe_advance_to",
    "swe_network_features",
    "swe_apply_correction",
    "swe_output_fields",
    "swe_bias_act_nhwc",
    "swe_ensemble_create",
    "swe_ensemble_destroy",
    "swe_ensemble_size",
    "swe_ensemble_set_rows_per_warp",
    "swe_ensemble_rows_per_warp",
    "swe_ensemble_advance",
    "swe_ensemble_advance_to",
    "swe_ensemble_member",
    "swe_ensemble_set_timing",
    "swe_ensemble_last_step_time",
    "swe_ensemble_last_launch_count",
    "swe_ensemble_network_features",
    "swe_ensemble_apply_correction",
    "swe_strip_create",
    "swe_strip_layout",
    "swe_strips_advance",
    "swe_comm_unique_id",
    "swe_comm_create",
    "swe_comm_destroy",
    "swe_strip_advance_nccl",
    "swe_generate_urban",
    "swe_generate_gamma_hyetograph",
    "swe_generate_lognormal_field",
    "swe_last_error",
    "swe_version",
)


class DomainDesc(ctypes.Structure):
    """Mirror of ``swe_domain_desc``."""

    _fields_ = [
        ("rows", ctypes.c_int32), ("cols", ctypes.c_int32),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("gravity", ctypes.c_double), ("cfl", ctypes.c_double),
        ("dry_tolerance", ctypes.c_double), ("max_dt", ctypes.c_double),
        ("default_rainfall", ctypes.c_double),
        ("boundary", ctypes.c_int32 * 4),
        ("n_rain", ctypes.c_int32),
        ("rain_times", ctypes.c_void_p), ("rain_rates", ctypes.c_void_p),
        ("bed", ctypes.c_void_p), ("manning_n", ctypes.c_void_p),
        ("domain_mask", ctypes.c_void_p), ("rainfall_multiplier", ctypes.c_void_p),
        ("fields_on_host", ctypes.c_int32), ("arithmetic", ctypes.c_int32),
    ]


class UrbanDesc(ctypes.Structure):
    """Mirror of ``swe_urban_desc``."""

    _fields_ = [
        ("rows", ctypes.c_int32), ("cols", ctypes.c_int32),
        ("dx", ctypes.c_double), ("slope", ctypes.c_double), ("coverage", ctypes.c_double),
        ("min_side", ctypes.c_int32), ("max_side", ctypes.c_int32),
        ("block_raise_m", ctypes.c_double), ("street_offset_m", ctypes.c_double),
        ("n_block", ctypes.c_double), ("n_street", ctypes.c_double), ("n_scale", ctypes.c_double),
        ("seed", ctypes.c_uint64),
        ("n_rects", ctypes.c_int32), ("rects", ctypes.c_void_p),
    ]


class RunResult(ctypes.Structure):
    """Mirror of ``swe_run_result``."""

    _fields_ = [
        ("final_time_s", ctypes.c_double),
        ("outputs_written", ctypes.c_int32),
        ("steps_used", ctypes.c_int32),
        ("status", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("ledger", ctypes.c_double * 6),
    ]


_LIB = None
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_i32 = ctypes.c_int32
_f64 = ctypes.c_double


def library_path() -> pathlib.Path:
    return _build.LIB


def load(path: pathlib.Path | None = None) -> ctypes.CDLL:
    """Load the library (once).  Raises ``RuntimeError`` if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = pathlib.Path(path) if path else _build.LIB
    if not path.exists():
        raise RuntimeError(
            f"{path} is missing: build it with `python -m hybrid_flood_b200.build` "
            "(the CUDA path has no CPU fallback)."
        )
    lib = ctypes.CDLL(str(path))
    sig = {
        "swe_domain_create": (ctypes.c_int, [ctypes.POINTER(DomainDesc), ctypes.POINTER(_vp)]),
        "swe_domain_destroy": (ctypes.c_int, [_vp]),
        "swe_step": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _i64, _f64, _f64, _vp]),
        "swe_max_inverse_dt": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, ctypes.POINTER(ctypes.c_float), _vp]),
        "swe_cfl_dt": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, ctypes.POINTER(_f64), _vp]),
        "swe_rainfall_rate": (ctypes.c_int, [_vp, _f64, ctypes.POINTER(_f64)]),
        "swe_run": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, _vp, _i32, _i32, _vp, _vp, _vp,
                                   ctypes.POINTER(RunResult), _vp]),
        "swe_run_host": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, _vp, _i32, _i32, _vp, _vp, _vp,
                                        ctypes.POINTER(RunResult), _vp]),
        "swe_advance": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, _i32, _f64,
                                       ctypes.POINTER(RunResult), _vp]),
        "swe_last_launch_count": (ctypes.c_int64, [_vp]),
        "swe_resident_load": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, _f64, _vp]),
        "swe_resident_steps": (ctypes.c_int, [_vp, _i32, _vp]),
        "swe_resident_prepare": (ctypes.c_int, [_vp, _i32]),
        "swe_resident_store": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, ctypes.POINTER(RunResult), _vp]),
        "swe_set_timing": (ctypes.c_int, [_vp, _i32]),
        "swe_last_step_time": (ctypes.c_int, [_vp, ctypes.POINTER(_f64), ctypes.POINTER(_i64)]),
        "swe_max_inverse_dt_noalloc": (ctypes.c_int, [_vp, _vp, _vp, _i64, _vp, _i32, _i32, _f64,
                                                      _f64, _f64, _f64, _vp, _vp]),
        "swe_domain_set_rain_scale": (ctypes.c_int, [_vp, _f64]),
        "swe_domain_set_manning": (ctypes.c_int, [_vp, _vp, _i32, _vp]),
        "swe_adjoint_step": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _vp,
                                            _i64, _vp, _vp, _f64, _f64, _vp]),
        "swe_rollout_forward": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, _i32, _f64, _f64, _vp, _vp, _i32, _i32,
                                               _vp, _vp, _i32, _vp]),
        "swe_rollout_backward": (ctypes.c_int, [_vp, _vp, _i32, _i32, _f64, _f64, _vp, _vp, _i32, _i32, _vp, _vp,
                                                _vp, _vp, _i64, _i32, _vp, _vp, _vp, _vp]),
        "swe_advance_to": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, _f64, _f64, _i32, _vp,
                                          ctypes.POINTER(RunResult), _vp]),
        "swe_network_features": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, _i32, _vp, _vp, ctypes.c_float, _vp,
                                                _vp, _vp, _i32, _vp]),
        "swe_apply_correction": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, _vp, _i32, _i64, _i64, _i64, _i32,
                                                _vp, _f64, _vp, _vp, _vp, _i64, _vp]),
        "swe_output_fields": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _i64, _vp]),
        "swe_bias_act_nhwc": (ctypes.c_int, [_vp, _i64, _i32, _vp, _i32, _i32, _i32, _vp]),
        "swe_ensemble_create": (ctypes.c_int, [ctypes.POINTER(DomainDesc), _i32, ctypes.POINTER(_vp)]),
        "swe_ensemble_destroy": (ctypes.c_int, [_vp]),
        "swe_ensemble_size": (ctypes.c_int, [_vp]),
        "swe_ensemble_set_rows_per_warp": (ctypes.c_int, [_vp, _i32]),
        "swe_ensemble_rows_per_warp": (_i32, [_vp]),
        "swe_ensemble_advance": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _i32, _vp,
                                                ctypes.POINTER(RunResult), _vp]),
        "swe_ensemble_advance_to": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _f64, _i32, _vp,
                                                   ctypes.POINTER(RunResult), _vp]),
        "swe_ensemble_member": (ctypes.c_int, [_vp, _i32, ctypes.POINTER(_vp)]),
        "swe_ensemble_set_timing": (ctypes.c_int, [_vp, _i32]),
        "swe_ensemble_last_step_time": (ctypes.c_int, [_vp, ctypes.POINTER(_f64), ctypes.POINTER(_i64)]),
        "swe_ensemble_last_launch_count": (ctypes.c_int64, [_vp]),
        "swe_ensemble_network_features": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _i32, _vp, _vp, _vp, _vp, _vp,
                                                         _vp, _i64, _i32, _vp]),
        "swe_ensemble_apply_correction": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _i32, _i64, _i64, _i64,
                                                         _i64, _i32, _vp, _f64, _vp, _vp, _vp, _vp, _vp]),
        "swe_strip_create": (ctypes.c_int, [ctypes.POINTER(DomainDesc), _i32, _i32, ctypes.POINTER(_vp)]),
        "swe_strip_layout": (ctypes.c_int, [_vp, ctypes.POINTER(_i32), ctypes.POINTER(_i32), ctypes.POINTER(_i32)]),
        "swe_strips_advance": (ctypes.c_int, [_vp, _i32, _vp, _vp, _vp, _vp, _i32, _f64, ctypes.POINTER(RunResult),
                                              _vp]),
        "swe_comm_unique_id": (ctypes.c_int, [_vp]),
        "swe_comm_create": (ctypes.c_int, [_vp, _i32, _i32, ctypes.POINTER(_vp)]),
        "swe_comm_destroy": (ctypes.c_int, [_vp]),
        "swe_strip_advance_nccl": (ctypes.c_int, [_vp, _vp, _i32, _i32, _vp, _vp, _vp, _i64, _i32, _f64,
                                                  ctypes.POINTER(RunResult), _vp]),
        "swe_generate_urban": (ctypes.c_int, [ctypes.POINTER(UrbanDesc), _vp, _vp, _vp, ctypes.POINTER(_i32), _vp]),
        "swe_generate_gamma_hyetograph": (ctypes.c_int, [_i32, _f64, _f64, _f64, _f64, ctypes.c_uint64, _vp, _vp,
                                                         _vp]),
        "swe_generate_lognormal_field": (ctypes.c_int, [_i32, _i32, _f64, _f64, _i32, ctypes.c_uint64, _vp, _vp,
                                                        _vp]),
        "swe_last_error": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
        "swe_version": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def last_error() -> str:
    lib = load()
    buf = ctypes.create_string_buffer(1024)
    lib.swe_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int, what: str) -> None:
    """Map a status code to the exception the reference raises for the same failure."""
    if rc == SWE_OK:
        return
    msg = f"{what}: {last_error()}"
    if rc == SWE_ERR_INVALID:
        raise ValueError(msg)
    if rc in (SWE_ERR_MAX_STEPS, SWE_ERR_NONFINITE):
        raise RuntimeError(msg)
    raise RuntimeError(f"{msg} (status {rc})")
