"""ctypes binding of ``libhitb200.so`` (C ABI in ``include/hitb200.h``).

The shared library is the product; this module only loads it, mirrors the
descriptor struct, and maps status codes to the exceptions the reference
raises (ValueError for configuration errors, FloatingPointError for a
non-finite or non-positive state, RuntimeError for a missing backend).
There is no fallback: if the library is missing or CUDA is unavailable every
entry point raises.
"""

from __future__ import annotations

import ctypes
import math
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libhitb200.so"

OK, ERR_INVALID, ERR_CUDA, ERR_NONFINITE, ERR_NONPOSITIVE, ERR_OOM, ERR_UNSUPPORTED = range(7)

TERM_INVISCID, TERM_VISCOUS, TERM_FORCING, TERM_DRAG, TERM_COOLING = 1, 2, 4, 8, 16
TERM_ALL = 31

# scalar slots (enum hitb200_scalar)
S_ALPHA_X, S_ALPHA_Y, S_DIV_RMS, S_VORT_RMS, S_DT, S_TIME, S_STEP, S_ACTIVE, S_MACH = range(9)
(S_POWER, S_POWER_DESIRED, S_F_ALPHA, S_F_ALPHA_TARGET, S_F_POWER_BEFORE, S_F_INJECTED,
 S_F_FXX, S_F_FYY, S_F_FXY, S_F_AF, S_F_DECAY, S_F_SCALE, S_MAX_STEPS, S_STATUS,
 S_NEAR_THRESHOLD, S_HV_APPLIED) = range(9, 25)
S_COUNT = 32
# bits of the S_STATUS slot (HITB200_ST_*)
ST_NONFINITE, ST_NONPOS_RHO, ST_NONPOS_P, ST_BARRIER, ST_NOISE = 1, 2, 4, 8, 16
(TUNE_SWEEP_X, TUNE_SWEEP_Y, TUNE_PREPASS, TUNE_FUSED_SENSOR, TUNE_Y_PANEL, TUNE_PERSISTENT,
 TUNE_COUNT) = range(7)

NAN = float("nan")


class Desc(ctypes.Structure):
    """Mirror of ``hitb200_desc``."""

    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
        ("x_min", ctypes.c_double), ("x_max", ctypes.c_double),
        ("y_min", ctypes.c_double), ("y_max", ctypes.c_double),
        ("periodic", ctypes.c_int32), ("precision", ctypes.c_int32), ("scheme", ctypes.c_int32),
        ("gamma", ctypes.c_double),
        ("sensor_width", ctypes.c_int32), ("boundary_guard", ctypes.c_int32),
        ("compression_threshold", ctypes.c_double), ("jump_threshold", ctypes.c_double),
        ("shear_threshold", ctypes.c_double),
        ("viscosity", ctypes.c_double), ("prandtl", ctypes.c_double),
        ("gas_constant", ctypes.c_double),
        ("hv_mn", ctypes.c_double), ("hv_weight", ctypes.c_double * 4),
        ("hv_interval", ctypes.c_int32), ("guard_cells", ctypes.c_int32),
        ("drag_coefficient", ctypes.c_double), ("drag_kmax", ctypes.c_double),
        ("cooling_time", ctypes.c_double), ("cooling_target_pressure", ctypes.c_double),
        ("forcing_on", ctypes.c_int32),
        ("forcing_kmin", ctypes.c_double), ("forcing_kmax", ctypes.c_double),
        ("forcing_correlation_time", ctypes.c_double), ("forcing_rms", ctypes.c_double),
        ("target_power", ctypes.c_double), ("min_power", ctypes.c_double),
        ("max_rescale", ctypes.c_double), ("alpha_memory", ctypes.c_double),
        ("mach_control", ctypes.c_int32),
        ("mach_target", ctypes.c_double), ("mach_memory", ctypes.c_double),
        ("mach_exponent", ctypes.c_double), ("mach_min_power", ctypes.c_double),
        ("mach_max_power", ctypes.c_double),
        ("cfl", ctypes.c_double), ("tfinal", ctypes.c_double),
        ("fixed_dt", ctypes.c_int32), ("noise_mode", ctypes.c_int32),
        ("seed", ctypes.c_uint64),
    ]

    def key(self) -> tuple:
        out = []
        for name, _ in self._fields_:
            v = getattr(self, name)
            if name == "hv_weight":
                v = tuple(v)
            if isinstance(v, float) and math.isnan(v):
                v = "nan"
            out.append(v)
        return tuple(out)


def none_to_nan(v):
    return NAN if v is None else float(v)


# (name, restype, argtypes) of every exported entry point
_VP = ctypes.c_void_p
_DP = ctypes.c_void_p  # device pointers are passed as integers
SIGNATURES = [
    ("hitb200_version", ctypes.c_char_p, []),
    ("hitb200_status_string", ctypes.c_char_p, [ctypes.c_int]),
    ("hitb200_desc_size", ctypes.c_size_t, []),
    ("hitb200_desc_init", ctypes.c_int, [ctypes.POINTER(Desc)]),
    ("hitb200_plan_create", ctypes.c_int, [ctypes.POINTER(Desc), ctypes.POINTER(_VP)]),
    ("hitb200_plan_destroy", ctypes.c_int, [_VP]),
    ("hitb200_plan_device_bytes", ctypes.c_size_t, [ctypes.POINTER(Desc)]),
    ("hitb200_release_cached_blocks", ctypes.c_int, []),
    ("hitb200_cached_block_bytes", ctypes.c_size_t, []),
    ("hitb200_enforce", ctypes.c_int, [_VP, _DP, _DP, _VP]),
    ("hitb200_enforce_state", ctypes.c_int,
     [_DP, _DP, ctypes.c_int64, ctypes.c_double, _VP]),
    ("hitb200_sensor", ctypes.c_int, [_VP, _DP, _DP, ctypes.c_int, _VP]),
    ("hitb200_axis_derivative", ctypes.c_int, [_VP, _DP, _DP, ctypes.c_int, _DP, _VP]),
    ("hitb200_rhs", ctypes.c_int, [_VP, _DP, ctypes.c_int, _DP, _DP, _DP, _VP]),
    ("hitb200_viscous_rhs", ctypes.c_int, [_VP, _DP, _DP, _VP]),
    ("hitb200_hyperviscosity", ctypes.c_int, [_VP, _DP, _DP, _DP, _VP]),
    ("hitb200_outflow_guard", ctypes.c_int, [_VP, _DP, _VP]),
    ("hitb200_stable_time_step", ctypes.c_int,
     [_VP, _DP, ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]),
    ("hitb200_validate", ctypes.c_int, [_VP, _DP]),
    ("hitb200_stable_time_step_noalloc", ctypes.c_int,
     [_DP, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
      ctypes.c_double, ctypes.c_double, _DP, _VP]),
    ("hitb200_hit_streamfunction", ctypes.c_int,
     [_DP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
      ctypes.c_double, ctypes.c_double, _DP, _VP]),
    ("hitb200_hit_compose_workspace_bytes", ctypes.c_size_t, []),
    ("hitb200_hit_compose", ctypes.c_int,
     [_DP, _DP, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
      _DP, _DP, _VP, ctypes.c_size_t, _VP]),
    ("hitb200_riemann_initial_state", ctypes.c_int,
     [ctypes.POINTER(ctypes.c_double), ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
      ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
      ctypes.c_double, _DP, _VP]),
    ("hitb200_spectra_workspace_bytes", ctypes.c_size_t,
     [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    ("hitb200_spectra_fields", ctypes.c_int,
     [_DP, _DP, _DP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _DP, _VP,
      ctypes.c_size_t, _VP]),
    ("hitb200_spectra_state_fields", ctypes.c_int,
     [_DP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _DP, _VP,
      ctypes.c_size_t, _VP]),
    ("hitb200_spectra_shells", ctypes.c_int,
     [_VP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double, _DP,
      _DP, _VP, ctypes.c_size_t, _VP]),
    ("hitb200_forcing_update", ctypes.c_int,
     [_VP, _DP, _DP, ctypes.c_double, ctypes.c_double, _DP, _DP, _VP]),
    ("hitb200_step", ctypes.c_int, [_VP, _DP, _DP, _VP]),
    ("hitb200_run", ctypes.c_int, [_VP, _DP, ctypes.c_int32, _VP]),
    ("hitb200_step_profile", ctypes.c_int,
     [_VP, _DP, _DP, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double),
      ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), ctypes.c_char_p, ctypes.c_size_t, _VP]),
    ("hitb200_batch_step_profile", ctypes.c_int,
     [_VP, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double), ctypes.c_int32,
      ctypes.POINTER(ctypes.c_int32), ctypes.c_char_p, ctypes.c_size_t, _VP]),
    ("hitb200_set_time", ctypes.c_int,
     [_VP, ctypes.c_double, ctypes.c_int64, ctypes.c_double, ctypes.c_int64]),
    ("hitb200_read_scalars", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_double), ctypes.c_int32]),
    ("hitb200_copy_scalars_async", ctypes.c_int, [_VP, _DP, ctypes.c_int32, _VP]),
    ("hitb200_state_block_size", ctypes.c_size_t, []),
    ("hitb200_save_state_block", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_double), ctypes.c_size_t]),
    ("hitb200_load_state_block", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_double), ctypes.c_size_t]),
    ("hitb200_set_barrier_test", ctypes.c_int, [ctypes.c_int32, ctypes.c_double]),
    ("hitb200_set_noise_stream", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_uint64)]),
    ("hitb200_get_noise_stream", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_uint64)]),
    ("hitb200_noise_field", ctypes.c_int, [_VP, _DP, _VP]),
    ("hitb200_spectral_workspace_bytes", ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32]),
    ("hitb200_spectral_diagnostics", ctypes.c_int,
     [_VP, _DP, ctypes.c_double, ctypes.POINTER(ctypes.c_double), _DP, _DP, _DP, ctypes.c_size_t, _VP]),
    ("hitb200_hit_velocity_workspace_bytes", ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32]),
    ("hitb200_hit_velocity", ctypes.c_int,
     [_DP, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double, _DP, _DP, _DP,
      ctypes.c_size_t, _VP]),
    ("hitb200_rfft2_workspace_bytes", ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32]),
    ("hitb200_rfft2", ctypes.c_int,
     [_DP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _DP, _DP, ctypes.c_size_t, _VP]),
    ("hitb200_diagnostics", ctypes.c_int,
     [_VP, _DP, ctypes.POINTER(ctypes.c_double), ctypes.c_int32]),
    ("hitb200_batch_create", ctypes.c_int,
     [ctypes.POINTER(Desc), ctypes.c_int32, ctypes.POINTER(_VP)]),
    ("hitb200_batch_destroy", ctypes.c_int, [_VP]),
    ("hitb200_batch_from_plans", ctypes.c_int,
     [ctypes.POINTER(_VP), ctypes.c_int32, ctypes.POINTER(_VP)]),
    ("hitb200_plan_set_tuning", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32]),
    ("hitb200_plan_get_tuning", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32]),
    ("hitb200_batch_set_tuning", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32]),
    ("hitb200_batch_get_tuning", ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32]),
    ("hitb200_batch_plan", _VP, [_VP, ctypes.c_int32]),
    ("hitb200_batch_bind", ctypes.c_int, [_VP, ctypes.POINTER(_VP)]),
    ("hitb200_batch_step", ctypes.c_int, [_VP, _VP]),
    ("hitb200_batch_run", ctypes.c_int, [_VP, ctypes.c_int32, _VP]),
]

_lib = None


def load(path: Path | str | None = None) -> ctypes.CDLL:
    """Load the shared library (once).  Raises RuntimeError if it is absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"B200 backend library {p} is not built; run `python -m hit_solver_b200.build` "
            "(nvcc for sm_100a) first")
    lib = ctypes.CDLL(str(p))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.hitb200_desc_size() != ctypes.sizeof(Desc):
        raise RuntimeError("hitb200_desc layout mismatch between library and binding")
    if path is None:
        _lib = lib
    return lib


def check_step_status(bits: int, label: str) -> None:
    """Raise for the status bits a run loop must not continue past: a grid
    barrier that timed out (RuntimeError: the step's results are invalid)
    and a non-finite state (FloatingPointError, as the reference's loops
    raise).  The validation bits are left to the Riemann validation."""
    bits = int(bits)
    if bits & ST_BARRIER:
        raise RuntimeError(f"{label}: a bounded device wait (the fused prepass/sensor's grid barrier "
                           "or a persistent stage's queue) timed out")
    if bits & ST_NOISE:
        raise RuntimeError(f"{label}: the device forcing-noise stream ran short of draws")
    if bits & ST_NONFINITE:
        raise FloatingPointError(f"NaN or infinite value detected in {label}")


def check(status: int) -> None:
    """Raise the reference's exception type for a non-zero status."""
    if status == OK:
        return
    msg = load().hitb200_status_string(status).decode()
    if status == ERR_INVALID:
        raise ValueError(msg)
    if status in (ERR_NONFINITE, ERR_NONPOSITIVE):
        raise FloatingPointError(msg)
    if status == ERR_OOM:
        raise MemoryError(msg)
    raise RuntimeError(msg)


def default_desc() -> Desc:
    d = Desc()
    check(load().hitb200_desc_init(ctypes.byref(d)))
    return d
