"""CPU checks of the drop-in boundary: the C-ABI library loads, exports every
symbol its header declares, agrees on the descriptor layout, and the host
logic (descriptor defaults, error mapping, configuration validation) matches
the reference's conventions.  No compute call is made (no GPU here)."""

import ctypes
import math
import re
from pathlib import Path

import pytest

from hit_solver_b200 import _lib
from hit_solver_b200.build import build

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def lib():
    build()
    return _lib.load()


def declared_symbols():
    text = (ROOT / "include" / "hitb200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hitb200_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(lib):
    names = declared_symbols()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name


def test_binding_covers_header():
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(declared_symbols()) <= bound


def test_tuning_knob_indices_match_header():
    """The binding's tuning-knob indices (and their count, which bounds the
    knob arrays passed to hitb200_*_set_tuning) are the header's."""
    text = (ROOT / "include" / "hitb200.h").read_text()
    defs = dict(re.findall(r"#define HITB200_TUNE_([A-Z_]+) (\d+)", text))
    assert {k: int(v) for k, v in defs.items()} == {
        "SWEEP_X": _lib.TUNE_SWEEP_X, "SWEEP_Y": _lib.TUNE_SWEEP_Y, "PREPASS": _lib.TUNE_PREPASS,
        "FUSED_SENSOR": _lib.TUNE_FUSED_SENSOR, "Y_PANEL": _lib.TUNE_Y_PANEL,
        "PERSISTENT": _lib.TUNE_PERSISTENT, "COUNT": _lib.TUNE_COUNT}


def test_desc_layout_and_defaults(lib):
    assert lib.hitb200_desc_size() == ctypes.sizeof(_lib.Desc)
    d = _lib.default_desc()
    # HIT2DConfig defaults (OOP/hit2d.py:36-80)
    assert (d.nx, d.ny) == (128, 128)
    assert d.gamma == 1.4 and d.cfl == 0.05 and d.tfinal == 1.0
    assert d.sensor_width == 4 and d.jump_threshold == 0.04 and d.compression_threshold == 2.5
    assert math.isnan(d.shear_threshold)
    assert d.viscosity == 1e-3 and d.prandtl == 0.72
    assert d.hv_mn == 0.002 and d.hv_interval == 5
    assert tuple(d.hv_weight) == (0.25, 1.0, 1.0, 0.25)
    assert d.target_power == 1e-3 and d.min_power == 1e-6 and d.max_rescale == 20.0
    assert d.alpha_memory == 0.2 and d.mach_memory == 0.995 and d.mach_exponent == 2.0
    assert d.x_max == pytest.approx(2 * math.pi)


def test_plan_device_bytes_is_host_only(lib):
    d = _lib.default_desc()
    d.nx = d.ny = 512
    b = lib.hitb200_plan_device_bytes(ctypes.byref(d))
    # two stage buffers, rhs buffer, viscous buffer, forcing fields, noise
    assert 512 * 512 * (2 * 32 + 32 + 24 + 16 + 8) <= b < 512 * 512 * 200
    d.precision = 1
    assert lib.hitb200_plan_device_bytes(ctypes.byref(d)) < b


@pytest.mark.parametrize("field,value", [
    ("nx", 0), ("precision", 3), ("scheme", 2), ("sensor_width", 9), ("nx", 2048)])
def test_invalid_descriptors_are_rejected_without_gpu(lib, field, value):
    d = _lib.default_desc()
    setattr(d, field, value)
    assert lib.hitb200_plan_device_bytes(ctypes.byref(d)) == 0
    h = ctypes.c_void_p()
    st = lib.hitb200_plan_create(ctypes.byref(d), ctypes.byref(h))
    assert st in (_lib.ERR_INVALID, _lib.ERR_UNSUPPORTED)
    assert not h.value


def test_forcing_validation_messages(lib):
    d = _lib.default_desc()
    d.forcing_kmin, d.forcing_kmax = 5.0, 3.0
    h = ctypes.c_void_p()
    assert lib.hitb200_plan_create(ctypes.byref(d), ctypes.byref(h)) == _lib.ERR_INVALID
    assert b"0 <= k_min <= k_max" in lib.hitb200_status_string(_lib.ERR_INVALID)
    with pytest.raises(ValueError, match="k_min"):
        _lib.check(_lib.ERR_INVALID)


def test_status_mapping():
    with pytest.raises(FloatingPointError):
        _lib.check(_lib.ERR_NONFINITE)
    with pytest.raises(FloatingPointError):
        _lib.check(_lib.ERR_NONPOSITIVE)
    with pytest.raises(MemoryError):
        _lib.check(_lib.ERR_OOM)
    with pytest.raises(RuntimeError):
        _lib.check(_lib.ERR_CUDA)
    _lib.check(_lib.OK)


def test_null_arguments_are_rejected(lib):
    assert lib.hitb200_plan_create(None, None) == _lib.ERR_INVALID
    assert lib.hitb200_enforce_state(None, None, 10, 1.4, None) == _lib.ERR_INVALID
    assert lib.hitb200_step(None, None, None, None) == _lib.ERR_INVALID
    assert lib.hitb200_plan_destroy(None) == _lib.OK


def test_step_status_bits_map_to_exceptions():
    """The run loops' host check of the S_STATUS bits: a timed-out grid
    barrier is a RuntimeError (the step's results are invalid), a non-finite
    state a FloatingPointError; the validation bits are left to the Riemann
    validation and pass."""
    import pytest

    from hit_solver_b200 import _lib

    _lib.check_step_status(0, "x")
    _lib.check_step_status(float(_lib.ST_NONPOS_RHO | _lib.ST_NONPOS_P), "x")
    with pytest.raises(RuntimeError, match="barrier"):
        _lib.check_step_status(_lib.ST_BARRIER | _lib.ST_NONFINITE, "x")
    with pytest.raises(FloatingPointError, match="NaN"):
        _lib.check_step_status(float(_lib.ST_NONFINITE), "HIT2D state")
