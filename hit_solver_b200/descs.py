"""Build native solve descriptors from the reference-style configuration."""

from __future__ import annotations

from . import _lib
from .domain import Domain2D

FP64, FP32_BULK = 0, 1


def precision_code(precision) -> int:
    if precision in (0, "fp64", "float64"):
        return FP64
    if precision in (1, "fp32", "fp32-bulk", "float32"):
        return FP32_BULK
    raise ValueError("precision must be 'fp64' or 'fp32-bulk'")


def grid_desc(domain: Domain2D, gamma: float, periodic: bool, precision=FP64) -> _lib.Desc:
    """A descriptor with every optional term off."""
    d = _lib.default_desc()
    d.nx, d.ny = domain.nx, domain.ny
    d.x_min, d.x_max, d.y_min, d.y_max = domain.x_min, domain.x_max, domain.y_min, domain.y_max
    d.periodic = 1 if periodic else 0
    d.precision = precision_code(precision)
    d.gamma = gamma
    d.viscosity = 0.0
    d.hv_mn = 0.0
    d.hv_interval = 0
    d.forcing_on = 0
    d.drag_coefficient = 0.0
    d.cooling_time = _lib.NAN
    return d


def set_sensor(d: _lib.Desc, width, compression_threshold, jump_threshold, shear_threshold,
               boundary_guard=0) -> None:
    d.sensor_width = int(width)
    d.compression_threshold = float(compression_threshold)
    d.jump_threshold = float(jump_threshold)
    d.shear_threshold = _lib.none_to_nan(shear_threshold)
    d.boundary_guard = int(boundary_guard)
