"""Periodic hybrid compact/WENO7 operators on the B200 backend
(OOP/spatial_operator.py:252-435, OOP/parallel/spatial_operator.py:113-281).

Same constructor arguments and methods as the reference; arrays are torch
CUDA float64 tensors and every method runs the native sm_100a kernels.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import torch

from . import _lib, core
from .descs import grid_desc, set_sensor
from .domain import Domain2D
from .equations import EulerEquation2D


@dataclass(frozen=True)
class PeriodicEulerShockSensor2D:
    """Hybrid-switch mask (OOP/spatial_operator.py:252-304)."""

    domain: Domain2D
    equation: EulerEquation2D
    width: int = 4
    compression_threshold: float = 2.5
    jump_threshold: float = 0.04
    shear_threshold: float | None = None
    precision: str = "fp64"

    def descriptor(self) -> _lib.Desc:
        d = grid_desc(self.domain, self.equation.gamma, True, self.precision)
        set_sensor(d, self.width, self.compression_threshold, self.jump_threshold,
                   self.shear_threshold)
        return d

    def detect(self, q):
        """bool[ny, nx] mask of WENO nodes, on q as given."""
        q = core.as_state(q)
        return core.plan_for(self.descriptor()).sensor(q, enforce_first=False)


@dataclass
class PeriodicHybridEuler2DOperator:
    """-dF/dx - dG/dy with the hybrid scheme (OOP/spatial_operator.py:307-377)."""

    domain: Domain2D
    equation: EulerEquation2D
    sensor: PeriodicEulerShockSensor2D
    _desc: _lib.Desc = field(init=False, repr=False, default=None)

    def __post_init__(self) -> None:
        self._desc = self.sensor.descriptor()

    @property
    def plan(self) -> core.Plan:
        return core.plan_for(self._desc)

    def axis_derivative(self, q, shock_mask, axis: int):
        """d/dx (axis 0) or d/dy (axis 1) of the flux on enforce(q) with a given
        node mask (``_axis_derivative``, OOP/spatial_operator.py:321-342)."""
        q = core.as_state(q)
        m = core.as_field(shock_mask, q.shape[1:], "shock_mask", torch.uint8)
        return self.plan.axis_derivative(q, m, axis)

    def rhs(self, q):
        return self.plan.rhs(core.as_state(q), _lib.TERM_INVISCID)

    def stable_time_step(self, q, cfl: float, remaining_time: float | None = None) -> float:
        return self.plan.stable_time_step(core.as_state(q), cfl, remaining_time)


@dataclass(frozen=True)
class PeriodicHyperviscosity2D:
    """Biharmonic filter on compact-FD nodes only (OOP/spatial_operator.py:380-435)."""

    domain: Domain2D
    mn: float = 0.002
    density_weight: float = 0.25
    momentum_weight: float = 1.0
    energy_weight: float = 0.25
    precision: str = "fp64"

    def apply(self, q, equation: EulerEquation2D, active_mask=None):
        if active_mask is None:
            raise ValueError(
                "active_mask is required: hyperviscosity may only be "
                "applied on compact-FD nodes")
        q = core.as_state(q)
        if tuple(active_mask.shape) != tuple(q.shape[-2:]):
            raise ValueError(
                f"active_mask shape {tuple(active_mask.shape)} does not match grid "
                f"{tuple(q.shape[-2:])}")
        d = grid_desc(self.domain, equation.gamma, True, self.precision)
        d.hv_mn = self.mn
        for i, w in enumerate((self.density_weight, self.momentum_weight, self.momentum_weight,
                               self.energy_weight)):
            d.hv_weight[i] = w
        active = core.as_field(active_mask, q.shape[1:], "active_mask", torch.uint8)
        return core.plan_for(d).hyperviscosity(q, active)


# Names of the reference's backend-aware twins (OOP/parallel/spatial_operator.py).
ParallelPeriodicEulerShockSensor2D = PeriodicEulerShockSensor2D
ParallelPeriodicHybridEuler2DOperator = PeriodicHybridEuler2DOperator
ParallelPeriodicHyperviscosity2D = PeriodicHyperviscosity2D
