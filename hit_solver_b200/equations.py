"""Ideal-gas Euler / Navier-Stokes helpers on torch CUDA state tensors
(OOP/equations.py:125-267, OOP/parallel/equations.py:11-141).

``enforce_physical_state`` and ``viscous_rhs`` run the native kernels.  The
primitive/flux helpers are host-API conveniences (elementwise torch on the
device) used by drivers and diagnostics, not by the fused step.
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

from . import _lib, core
from .descs import grid_desc
from .domain import Domain2D


@dataclass(frozen=True)
class EulerEquation2D:
    """State ordering [rho, rho*u, rho*v, E] (OOP/equations.py:126-130)."""

    gamma: float = 1.4
    rho_floor: float = 1e-10
    pressure_floor: float = 1e-10

    def primitive_from_conservative(self, q):
        rho = torch.clamp(q[0], min=self.rho_floor)
        u = q[1] / rho
        v = q[2] / rho
        kinetic = 0.5 * rho * (u ** 2 + v ** 2)
        pressure = (self.gamma - 1.0) * (q[3] - kinetic)
        return rho, u, v, torch.clamp(pressure, min=self.pressure_floor)

    def conservative_from_primitive(self, rho, u, v, pressure):
        rho, u, v, pressure = torch.broadcast_tensors(*(torch.as_tensor(a) for a in (rho, u, v, pressure)))
        rho = torch.clamp(rho, min=self.rho_floor)
        pressure = torch.clamp(pressure, min=self.pressure_floor)
        q = torch.zeros((4, *rho.shape), dtype=torch.float64, device=rho.device)
        q[0] = rho
        q[1] = rho * u
        q[2] = rho * v
        q[3] = pressure / (self.gamma - 1.0) + 0.5 * rho * (u ** 2 + v ** 2)
        return q

    def enforce_physical_state(self, q):
        """Native clean filter (OOP/equations.py:165-181)."""
        core.require_cuda()
        q = core.as_state(q)
        out = torch.empty_like(q)
        _lib.check(_lib.load().hitb200_enforce_state(q.data_ptr(), out.data_ptr(),
                                                     q.shape[1] * q.shape[2], float(self.gamma),
                                                     core.stream_handle()))
        return out

    def flux_x(self, q):
        rho, u, v, p = self.primitive_from_conservative(q)
        return torch.stack([q[1], rho * u ** 2 + p, rho * u * v, (q[3] + p) * u])

    def flux_y(self, q):
        rho, u, v, p = self.primitive_from_conservative(q)
        return torch.stack([q[2], rho * u * v, rho * v ** 2 + p, (q[3] + p) * v])

    def sound_speed(self, q):
        rho, _u, _v, p = self.primitive_from_conservative(q)
        return torch.sqrt(self.gamma * p / rho)

    def max_wave_speed(self, q) -> float:
        rho, u, v, p = self.primitive_from_conservative(q)
        c = torch.sqrt(self.gamma * p / rho)
        return float(torch.max(torch.maximum(u.abs() + c, v.abs() + c)))


@dataclass(frozen=True)
class CompressibleNavierStokes2D(EulerEquation2D):
    """Adds the periodic viscous / thermal RHS (OOP/equations.py:211-267)."""

    viscosity: float = 0.0
    prandtl: float = 0.72
    gas_constant: float = 1.0

    def temperature(self, rho, pressure):
        return pressure / (rho * self.gas_constant)

    def viscous_rhs(self, q, dx: float, dy: float):
        q = core.as_state(q)
        if self.viscosity == 0.0:
            return torch.zeros_like(q)
        ny, nx = q.shape[1:]
        d = grid_desc(Domain2D(0.0, nx * dx, 0.0, ny * dy, nx, ny), self.gamma, True)
        d.viscosity, d.prandtl, d.gas_constant = self.viscosity, self.prandtl, self.gas_constant
        return core.plan_for(d).viscous_rhs(q)


# Names of the reference's backend-aware twins (OOP/parallel/equations.py).
ParallelEulerEquation2D = EulerEquation2D
ParallelCompressibleNavierStokes2D = CompressibleNavierStokes2D
