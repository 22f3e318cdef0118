"""Boundary conditions on state arrays whose last axis is x
(OOP/boundary_conditions.py:8-64), for torch tensors."""

from __future__ import annotations

from dataclasses import dataclass


class BoundaryCondition:
    def apply(self, state):
        raise NotImplementedError


@dataclass(frozen=True)
class PeriodicBoundary(BoundaryCondition):
    """Stencils wrap, so only a defensive copy is made."""

    def apply(self, state):
        return state.clone()


@dataclass(frozen=True)
class ExtrapolatedBoundary2D(BoundaryCondition):
    """Zero-gradient guard cells on both axes (OOP/boundary_conditions.py:46-64)."""

    guard_cells: int = 0

    def apply(self, state):
        arr = state.clone()
        g = self.guard_cells
        if g == 0:
            return arr
        if arr.shape[-1] <= 2 * g or arr.shape[-2] <= 2 * g:
            raise ValueError("state is too small for the requested guard cells")
        arr[..., :, :g] = arr[..., :, g:g + 1]
        arr[..., :, -g:] = arr[..., :, -g - 1:-g]
        arr[..., :g, :] = arr[..., g:g + 1, :]
        arr[..., -g:, :] = arr[..., -g - 1:-g, :]
        return arr
