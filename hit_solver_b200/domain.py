"""Uniform cell-centred grids (OOP/domain.py:8-87); pure host objects."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Domain2D:
    """Cell-centred [x_min, x_max] x [y_min, y_max] grid with nx x ny cells;
    node (j, i) sits at x_min + dx (i + 1/2), y_min + dy (j + 1/2)
    (OOP/domain.py:49-87)."""

    x_min: float
    x_max: float
    y_min: float
    y_max: float
    nx: int
    ny: int

    def __post_init__(self) -> None:
        if self.nx <= 0 or self.ny <= 0:
            raise ValueError("nx and ny must be positive")
        if self.x_max <= self.x_min:
            raise ValueError("x_max must be greater than x_min")
        if self.y_max <= self.y_min:
            raise ValueError("y_max must be greater than y_min")

    @property
    def dx(self) -> float:
        return (self.x_max - self.x_min) / self.nx

    @property
    def dy(self) -> float:
        return (self.y_max - self.y_min) / self.ny

    @property
    def x(self) -> np.ndarray:
        return self.x_min + self.dx * (np.arange(self.nx) + 0.5)

    @property
    def y(self) -> np.ndarray:
        return self.y_min + self.dy * (np.arange(self.ny) + 0.5)

    def mesh(self):
        """X, Y of shape (ny, nx) matching state[:, y, x]."""
        return np.meshgrid(self.x, self.y, indexing="xy")
