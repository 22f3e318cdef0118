"""Solenoidal Ornstein-Uhlenbeck shell forcing on the B200 backend
(OOP/forcing.py:11-130).

The OU potential, the power-rescaling coefficient and every statistic live in
the native plan's device scalar block; the shell transform, the OU update and
the synthesis of (fx, fy) run as native kernels.  White noise comes either
from the reference's own NumPy stream (``noise="numpy"``:
``default_rng(seed).standard_normal((ny, nx))`` per update, uploaded, so a run
follows the reference's CPU forcing trajectory exactly) or is drawn on the
device (``noise="device"``: the shell coefficients of the same white-noise
distribution from a counter-based generator).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, core
from .descs import grid_desc
from .domain import Domain2D


@dataclass
class IsotropicShellOUForcing2D:
    domain: Domain2D
    k_min: float
    k_max: float
    correlation_time: float = 1.0
    force_rms: float = 1.0
    target_power: float | None = 1.0e-3
    min_power: float = 1.0e-6
    max_rescale: float | None = 20.0
    alpha_memory: float = 0.2
    seed: int = 1234
    xp: object = None
    noise: str = "numpy"
    _plan: core.Plan = field(default=None, init=False, repr=False)
    _rng: object = field(default=None, init=False, repr=False)

    def __post_init__(self) -> None:
        if self.k_min < 0.0 or self.k_max <= 0.0 or self.k_min > self.k_max:
            raise ValueError("forcing shell must satisfy 0 <= k_min <= k_max")
        if self.correlation_time <= 0.0:
            raise ValueError("forcing correlation time must be positive")
        if not 0.0 <= self.alpha_memory < 1.0:
            raise ValueError("alpha_memory must be in [0, 1)")
        if self.noise not in ("numpy", "device"):
            raise ValueError("noise must be 'numpy' or 'device'")
        d = grid_desc(self.domain, 1.4, True)
        d.forcing_on = 1
        d.forcing_kmin, d.forcing_kmax = float(self.k_min), float(self.k_max)
        d.forcing_correlation_time = self.correlation_time
        d.forcing_rms = self.force_rms
        d.target_power = _lib.none_to_nan(self.target_power)
        d.min_power = self.min_power
        d.max_rescale = _lib.none_to_nan(self.max_rescale)
        d.alpha_memory = self.alpha_memory
        d.noise_mode = 0 if self.noise == "numpy" else 1
        d.seed = int(self.seed)
        self._plan = core.Plan(d)
        self._rng = np.random.default_rng(self.seed)

    @property
    def alpha(self) -> float:
        return self._plan.scalars()[_lib.S_F_ALPHA]

    def update(self, dt: float, rho, u, v):
        """Advance the OU state once; returns fx, fy (torch CUDA) and the info
        dict of the reference (OOP/forcing.py:70-130)."""
        if dt <= 0.0:
            raise ValueError("forcing update requires dt > 0")
        ny, nx = self.domain.ny, self.domain.nx
        q = torch.empty((4, ny, nx), dtype=torch.float64, device=rho.device)
        q[0] = rho
        q[1] = rho * u
        q[2] = rho * v
        q[3] = 1.0 + 0.5 * rho * (u * u + v * v)  # any positive pressure
        noise = None
        if self.noise == "numpy":
            noise = torch.from_numpy(self._rng.standard_normal((ny, nx))).to(rho.device)
        fx, fy = self._plan.forcing_update(q, noise, dt, self.target_power)
        s = self._plan.scalars()
        info = {
            "alpha": s[_lib.S_F_ALPHA],
            "alpha_target": s[_lib.S_F_ALPHA_TARGET],
            "target_power": float("nan") if self.target_power is None else float(self.target_power),
            "power_before_rescale": s[_lib.S_F_POWER_BEFORE],
            "injected_power": s[_lib.S_F_INJECTED],
            "Fxx": s[_lib.S_F_FXX],
            "Fyy": s[_lib.S_F_FYY],
            "Fxy": s[_lib.S_F_FXY],
            "A_F": s[_lib.S_F_AF],
            "ou_decay": s[_lib.S_F_DECAY],
        }
        return fx, fy, info
