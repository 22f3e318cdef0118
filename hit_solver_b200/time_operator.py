"""SSP-RK3 and the minimal time loop (OOP/time_operator.py:17-69).

These are the reference's generic integrators, kept for API compatibility:
they accept any RHS callable and array type.  The production path advances a
whole step in the native library (:meth:`hit_solver_b200.core.Plan.step`),
which fuses the three stages, their RHS evaluations and the clean filter.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable

from .boundary_conditions import BoundaryCondition, PeriodicBoundary

State = object
RHS = Callable[[State], State]
StateFilter = Callable[[State], State]
StepHook = Callable[[int, State], State]


@dataclass(frozen=True)
class SSPRK3:
    """Shu-Osher third-order SSP Runge-Kutta with a clean filter per stage."""

    def step(self, state, rhs: RHS, dt: float, clean: StateFilter | None = None):
        cl = clean if clean is not None else (lambda value: value)
        q0 = state
        q1 = cl(q0 + dt * rhs(q0))
        q2 = cl(0.75 * q0 + 0.25 * (q1 + dt * rhs(q1)))
        return cl((1.0 / 3.0) * q0 + (2.0 / 3.0) * (q2 + dt * rhs(q2)))


@dataclass
class TimeOperator:
    """Fixed-dt loop with boundary/filter hooks (OOP/time_operator.py:29-69)."""

    state: State
    rhs: RHS
    dt: float
    boundary: BoundaryCondition = field(default_factory=PeriodicBoundary)
    integrator: SSPRK3 = field(default_factory=SSPRK3)
    state_filter: StateFilter | None = None
    step_hooks: list = field(default_factory=list)

    def __post_init__(self) -> None:
        self.state = self.clean(self.state)

    def clean(self, state):
        if self.state_filter is not None:
            state = self.state_filter(state)
        return self.boundary.apply(state)

    def step(self, step_index: int):
        self.state = self.integrator.step(self.state, self.rhs, self.dt, clean=self.clean)
        for hook in self.step_hooks:
            self.state = self.clean(hook(step_index, self.state))
        return self.state

    def run(self, t_end: float, save_every: int | None = None):
        import math

        n_steps = int(math.ceil(t_end / self.dt))
        if n_steps > 0:
            self.dt = t_end / n_steps
        if save_every is None:
            save_every = n_steps
        times = [0.0]
        states = [self.state.clone()]
        for step_index in range(n_steps):
            self.step(step_index)
            if (step_index + 1) % save_every == 0 or step_index + 1 == n_steps:
                times.append((step_index + 1) * self.dt)
                states.append(self.state.clone())
        return times, states
