"""Continuous-batching request loop for HIT and Riemann solves on one GPU.

Requests (a Riemann quadrant problem or a forced-HIT run of a given size)
arrive over time.  The loop admits each one as soon as its device footprint
(plan scratch plus state) fits in the memory budget, builds its resident
state on the device, and advances every admitted solve together: one batch
(``hitb200_batch_from_plans``) whose launches cover all members, replayed from
a captured graph for ``steps_per_round`` steps at a time.  A member that
reaches its end (tfinal, or its step count) turns into a device-side no-op; at
the next round boundary it is retired, its memory returned, and waiting
requests take its place.  Solves of different sizes and kinds share every
launch, so work that arrives while others run overlaps with them on the device.

Each solve's arithmetic does not depend on its batch companions: every kernel
works on one solve's data, and each reduction runs in a fixed order over that
solve's own tiles.  A result is therefore the same alone and in any mix.

The loop reports per-request time-to-tfinal (arrival to the end of the round
in which the solve finished) and aggregate cell-updates/s.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, core
from .batch import Batch
from .hit2d import HIT2DConfig, HITSolver
from .problems.riemann import RiemannConfig3, RiemannConfig6, RiemannSolver

KINDS = ("riemann3", "riemann6", "hit")


@dataclass
class Request:
    """One solve to run to its end.

    kind     "riemann3" / "riemann6" (Lax-Liu configurations 3 and 6 on the
             unit square, run to their tfinal) or "hit" (forced HIT, run for
             ``steps`` steps)
    n        grid size (n x n)
    arrival  seconds after the loop starts
    split    Riemann quadrant intersection x0 = y0
    seed     HIT initial-condition and forcing seed
    mach     HIT turbulent Mach number (initial and Mach-control target)
    initial_state
             optional conservative state [4, n, n] (host or device) that
             replaces the generated initial condition at admission: a
             restart, or a caller's own initial field
    """

    rid: int
    kind: str
    n: int
    arrival: float = 0.0
    split: float = 0.5
    seed: int = 0
    mach: float = 0.25
    steps: int = 200
    initial_state: torch.Tensor | None = field(default=None, repr=False)


@dataclass
class Result:
    rid: int
    kind: str
    n: int
    arrival: float
    admitted: float
    finished: float
    steps: int
    time: float
    status: int
    state: torch.Tensor | None = field(default=None, repr=False)
    # set when the solve was evicted: the exception type the reference's loops
    # raise for its state (FloatingPointError / RuntimeError) and the message
    error: str | None = None
    error_type: str | None = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def hit_request_config(n: int, seed: int, mach: float, steps: int, precision: str) -> HIT2DConfig:
    """The production forced-HIT physics (OU shell 3..5, tau 0.5, Mach control,
    nu 7.5e-4, hyperviscosity every 5 steps, drag on |k| <= 2, cooling 5.0,
    CFL 0.05) at size n, seed and Mach; device forcing noise and initial
    state; ``steps`` steps."""
    return HIT2DConfig(
        nx=n, ny=n, tfinal=math.inf, target_mach=mach, initial_kmin=3, initial_kmax=5,
        forcing_kmin=3.0, forcing_kmax=5.0, forcing_correlation_time=0.5,
        forcing_alpha_memory=0.2, target_energy_injection=1.0e-3, viscosity=7.5e-4,
        hyperviscosity_mn=0.002, hyperviscosity_interval=5, large_scale_drag=0.10,
        large_scale_drag_kmax=2.0, cooling_time=5.0, mach_control=True,
        mach_control_target=mach, forcing_seed=seed, cfl=0.05, precision=precision,
        forcing_noise="device", max_steps=steps, initial_condition="device")


def riemann_request_config(kind: str, n: int, split: float, precision: str) -> RiemannConfig3:
    cls = RiemannConfig6 if kind == "riemann6" else RiemannConfig3
    return cls(nx=n, ny=n, x_split=split, y_split=split, precision=precision)


def make_solver(req: Request, precision: str):
    """The resident solve of a request: a HITSolver or RiemannSolver whose
    plan and state live on the device, positioned at step 0."""
    if req.kind not in KINDS:
        raise ValueError(f"unknown request kind {req.kind!r}; expected one of {KINDS}")
    if req.n <= 0:
        raise ValueError("grid size must be positive")
    if req.kind == "hit":
        solver = HITSolver(hit_request_config(req.n, req.seed, req.mach, req.steps, precision))
    else:
        solver = RiemannSolver(riemann_request_config(req.kind, req.n, req.split, precision))
    if req.initial_state is not None:
        if tuple(req.initial_state.shape) != tuple(solver.q.shape):
            raise ValueError(f"request {req.rid}: initial_state must have shape {tuple(solver.q.shape)}")
        solver.q.copy_(req.initial_state)
    return solver


def member_error(kind: str, bits: int) -> tuple[str, str] | None:
    """The exception a solve's status bits call for, as the reference's loops
    raise it: FloatingPointError for a non-finite state (OOP/hit2d.py:716-717)
    and, for Riemann solves, a non-positive raw density or pressure
    (OOP/problems/riemann_config3.py:442-452); RuntimeError for a fused grid
    barrier that timed out.  None while the solve is sound."""
    bits = int(bits)
    if bits & _lib.ST_BARRIER:
        return "RuntimeError", "a bounded device wait (grid barrier or persistent stage queue) timed out"
    if bits & _lib.ST_NONFINITE:
        return "FloatingPointError", "NaN or infinite value detected in the state"
    if kind != "hit" and bits & _lib.ST_NONPOS_RHO:
        return "FloatingPointError", "state contains non-positive density"
    if kind != "hit" and bits & _lib.ST_NONPOS_P:
        return "FloatingPointError", "state contains non-positive pressure"
    return None


def footprint(req: Request, precision: str) -> int:
    """Device bytes a request holds while admitted: its plan's scratch plus
    its state (and the batch tables' share, rounded into a 1 MB margin)."""
    if req.kind == "hit":
        from .hit2d import create_grid, hit_descriptor

        cfg = hit_request_config(req.n, req.seed, req.mach, req.steps, precision)
        desc = hit_descriptor(cfg, create_grid(cfg)[0])
    else:
        from .problems.riemann import riemann_descriptor

        desc = riemann_descriptor(riemann_request_config(req.kind, req.n, req.split, precision))
    plan_bytes = int(_lib.load().hitb200_plan_device_bytes(desc))
    return plan_bytes + 4 * req.n * req.n * 8 + (1 << 20)


@dataclass
class _Member:
    req: Request
    solver: object
    bytes: int
    admitted: float


class SolveServer:
    """Admit, batch and retire solves as they arrive and finish.

    hbm_budget       device bytes the admitted solves may hold (default: 80 %
                     of the free device memory at construction)
    steps_per_round  steps replayed between admission/retirement points
    keep_states      keep each finished solve's final state (a device tensor)
    """

    def __init__(self, precision: str = "fp32-bulk", hbm_budget: int | None = None,
                 steps_per_round: int = 16, keep_states: bool = False):
        core.require_cuda()
        if steps_per_round <= 0:
            raise ValueError("steps_per_round must be positive")
        self.precision = precision
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info()
            hbm_budget = int(0.8 * free)
        self.hbm_budget = int(hbm_budget)
        self.steps_per_round = int(steps_per_round)
        self.keep_states = keep_states
        self.stats: dict = {}

    def serve(self, requests, clock=time.perf_counter) -> list[Result]:
        """Run every request to its end; returns results in completion order."""
        for r in requests:
            if footprint(r, self.precision) > self.hbm_budget:
                raise MemoryError(f"request {r.rid} ({r.kind} {r.n}^2) exceeds the HBM budget")
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        active: list[_Member] = []
        results: list[Result] = []
        used = 0
        batch = None
        dirty = False
        scal = torch.empty((64, _lib.S_COUNT), dtype=torch.float64).pin_memory()
        stream = torch.cuda.current_stream()
        rounds = 0
        cell_steps = 0.0
        # host time by phase: admission (plan and initial state), batch
        # rebuilds, rounds (launch, graph capture after a rebuild, the wait)
        phase = {"admit_s": 0.0, "rebuild_s": 0.0, "round_s": 0.0, "rebuilds": 0}
        t0 = clock()
        while pending or active:
            now = clock() - t0
            # ---- admission: FIFO while the head of the queue fits ----
            while pending and pending[0].arrival <= now:
                fp = footprint(pending[0], self.precision)
                if used + fp > self.hbm_budget:
                    break
                req = pending.pop(0)
                ta = clock()
                active.append(_Member(req, make_solver(req, self.precision), fp, ta - t0))
                phase["admit_s"] += clock() - ta
                used += fp
                dirty = True
            if not active:
                wait = pending[0].arrival - (clock() - t0)
                if wait > 0:
                    time.sleep(wait)
                continue
            if dirty:
                tr = clock()
                phase["rebuilds"] += 1
                if batch is not None:
                    batch.close()
                batch = Batch.from_plans([m.solver.plan for m in active],
                                         [m.solver.q for m in active])
                if scal.shape[0] < len(active):
                    scal = torch.empty((2 * len(active), _lib.S_COUNT),
                                       dtype=torch.float64).pin_memory()
                dirty = False
                phase["rebuild_s"] += clock() - tr
            tq = clock()
            batch.run(self.steps_per_round)
            rounds += 1
            for i, m in enumerate(active):
                m.solver.plan.lib.hitb200_copy_scalars_async(
                    m.solver.plan.handle, scal[i].data_ptr(), _lib.S_COUNT, stream.cuda_stream)
            stream.synchronize()
            phase["round_s"] += clock() - tq
            done_at = clock() - t0
            keep = []
            for i, m in enumerate(active):
                s = scal[i]
                # S_ACTIVE turns 0 at the first step past the end; a member
                # whose step count reached max_steps is done already; a member
                # whose state went bad is evicted (its companions are unaffected:
                # every kernel works on one solve's data)
                err = member_error(m.req.kind, s[_lib.S_STATUS])
                done = err is not None or s[_lib.S_ACTIVE] == 0.0 or (
                    s[_lib.S_MAX_STEPS] >= 0.0 and s[_lib.S_STEP] >= s[_lib.S_MAX_STEPS])
                if not done:
                    keep.append(m)
                    continue
                steps = int(s[_lib.S_STEP])
                cell_steps += float(m.req.n) * m.req.n * steps
                results.append(Result(m.req.rid, m.req.kind, m.req.n, m.req.arrival, m.admitted,
                                      done_at, steps, float(s[_lib.S_TIME]),
                                      int(s[_lib.S_STATUS]),
                                      m.solver.q if self.keep_states else None,
                                      error=None if err is None else err[1],
                                      error_type=None if err is None else err[0]))
                used -= m.bytes
            if len(keep) != len(active):
                batch.close()  # hands the plans back before finished ones are freed
                batch = None
                active = keep
                dirty = True
        if batch is not None:
            batch.close()
        makespan = clock() - t0
        lat = np.array([r.latency for r in results]) if results else np.zeros(1)
        self.stats = {
            "requests": len(results), "rounds": rounds, "makespan_s": makespan,
            "cell_updates_per_s": cell_steps / makespan if makespan > 0 else 0.0,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "steps_per_round": self.steps_per_round, "hbm_budget": self.hbm_budget,
            "failed": sum(1 for r in results if r.error is not None),
            **phase,
        }
        return results


def poisson_requests(count: int, rate: float, seed: int = 0, riemann_sizes=(256, 1024),
                     hit_sizes=(128, 512), hit_steps: int = 200, hit_fraction: float = 0.5,
                     size_step: int = 64) -> list[Request]:
    """A seeded Poisson stream mixing Riemann config 3/6 solves (x0 = y0 in
    [0.3, 0.8]) and forced-HIT solves (random seed, Mach in [0.1, 0.4]).
    Grid sizes are drawn uniformly on multiples of ``size_step``."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        if rng.random() < hit_fraction:
            lo, hi = hit_sizes
            n = int(rng.integers(lo // size_step, hi // size_step + 1)) * size_step
            out.append(Request(i, "hit", n, t, seed=int(rng.integers(0, 2 ** 31)),
                               mach=float(rng.uniform(0.1, 0.4)), steps=hit_steps))
        else:
            lo, hi = riemann_sizes
            n = int(rng.integers(lo // size_step, hi // size_step + 1)) * size_step
            kind = "riemann3" if rng.random() < 0.5 else "riemann6"
            out.append(Request(i, kind, n, t, split=float(rng.uniform(0.3, 0.8))))
    return out


def run_alone(req: Request, precision: str = "fp32-bulk") -> torch.Tensor:
    """The request's final state when it runs by itself through the plain
    single-solve path (its own plan and captured graph), the reference for
    the same request inside a mix."""
    solver = make_solver(req, precision)
    while True:
        s = solver.plan.scalars(_lib.S_COUNT)
        if s[_lib.S_ACTIVE] == 0.0 or (0.0 <= s[_lib.S_MAX_STEPS] <= s[_lib.S_STEP]):
            return solver.q
        solver.advance(64)


__all__ = ["Request", "Result", "SolveServer", "footprint", "hit_request_config",
           "make_solver", "member_error", "poisson_requests", "riemann_request_config",
           "run_alone"]
