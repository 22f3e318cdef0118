"""Lax-Liu four-quadrant Riemann problems on the B200 backend
(OOP/problems/riemann_config3.py, riemann_config3_08.py, riemann_config6.py).

Same configuration dataclasses, operator classes, diagnostics and output
formats as the reference.  ``run_riemann`` keeps the state on the device and
replays one captured CUDA graph per step (SSP-RK3 with the enforce + outflow
guard clean, hyperviscosity every ``hyperviscosity_interval`` steps).
"""

from __future__ import annotations

import ctypes
import json
import math
from dataclasses import asdict, dataclass, field
from pathlib import Path
from typing import ClassVar

import numpy as np
import torch

from .. import _lib, core
from ..backend import select_array_module, to_numpy
from ..descs import grid_desc, set_sensor
from ..domain import Domain2D
from ..equations import EulerEquation2D
from ..run_utils import make_run_id, write_json


@dataclass(frozen=True)
class RiemannConfig3:
    """Lax-Liu / Kurganov-Tadmor configuration 3 (riemann_config3.py:19-99).
    Additive field: ``precision`` ("fp64" plain form or "fp32-bulk")."""

    configuration_number: ClassVar[int] = 3

    nx: int = 512
    ny: int = 512
    tfinal: float = 0.3
    cfl: float = 0.4
    gamma: float = 1.4
    x_min: float = 0.0
    x_max: float = 1.0
    y_min: float = 0.0
    y_max: float = 1.0
    x_split: float = 0.5
    y_split: float = 0.5
    backend: str = "b200"
    scheme: str = "hybrid"
    sensor_width: int = 4
    jump_threshold: float = 0.025
    compression_threshold: float = 2.5
    shear_threshold: float | None = 0.0
    boundary_guard: int = 4
    mn: float = 0.001
    hyperviscosity_interval: int = 1
    hyperviscosity_density_weight: float = 1.0
    hyperviscosity_momentum_weight: float = 1.0
    hyperviscosity_energy_weight: float = 1.0
    progress_every: int = 500
    guard_cells: int = 2
    save_final_npz: bool = True
    precision: str = "fp64"

    @property
    def domain(self) -> Domain2D:
        return Domain2D(self.x_min, self.x_max, self.y_min, self.y_max, self.nx, self.ny)

    @property
    def equation(self) -> EulerEquation2D:
        return EulerEquation2D(gamma=self.gamma)

    # quadrant states (rho, u, v, p): lower-left, lower-right, upper-left, upper-right
    _STATES: ClassVar[dict] = {
        "ll": (0.138, 1.206, 1.206, 0.029), "lr": (0.5323, 0.0, 1.206, 0.3),
        "ul": (0.5323, 1.206, 0.0, 0.3), "ur": (1.5, 0.0, 0.0, 1.5)}

    def initial_state(self):
        """Piecewise-constant quadrants (riemann_config3.py:59-99); a cell is
        upper/right when its centre is >= the split.  Filled on the device
        (``hitb200_riemann_initial_state``), bit for bit the reference's
        values."""
        core.require_cuda()
        dom = self.domain
        states = (ctypes.c_double * 16)(*[float(c) for key in ("ll", "lr", "ul", "ur")
                                          for c in self._STATES[key]])
        q = torch.empty((4, self.ny, self.nx), dtype=torch.float64, device="cuda")
        _lib.check(_lib.load().hitb200_riemann_initial_state(
            states, self.nx, self.ny, float(dom.x_min), float(dom.dx), float(dom.y_min),
            float(dom.dy), float(self.x_split), float(self.y_split), float(self.gamma),
            q.data_ptr(), core.stream_handle()))
        return q


@dataclass(frozen=True)
class RiemannConfig3Offset08(RiemannConfig3):
    """Configuration 3 with the intersection at x0 = y0 = 0.8 (riemann_config3_08.py:9-19)."""

    scenario_name: ClassVar[str] = "riemann_config3_08"
    configuration_label: ClassVar[str] = "Configuration 3 (x0=y0=0.8)"

    x_split: float = 0.8
    y_split: float = 0.8
    hyperviscosity_interval: int = 5


@dataclass(frozen=True)
class RiemannConfig6(RiemannConfig3):
    """Lax-Liu configuration 6: four contact discontinuities (riemann_config6.py:17-64)."""

    configuration_number: ClassVar[int] = 6
    _STATES: ClassVar[dict] = {
        "ll": (1.0, -0.75, 0.5, 1.0), "lr": (3.0, -0.75, -0.5, 1.0),
        "ul": (2.0, 0.75, 0.5, 1.0), "ur": (1.0, 0.75, -0.5, 1.0)}

    tfinal: float = 0.25


@dataclass(frozen=True)
class RiemannDiagnostics:
    backend: str
    scheme: str
    hyperviscosity_enabled: bool
    hyperviscosity_applications: int
    final_sensor_fraction: float
    density_min: float
    density_max: float
    pressure_min: float
    pressure_max: float
    max_abs_vorticity: float
    has_nonfinite: bool
    density_positive: bool
    pressure_positive: bool
    time: float
    steps: int


def _outflow_desc(domain: Domain2D, gamma: float, precision="fp64") -> _lib.Desc:
    return grid_desc(domain, gamma, False, precision)


@dataclass(frozen=True)
class NonPeriodicEulerShockSensor2D:
    """Outflow-grid sensor with a forced boundary band (riemann_config3.py:278-326)."""

    domain: Domain2D
    equation: EulerEquation2D
    width: int = 4
    compression_threshold: float = 2.5
    jump_threshold: float = 0.04
    shear_threshold: float | None = 2.0
    boundary_guard: int = 4
    precision: str = "fp64"

    def descriptor(self) -> _lib.Desc:
        d = _outflow_desc(self.domain, self.equation.gamma, self.precision)
        set_sensor(d, self.width, self.compression_threshold, self.jump_threshold,
                   self.shear_threshold, self.boundary_guard)
        return d

    def detect(self, q):
        q = core.as_state(q)
        return core.plan_for(self.descriptor()).sensor(q, enforce_first=False)


@dataclass
class NonPeriodicHybridEuler2DOperator:
    """Hybrid (or WENO-only) operator with clamped stencils, n+1 faces and the
    identity-end-row compact solve (riemann_config3.py:329-378)."""

    domain: Domain2D
    equation: EulerEquation2D
    sensor: NonPeriodicEulerShockSensor2D
    scheme: str = "hybrid"
    _desc: _lib.Desc = field(init=False, repr=False, default=None)

    def __post_init__(self):
        if self.scheme not in {"hybrid", "weno"}:
            raise ValueError("scheme must be 'hybrid' or 'weno'")
        self._desc = self.sensor.descriptor()
        self._desc.scheme = 0 if self.scheme == "hybrid" else 1

    @property
    def plan(self) -> core.Plan:
        return core.plan_for(self._desc)

    def axis_derivative(self, q, shock_mask, axis: int):
        q = core.as_state(q)
        m = core.as_field(shock_mask, q.shape[1:], "shock_mask", torch.uint8)
        return self.plan.axis_derivative(q, m, axis)

    def rhs(self, q):
        return self.plan.rhs(core.as_state(q), _lib.TERM_INVISCID)

    def fixed_time_step(self, q, cfl: float, t_end: float):
        dt = self.plan.stable_time_step(core.as_state(q), cfl, None)
        n_steps = int(math.ceil(t_end / dt))
        return t_end / n_steps, n_steps


@dataclass(frozen=True)
class LocalHyperviscosity2D:
    """Edge-padded biharmonic filter on compact nodes (riemann_config3.py:381-416)."""

    domain: Domain2D
    mn: float = 0.001
    density_weight: float = 1.0
    momentum_weight: float = 1.0
    energy_weight: float = 1.0
    precision: str = "fp64"

    def apply(self, q, compact_mask, equation):
        q = core.as_state(q)
        if tuple(compact_mask.shape) != tuple(q.shape[-2:]):
            raise ValueError(
                f"compact_mask shape {tuple(compact_mask.shape)} does not match grid "
                f"{tuple(q.shape[-2:])}")
        d = _outflow_desc(self.domain, equation.gamma, self.precision)
        d.hv_mn = self.mn
        for i, w in enumerate((self.density_weight, self.momentum_weight, self.momentum_weight,
                               self.energy_weight)):
            d.hv_weight[i] = w
        active = core.as_field(compact_mask, q.shape[1:], "compact_mask", torch.uint8)
        return core.plan_for(d).hyperviscosity(q, active)


def apply_outflow_guard(q, guard_cells: int = 2):
    """Zero-gradient guard cells, x first then y (riemann_config3.py:419-429)."""
    q = core.as_state(q)
    if guard_cells <= 0:
        return q
    ny, nx = q.shape[1:]
    d = _outflow_desc(Domain2D(0.0, 1.0, 0.0, 1.0, nx, ny), 1.4)
    d.guard_cells = int(guard_cells)
    return core.plan_for(d).outflow_guard(q)


def validate_raw_physical_state(q, equation, label: str = "state") -> None:
    """Raise FloatingPointError on non-finite or non-positive raw state
    (riemann_config3.py:442-452)."""
    q = core.as_state(q)
    ny, nx = q.shape[1:]
    plan = core.plan_for(_outflow_desc(Domain2D(0.0, 1.0, 0.0, 1.0, nx, ny), equation.gamma))
    st = plan.validate(q)
    if st == _lib.ERR_NONFINITE:
        raise FloatingPointError(f"{label} contains NaN or Inf values")
    if st == _lib.ERR_NONPOSITIVE:
        rho = q[0]
        if bool((rho <= 0.0).any()):
            raise FloatingPointError(f"{label} contains non-positive density")
        raise FloatingPointError(f"{label} contains non-positive pressure")
    _lib.check(st)


def vorticity_z(q, domain: Domain2D, equation):
    """dv/dx - du/dy with one-sided edge differences (riemann_config3.py:459-463)."""
    _, u, v, _ = equation.primitive_from_conservative(q)

    def fd(a, h, axis):
        out = torch.empty_like(a)
        m = a.movedim(axis, -1)
        o = out.movedim(axis, -1)
        o[..., 1:-1] = (m[..., 2:] - m[..., :-2]) / (2.0 * h)
        o[..., 0] = (m[..., 1] - m[..., 0]) / h
        o[..., -1] = (m[..., -1] - m[..., -2]) / h
        return out

    return fd(v, domain.dx, -1) - fd(u, domain.dy, -2)


def hyperviscosity_enabled_for_config(config: RiemannConfig3) -> bool:
    """WENO-only runs have no compact nodes, so no hyperviscosity
    (riemann_config3.py:667-678)."""
    return config.scheme == "hybrid" and config.mn > 0.0 and config.hyperviscosity_interval > 0


def riemann_descriptor(config: RiemannConfig3) -> _lib.Desc:
    d = _outflow_desc(config.domain, config.gamma, config.precision)
    set_sensor(d, config.sensor_width, config.compression_threshold, config.jump_threshold,
               config.shear_threshold, config.boundary_guard)
    d.scheme = 0 if config.scheme == "hybrid" else 1
    d.guard_cells = config.guard_cells
    if hyperviscosity_enabled_for_config(config):
        d.hv_mn = config.mn
        d.hv_interval = config.hyperviscosity_interval
        for i, w in enumerate((config.hyperviscosity_density_weight,
                               config.hyperviscosity_momentum_weight,
                               config.hyperviscosity_momentum_weight,
                               config.hyperviscosity_energy_weight)):
            d.hv_weight[i] = w
    d.cfl, d.tfinal = config.cfl, config.tfinal
    d.fixed_dt = 1
    return d


def _diagnostics(q, config, time, steps, hv_apps, plan: core.Plan) -> RiemannDiagnostics:
    vals = plan.diagnostics(q)
    rho_min, rho_max, p_min, p_max = vals[13:17]
    omega = vorticity_z(q, config.domain, config.equation)
    has_nonfinite = plan.validate(q) == _lib.ERR_NONFINITE
    sensor_fraction = float(plan.sensor(q, enforce_first=False).double().mean())
    return RiemannDiagnostics(
        backend=config.backend, scheme=config.scheme,
        hyperviscosity_enabled=hyperviscosity_enabled_for_config(config),
        hyperviscosity_applications=hv_apps, final_sensor_fraction=sensor_fraction,
        density_min=rho_min, density_max=rho_max, pressure_min=p_min, pressure_max=p_max,
        max_abs_vorticity=float(omega.abs().max()), has_nonfinite=bool(has_nonfinite),
        density_positive=bool(rho_min > 0.0), pressure_positive=bool(p_min > 0.0),
        time=time, steps=steps)


class RiemannSolver:
    """A resident Riemann solve (state on the device)."""

    def __init__(self, config: RiemannConfig3):
        select_array_module(config.backend)
        self.config = config
        self.plan = core.Plan(riemann_descriptor(config))
        q = config.initial_state()
        q = config.equation.enforce_physical_state(q)
        self.q = apply_outflow_guard(q, config.guard_cells)
        validate_raw_physical_state(self.q, config.equation, "initial state")
        dt = self.plan.stable_time_step(self.q, config.cfl, None)
        self.n_steps = int(math.ceil(config.tfinal / dt))
        self.dt = config.tfinal / self.n_steps
        self.plan.set_time(0.0, 0, self.dt, self.n_steps)

    def advance(self, nsteps: int) -> None:
        self.plan.run(self.q, nsteps)

    def checkpoint(self) -> dict:
        """The state and the plan's scalar block (time, step, dt,
        hyperviscosity count): ``restore`` resumes the run bit for bit."""
        torch.cuda.synchronize()
        return {"q": self.q.detach().cpu().clone(), "block": self.plan.save_state_block()}

    def restore(self, ck: dict) -> None:
        if tuple(ck["q"].shape) != tuple(self.q.shape):
            raise ValueError("checkpoint state does not match the solver's grid")
        self.q.copy_(ck["q"])
        self.plan.load_state_block(ck["block"])


def print_diagnostic_summary(d: RiemannDiagnostics) -> None:
    print("Diagnostic summary:")
    print(f"  backend              : {d.backend}")
    print(f"  scheme               : {d.scheme}")
    print(f"  density min/max      : {d.density_min:.8e} / {d.density_max:.8e}")
    print(f"  pressure min/max     : {d.pressure_min:.8e} / {d.pressure_max:.8e}")
    print(f"  max |vorticity|      : {d.max_abs_vorticity:.8e}")
    print(f"  NaN/Inf present      : {d.has_nonfinite}")
    print(f"  density positive     : {d.density_positive}")
    print(f"  pressure positive    : {d.pressure_positive}")
    print(f"  final sensor fraction: {d.final_sensor_fraction:.6f}")
    print(f"  hyperviscosity       : {d.hyperviscosity_enabled} ({d.hyperviscosity_applications} applications)")


def as_config(config) -> RiemannConfig3:
    """The mirror's configuration for a configuration object of the reference
    (its RiemannConfig3 / RiemannConfig3Offset08 / RiemannConfig6 with
    ``backend="b200"``): the class of the same name, its fields copied."""
    if isinstance(config, RiemannConfig3):
        return config
    from dataclasses import fields

    cls = {"RiemannConfig3Offset08": RiemannConfig3Offset08,
           "RiemannConfig6": RiemannConfig6}.get(type(config).__name__, RiemannConfig3)
    names = {f.name for f in fields(cls)}
    return cls(**{k: getattr(config, k) for k in names if hasattr(config, k)})


def run_riemann(config: RiemannConfig3):
    """Driver of riemann_config3.py:681-749 on the B200 backend; returns (q, diagnostics)."""
    config = as_config(config)
    print("Using array backend: b200")
    solver = RiemannSolver(config)
    label = getattr(config, "configuration_label", f"Config {config.configuration_number}")
    print(f"Riemann {label}: nx={config.nx}, ny={config.ny}, dt={solver.dt:.5e}, "
          f"steps={solver.n_steps}, tfinal={config.tfinal}")
    hv_on = hyperviscosity_enabled_for_config(config)
    note = "enabled on compact-FD nodes only" if hv_on else "disabled"
    if config.scheme == "weno" and config.mn > 0.0:
        note += " (WENO-only scheme)"
    print(f"scheme={config.scheme}; local hyperviscosity {note} (mn={config.mn})")
    done = 0
    while done < solver.n_steps:
        chunk = min(config.progress_every - done % config.progress_every, solver.n_steps - done)
        solver.advance(chunk)
        done += chunk
        if done % config.progress_every == 0 or done == solver.n_steps:
            _lib.check_step_status(solver.plan.scalars()[_lib.S_STATUS], f"state at step {done}")
            validate_raw_physical_state(solver.q, config.equation, f"state at step {done}")
            print(f"step={done:6d}, time={done * solver.dt:.6f}")
    s = solver.plan.scalars()
    apps = int(s[_lib.S_HV_APPLIED])
    diagnostics = _diagnostics(solver.q, config, solver.n_steps * solver.dt, solver.n_steps, apps,
                               solver.plan)
    validate_raw_physical_state(solver.q, config.equation, "final state")
    print_diagnostic_summary(diagnostics)
    return solver.q, diagnostics


def run_riemann_config3(config: RiemannConfig3):
    return run_riemann(config)


def run_riemann_config3_08(config: RiemannConfig3Offset08):
    return run_riemann(config)


def run_riemann_config6(config: RiemannConfig6):
    return run_riemann(config)


def riemann_config_dict(config: RiemannConfig3) -> dict:
    values = {"configuration_number": config.configuration_number, **asdict(config)}
    for attr in ("scenario_name", "configuration_label"):
        v = getattr(config, attr, None)
        if v is not None:
            values[attr] = v
    return values


def save_riemann_npz(path: Path, q, config: RiemannConfig3, diagnostics: RiemannDiagnostics) -> Path:
    """Same keys as riemann_config3.py:497-519."""
    rho, u, v, p = config.equation.primitive_from_conservative(q)
    omega = vorticity_z(q, config.domain, config.equation)
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(
        path, x=config.domain.x, y=config.domain.y, q=to_numpy(q), rho=to_numpy(rho),
        u=to_numpy(u), v=to_numpy(v), pressure=to_numpy(p), omega_z=to_numpy(omega),
        time=np.asarray(diagnostics.time), steps=np.asarray(diagnostics.steps),
        configuration_number=np.asarray(config.configuration_number),
        config_json=np.asarray(json.dumps(riemann_config_dict(config), default=str)),
        diagnostics_json=np.asarray(json.dumps(asdict(diagnostics), default=str)))
    return path


def load_riemann_npz(path: Path, config_class=RiemannConfig3):
    data = np.load(path, allow_pickle=False)
    cfg = json.loads(str(data["config_json"])) if "config_json" in data else {}
    fields = config_class.__dataclass_fields__
    return data, config_class(**{k: v for k, v in cfg.items()
                                 if k != "configuration_number" and k in fields})


def save_run_outputs(q, config: RiemannConfig3, diagnostics: RiemannDiagnostics, output_dir: Path,
                     run_id: str | None = None, plot: bool = False, **_plot_options) -> dict:
    """config.json, diagnostics.json and the final .npz (riemann_config3.py:756-809).
    Figures are produced by the reference's plotting scripts from the .npz."""
    run_id = run_id or make_run_id(f"riemann{config.configuration_number}")
    run_dir = Path(output_dir) / run_id
    run_dir.mkdir(parents=True, exist_ok=True)
    write_json(run_dir / "config.json", riemann_config_dict(config))
    write_json(run_dir / "diagnostics.json", asdict(diagnostics))
    npz = save_riemann_npz(run_dir / f"{run_id}_final.npz", q, config, diagnostics)
    return {"npz": npz}
