"""Forced 2-D compressible HIT on the B200 backend (OOP/hit2d.py).

Same configuration dataclass, initial condition, source functions, output
formats and CLI as the reference, with ``backend="b200"``.  The time loop
advances whole steps in the native library (dt, Mach control, OU forcing,
SSP-RK3 with rhs_with_forcing, hyperviscosity), keeping every control scalar
on the device; the host reads scalars only when it writes diagnostics,
snapshots or checks for the end of the run.
"""

from __future__ import annotations

import argparse
import ctypes
import math
import sys
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import torch

from . import _lib, core
from .backend import select_array_module, to_numpy
from .descs import grid_desc, precision_code, set_sensor
from .domain import Domain2D
from .equations import CompressibleNavierStokes2D, EulerEquation2D
from .run_utils import dataclass_to_json_dict, write_json
from .spatial_operator import PeriodicEulerShockSensor2D

DEFAULT_SNAPSHOT_DIR = Path("2D") / "hit2d_snapshots"
NOISE_MODES = ("numpy", "numpy-host", "device")


@dataclass(frozen=True)
class HIT2DConfig:
    """Fields and defaults of OOP/hit2d.py:36-80; ``backend`` defaults to
    "b200".  Additive fields: ``precision`` ("fp64" plain form or "fp32-bulk"),
    ``forcing_noise`` ("numpy": the reference's NumPy stream, continued on
    the device draw for draw; "numpy-host": the same stream drawn by NumPy on
    the host and uploaded each step; "device": shell noise drawn with a
    counter-based RNG on the device), ``max_steps`` (stop after this
    many steps even before tfinal) and ``initial_condition`` ("host": the
    reference's NumPy arithmetic, bit for bit; "device": the same phases,
    synthesised on the GPU, equal to roundoff)."""

    nx: int = 128
    ny: int = 128
    length: float = 2.0 * np.pi
    gamma: float = 1.4
    cfl: float = 0.05
    tfinal: float = 1.0
    target_mach: float = 0.1
    initial_kmin: int = 1
    initial_kmax: int = 3
    forcing_kmin: float | None = None
    forcing_kmax: float = 3.0
    forcing_rms: float = 1.0
    forcing_correlation_time: float = 1.0
    forcing_alpha_memory: float = 0.2
    target_energy_injection: float | None = 1.0e-3
    min_forcing_power: float = 1.0e-6
    max_forcing_rescale: float | None = 20.0
    mach_control: bool = False
    mach_control_target: float | None = None
    mach_control_memory: float = 0.995
    mach_control_exponent: float = 2.0
    mach_control_min_power: float | None = None
    mach_control_max_power: float | None = None
    forcing_seed: int = 1234
    viscosity: float = 1.0e-3
    prandtl: float = 0.72
    sensor_width: int = 4
    jump_threshold: float = 0.04
    compression_threshold: float = 2.5
    shear_threshold: float | None = None
    hyperviscosity_mn: float = 0.002
    hyperviscosity_interval: int = 5
    large_scale_drag: float = 0.0
    large_scale_drag_kmax: float = 2.0
    cooling_time: float | None = None
    cooling_target_pressure: float | None = None
    diagnostics_every: int = 25
    snapshot_every: int = 100
    forcing_anisotropy_warning: float = 0.2
    flow_anisotropy_warning: float = 0.4
    weno_fraction_warning: float = 0.5
    output_dir: Path = field(default_factory=lambda: DEFAULT_SNAPSHOT_DIR)
    backend: str = "b200"
    precision: str = "fp64"
    forcing_noise: str = "numpy"
    max_steps: int | None = None
    initial_condition: str = "host"

    @classmethod
    def isotropic_128(cls, output_dir: Path = DEFAULT_SNAPSHOT_DIR, backend: str = "b200"):
        """Recommended 128x128 annular-shell OU-forced HIT configuration."""
        return cls(nx=128, ny=128, tfinal=15.0, target_mach=0.25, initial_kmin=3, initial_kmax=5,
                   forcing_kmin=3.0, forcing_kmax=5.0, forcing_correlation_time=0.5,
                   forcing_alpha_memory=0.2, target_energy_injection=1.0e-3, viscosity=7.5e-4,
                   hyperviscosity_mn=0.002, large_scale_drag=0.10, large_scale_drag_kmax=2.0,
                   cooling_time=5.0, snapshot_every=75, diagnostics_every=25,
                   output_dir=output_dir, backend=backend)


def create_grid(config: HIT2DConfig):
    domain = Domain2D(0.0, config.length, 0.0, config.length, config.nx, config.ny)
    x_grid, y_grid = domain.mesh()
    return domain, x_grid, y_grid


def _wavenumbers(domain: Domain2D):
    kx = 2.0 * np.pi * np.fft.fftfreq(domain.nx, d=domain.dx)
    ky = 2.0 * np.pi * np.fft.fftfreq(domain.ny, d=domain.dy)
    return np.meshgrid(kx, ky, indexing="xy")


def initialize_hit_2d(config: HIT2DConfig, domain: Domain2D, equation, rng, xp=None):
    """Low-k streamfunction initial condition (OOP/hit2d.py:158-204).  Runs
    once on the host (NumPy) and is uploaded; returns a CUDA tensor."""
    X, Y = domain.mesh()
    psi = np.zeros_like(X)
    for kx in range(-config.initial_kmax, config.initial_kmax + 1):
        for ky in range(-config.initial_kmax, config.initial_kmax + 1):
            if ky < 0 or (ky == 0 and kx <= 0):
                continue
            magnitude = np.sqrt(kx ** 2 + ky ** 2)
            if magnitude < config.initial_kmin or magnitude > config.initial_kmax:
                continue
            phase = rng.uniform(0.0, 2.0 * np.pi)
            psi += (1.0 / max(kx ** 2 + ky ** 2, 1)) * np.cos(kx * X + ky * Y + phase)
    KX, KY = _wavenumbers(domain)
    ph = np.fft.fft2(psi)
    u = np.fft.ifft2(1j * KY * ph).real
    v = -np.fft.ifft2(1j * KX * ph).real
    u = u - np.mean(u)
    v = v - np.mean(v)
    rho = np.ones_like(u)
    p = np.full_like(u, 1.0 / config.gamma)
    c = np.sqrt(equation.gamma * p / rho)
    vrms = np.sqrt(np.mean(u ** 2 + v ** 2))
    if float(vrms) <= np.finfo(float).eps:
        raise ValueError("initial streamfunction produced zero velocity")
    scale = config.target_mach * float(np.mean(c)) / vrms
    u, v = u * scale, v * scale
    q = np.zeros((4,) + u.shape)
    q[0] = rho
    q[1] = rho * u
    q[2] = rho * v
    q[3] = p / (config.gamma - 1.0) + 0.5 * rho * (u ** 2 + v ** 2)
    return torch.from_numpy(q).cuda()


def initial_modes(config: HIT2DConfig, rng) -> np.ndarray:
    """(kx, ky, amplitude, phase) of every streamfunction mode of
    initialize_hit_2d (OOP/hit2d.py:175-189), in the reference's loop order,
    each phase drawn from ``rng`` as the reference draws it."""
    rows = []
    for kx in range(-config.initial_kmax, config.initial_kmax + 1):
        for ky in range(-config.initial_kmax, config.initial_kmax + 1):
            if ky < 0 or (ky == 0 and kx <= 0):
                continue
            magnitude = np.sqrt(kx ** 2 + ky ** 2)
            if magnitude < config.initial_kmin or magnitude > config.initial_kmax:
                continue
            rows.append((float(kx), float(ky), 1.0 / max(kx ** 2 + ky ** 2, 1),
                         rng.uniform(0.0, 2.0 * np.pi)))
    return np.asarray(rows, dtype=np.float64).reshape(-1, 4)


def initialize_hit_2d_device(config: HIT2DConfig, domain: Domain2D, equation, rng) -> torch.Tensor:
    """initialize_hit_2d (OOP/hit2d.py:158-204) built on the device: the
    phases come from ``rng`` on the host (a few dozen draws, the reference's
    stream), the streamfunction sum over modes and cells runs in
    ``hitb200_hit_streamfunction``, its spectral derivatives in the library's
    line transforms (``hitb200_hit_velocity``, the reference's fft2 / ifft2),
    and the mean removal,
    Mach scaling and conservative state in ``hitb200_hit_compose``.  Equal to
    the host form to roundoff (cos and the transforms are not NumPy's)."""
    core.require_cuda()
    lib = _lib.load()
    nx, ny = domain.nx, domain.ny
    modes = torch.from_numpy(initial_modes(config, rng)).cuda()
    psi = torch.empty((ny, nx), dtype=torch.float64, device="cuda")
    stream = core.stream_handle()
    _lib.check(lib.hitb200_hit_streamfunction(modes.data_ptr(), modes.shape[0], nx, ny,
                                              float(domain.x_min), float(domain.dx),
                                              float(domain.y_min), float(domain.dy),
                                              psi.data_ptr(), stream))
    u = torch.empty_like(psi)
    v = torch.empty_like(psi)
    wsv = torch.empty(int(lib.hitb200_hit_velocity_workspace_bytes(nx, ny)), dtype=torch.uint8,
                      device="cuda")
    _lib.check(lib.hitb200_hit_velocity(psi.data_ptr(), nx, ny, float(domain.dx), float(domain.dy),
                                        u.data_ptr(), v.data_ptr(), wsv.data_ptr(), wsv.numel(),
                                        stream))
    # mean sound speed of rho = 1, p = 1/gamma as NumPy forms it (a constant field)
    p = np.full((ny, nx), 1.0 / config.gamma)
    c_mean = float(np.mean(np.sqrt(equation.gamma * p / np.ones_like(p))))
    q = torch.empty((4, ny, nx), dtype=torch.float64, device="cuda")
    vrms = torch.empty(1, dtype=torch.float64, device="cuda")
    ws = torch.empty(int(lib.hitb200_hit_compose_workspace_bytes()), dtype=torch.uint8,
                     device="cuda")
    _lib.check(lib.hitb200_hit_compose(u.data_ptr(), v.data_ptr(), nx, ny, float(config.gamma),
                                       float(config.target_mach), c_mean, q.data_ptr(),
                                       vrms.data_ptr(), ws.data_ptr(), ws.numel(), stream))
    if float(vrms.item()) <= np.finfo(float).eps:
        raise ValueError("initial streamfunction produced zero velocity")
    return q


def _source_plan(q, equation, domain: Domain2D | None = None, **kw) -> core.Plan:
    ny, nx = q.shape[1:]
    dom = domain or Domain2D(0.0, 2.0 * np.pi, 0.0, 2.0 * np.pi, nx, ny)
    d = grid_desc(dom, equation.gamma, True)
    for k, v in kw.items():
        setattr(d, k, v)
    return core.plan_for(d)


def forcing_source(q, equation, fx, fy):
    """[0, rho fx, rho fy, rho (u fx + v fy)] (OOP/hit2d.py:264-276)."""
    q = core.as_state(q)
    fx = core.as_field(fx, q.shape[1:], "fx")
    fy = core.as_field(fy, q.shape[1:], "fy")
    return _source_plan(q, equation).rhs(q, _lib.TERM_FORCING, fx, fy)


def large_scale_drag_source(q, equation, domain: Domain2D, coefficient: float, kmax: float):
    """Linear drag on |k| <= kmax momentum fluctuations (OOP/hit2d.py:370-399)."""
    q = core.as_state(q)
    if coefficient <= 0.0 or kmax <= 0.0:
        return torch.zeros_like(q)
    plan = _source_plan(q, equation, domain, drag_coefficient=float(coefficient),
                        drag_kmax=float(kmax))
    return plan.rhs(q, _lib.TERM_DRAG)


def cooling_source(q, equation, cooling_time, target_pressure=None):
    """Uniform mean-pressure relaxation (OOP/hit2d.py:402-426)."""
    q = core.as_state(q)
    if cooling_time is None or cooling_time <= 0.0:
        return torch.zeros_like(q)
    plan = _source_plan(q, equation, cooling_time=float(cooling_time),
                        cooling_target_pressure=_lib.none_to_nan(target_pressure))
    return plan.rhs(q, _lib.TERM_COOLING)


def turbulent_mach_from_primitive(rho, u, v, pressure, gamma) -> float:
    c = torch.sqrt(gamma * pressure / rho)
    return float(torch.sqrt(torch.mean(u ** 2 + v ** 2)) / torch.mean(c))


def update_mach_controlled_power(config, current_power, rho, u, v, pressure):
    """Host form of the Mach feedback (OOP/hit2d.py:293-349); the fused step
    runs the same logic on the device."""
    target_power = current_power
    target_mach = config.target_mach if config.mach_control_target is None else config.mach_control_target
    current_mach = turbulent_mach_from_primitive(rho, u, v, pressure, config.gamma)
    desired_power = math.nan if target_power is None else float(target_power)
    info = {"mach_control_mach": current_mach, "mach_control_target": float(target_mach),
            "mach_control_power_desired": desired_power}
    if not config.mach_control or target_power is None:
        return target_power, info
    if target_mach <= 0.0:
        raise ValueError("Mach control requires a positive target Mach number")
    if not 0.0 <= config.mach_control_memory < 1.0:
        raise ValueError("mach_control_memory must be in [0, 1)")
    if config.mach_control_exponent <= 0.0:
        raise ValueError("mach_control_exponent must be positive")
    ratio = (target_mach / max(current_mach, 1.0e-8)) ** config.mach_control_exponent
    desired_power = float(target_power * ratio)
    if config.mach_control_min_power is not None:
        desired_power = max(desired_power, config.mach_control_min_power)
    if config.mach_control_max_power is not None:
        desired_power = min(desired_power, config.mach_control_max_power)
    next_power = (config.mach_control_memory * target_power
                  + (1.0 - config.mach_control_memory) * desired_power)
    info["mach_control_power_desired"] = desired_power
    return next_power, info


def spectral_diagnostics(q, equation, domain: Domain2D, kmax: float = 0.0, fields: bool = False,
                         plan: core.Plan | None = None):
    """Spectral divergence and vorticity rms (OOP/hit2d.py:146-155, 459-468)
    and the low-k kinetic fraction for 0 < |k| <= kmax (:429-449) of the
    state q, by the library's own line transforms
    (hitb200_spectral_diagnostics).  Returns (div_rms, vort_rms, k_low) and,
    with ``fields``, the divergence and vorticity fields."""
    q = core.as_state(q)
    ny, nx = q.shape[1:]
    if plan is None:
        plan = core.plan_for(grid_desc(domain, equation.gamma, True))
    lib = plan.lib
    ws = torch.empty(int(lib.hitb200_spectral_workspace_bytes(nx, ny)), dtype=torch.uint8,
                     device=q.device)
    div = vort = None
    if fields:
        div = torch.empty((ny, nx), dtype=torch.float64, device=q.device)
        vort = torch.empty_like(div)
    out = (ctypes.c_double * 3)()
    _lib.check(lib.hitb200_spectral_diagnostics(
        plan.handle, q.data_ptr(), float(kmax), out, core.ptr(div), core.ptr(vort), ws.data_ptr(),
        ws.numel(), core.stream_handle()))
    res = (out[0], out[1], out[2])
    return (res, div, vort) if fields else res


def divergence_and_vorticity(u, v, domain: Domain2D):
    """Spectral divergence and vorticity fields (OOP/hit2d.py:459-468) of the
    velocity (u, v): the state [1, u, v, 1] through spectral_diagnostics
    (its velocity is u, v exactly)."""
    u = core.as_field(u, (domain.ny, domain.nx), "u")
    v = core.as_field(v, (domain.ny, domain.nx), "v")
    q = torch.stack([torch.ones_like(u), u, v, torch.ones_like(u)]).contiguous()
    _, div, vort = spectral_diagnostics(q, EulerEquation2D(gamma=1.4), domain, fields=True)
    return div, vort


def large_scale_kinetic_fraction(q, equation, domain: Domain2D, kmax: float) -> float:
    """Fraction of the kinetic energy of the velocity fluctuations in the band
    0 < |k| <= kmax (OOP/hit2d.py:429-449)."""
    if kmax <= 0.0:
        return 0.0
    return spectral_diagnostics(q, equation, domain, kmax)[2]


def source_power(source) -> float:
    return float(torch.mean(source[3]))


_DIAG_KEYS = ["kinetic_energy", "Kx", "Ky", "A_K", "C_uv", "rms_velocity", "turbulent_mach",
              "mean_density", "mean_pressure", "mass"]


def compute_diagnostics(q, equation, domain: Domain2D, initial_mass=None, forcing_info=None,
                        drag_power=0.0, cooling_power=0.0, large_scale_fraction=0.0,
                        weno_fraction=0.0, plan: core.Plan | None = None):
    """Scalar diagnostics with the keys of OOP/hit2d.py:471-548.  The moment
    sums run in the native diagnostics reduction; divergence and vorticity are
    spectral as in the reference."""
    q = core.as_state(q)
    if plan is None:
        plan = core.plan_for(grid_desc(domain, equation.gamma, True))
    vals = plan.diagnostics(q)
    d = dict(zip(_DIAG_KEYS, vals[:10]))
    d["mass"] = vals[9]
    div_rms, vort_rms, _ = spectral_diagnostics(q, equation, domain, plan=plan)
    diagnostics = {
        "kinetic_energy": d["kinetic_energy"], "Kx": d["Kx"], "Ky": d["Ky"], "A_K": d["A_K"],
        "C_uv": d["C_uv"], "rms_velocity": d["rms_velocity"],
        "turbulent_mach": d["turbulent_mach"], "mean_density": d["mean_density"],
        "mean_pressure": d["mean_pressure"],
        "divergence_rms": div_rms,
        "vorticity_rms": vort_rms,
        "mass": d["mass"],
        "mass_error": 0.0 if initial_mass is None else d["mass"] - initial_mass,
        "large_scale_kinetic_fraction": large_scale_fraction,
        "drag_power": drag_power, "cooling_power": cooling_power,
        "weno_fraction": weno_fraction,
    }
    diagnostics.update({"P_in": 0.0, "Fxx": 0.0, "Fyy": 0.0, "Fxy": 0.0, "A_F": 0.0,
                        "forcing_alpha": 0.0, "forcing_target_power": 0.0,
                        "mach_control_mach": diagnostics["turbulent_mach"],
                        "mach_control_target": 0.0, "mach_control_power_desired": 0.0})
    if forcing_info is not None:
        diagnostics.update({
            "P_in": forcing_info["injected_power"], "Fxx": forcing_info["Fxx"],
            "Fyy": forcing_info["Fyy"], "Fxy": forcing_info["Fxy"], "A_F": forcing_info["A_F"],
            "forcing_alpha": forcing_info["alpha"],
            "forcing_target_power": forcing_info.get("target_power", 0.0),
            "mach_control_mach": forcing_info.get("mach_control_mach", diagnostics["turbulent_mach"]),
            "mach_control_target": forcing_info.get("mach_control_target", 0.0),
            "mach_control_power_desired": forcing_info.get("mach_control_power_desired", 0.0)})
    return diagnostics


def save_run_config(output_dir: Path, config: HIT2DConfig) -> Path:
    payload = dataclass_to_json_dict(config)
    forcing_type = "disabled" if config.forcing_rms <= 0.0 else "solenoidal_shell_ou"
    payload.update({"problem": "hit2d", "forcing_type": forcing_type,
                    "spatial_discretization": "hybrid_compact_weno7",
                    "hyperviscosity_policy": "compact_nodes_only"})
    return write_json(Path(output_dir) / "config.json", payload)


def save_snapshot(output_dir: Path, step: int, time: float, q, equation, domain: Domain2D) -> Path:
    q = core.as_state(q)
    rho, u, v, p = equation.primitive_from_conservative(q)
    _, div, vort = spectral_diagnostics(q, equation, domain, fields=True)
    output_dir = Path(output_dir)
    output_dir.mkdir(parents=True, exist_ok=True)
    path = output_dir / f"hit2d_step{step:07d}.npz"
    np.savez_compressed(path, step=step, time=time, x=domain.x, y=domain.y, rho=to_numpy(rho),
                        u=to_numpy(u), v=to_numpy(v), pressure=to_numpy(p),
                        vorticity=to_numpy(vort), divergence=to_numpy(div))
    return path


def save_diagnostic_history(output_dir: Path, history, config: HIT2DConfig) -> Path:
    output_dir = Path(output_dir)
    output_dir.mkdir(parents=True, exist_ok=True)
    path = output_dir / "diagnostic_history.npz"
    keys = tuple(history[0])
    data = {key: np.asarray([record[key] for record in history]) for key in keys}
    nan = np.nan

    def opt(v):
        return np.asarray(nan if v is None else v)

    data.update({
        "forcing_kmin": np.asarray(0.0 if config.forcing_kmin is None else config.forcing_kmin),
        "forcing_kmax": np.asarray(config.forcing_kmax),
        "forcing_correlation_time": np.asarray(config.forcing_correlation_time),
        "large_scale_drag": np.asarray(config.large_scale_drag),
        "large_scale_drag_kmax": np.asarray(config.large_scale_drag_kmax),
        "cooling_time": opt(config.cooling_time),
        "cooling_target_pressure": opt(config.cooling_target_pressure),
        "target_energy_injection": opt(config.target_energy_injection),
        "mach_control": np.asarray(config.mach_control),
        "mach_control_target": opt(config.mach_control_target),
        "mach_control_memory": np.asarray(config.mach_control_memory),
        "mach_control_exponent": np.asarray(config.mach_control_exponent),
        "mach_control_min_power": opt(config.mach_control_min_power),
        "mach_control_max_power": opt(config.mach_control_max_power),
    })
    np.savez_compressed(path, **data)
    return path


def _make_equation(config: HIT2DConfig):
    if config.viscosity > 0.0:
        return CompressibleNavierStokes2D(gamma=config.gamma, viscosity=config.viscosity,
                                          prandtl=config.prandtl)
    return EulerEquation2D(gamma=config.gamma)


def hit_descriptor(config: HIT2DConfig, domain: Domain2D) -> _lib.Desc:
    """Native descriptor of a whole HIT run (every term of rhs_with_forcing)."""
    d = grid_desc(domain, config.gamma, True, config.precision)
    set_sensor(d, config.sensor_width, config.compression_threshold, config.jump_threshold,
               config.shear_threshold)
    d.viscosity, d.prandtl = config.viscosity, config.prandtl
    d.hv_mn = config.hyperviscosity_mn
    d.hv_interval = config.hyperviscosity_interval if config.hyperviscosity_mn > 0.0 else 0
    for i, w in enumerate((0.25, 1.0, 1.0, 0.25)):
        d.hv_weight[i] = w
    d.drag_coefficient, d.drag_kmax = config.large_scale_drag, config.large_scale_drag_kmax
    d.cooling_time = _lib.none_to_nan(config.cooling_time)
    d.cooling_target_pressure = _lib.none_to_nan(config.cooling_target_pressure)
    d.forcing_on = 1
    d.forcing_kmin = 0.0 if config.forcing_kmin is None else float(config.forcing_kmin)
    d.forcing_kmax = float(config.forcing_kmax)
    d.forcing_correlation_time = config.forcing_correlation_time
    d.forcing_rms = config.forcing_rms
    d.target_power = _lib.none_to_nan(config.target_energy_injection)
    d.min_power = config.min_forcing_power
    d.max_rescale = _lib.none_to_nan(config.max_forcing_rescale)
    d.alpha_memory = config.forcing_alpha_memory
    d.mach_control = 1 if config.mach_control else 0
    d.mach_target = config.target_mach if config.mach_control_target is None else config.mach_control_target
    d.mach_memory = config.mach_control_memory
    d.mach_exponent = config.mach_control_exponent
    d.mach_min_power = _lib.none_to_nan(config.mach_control_min_power)
    d.mach_max_power = _lib.none_to_nan(config.mach_control_max_power)
    d.cfl, d.tfinal = config.cfl, config.tfinal
    d.fixed_dt = 0
    d.noise_mode = {"numpy": 2, "numpy-host": 0, "device": 1}[config.forcing_noise]
    d.seed = int(config.forcing_seed) + 1
    return d


def _print_diagnostics(step, time, dt, d):
    print(f"step={step:6d}, t={time:.6f}, dt={dt:.3e}, KE={d['kinetic_energy']:.6e}, "
          f"Mt={d['turbulent_mach']:.4f}, A_K={d['A_K']:.3f}, Cuv={d['C_uv']:.3f}, "
          f"P_in={d['P_in']:.3e}, P_tgt={d['forcing_target_power']:.3e}, A_F={d['A_F']:.3f}, "
          f"K_low={d['large_scale_kinetic_fraction']:.3f}, P_drag={d['drag_power']:.3e}, "
          f"P_cool={d['cooling_power']:.3e}, WENO={d['weno_fraction']:.3f}, "
          f"rho_mean={d['mean_density']:.6f}, p_mean={d['mean_pressure']:.6f}, "
          f"div_rms={d['divergence_rms']:.3e}, vort_rms={d['vorticity_rms']:.3e}, "
          f"mass_err={d['mass_error']:.3e}")


def _warn_diagnostic_state(diagnostics, history, config) -> None:
    if not all(np.isfinite(value) for value in diagnostics.values()):
        raise FloatingPointError("NaN or infinite value detected in HIT2D diagnostics")
    if history:
        fxx = float(np.mean([h["Fxx"] for h in history]))
        fyy = float(np.mean([h["Fyy"] for h in history]))
        fxy = float(np.mean([h["Fxy"] for h in history]))
        s = fxx + fyy
        caf = abs(fxx - fyy) / s if s > 0.0 else 0.0
        nfxy = abs(fxy) / s if s > 0.0 else 0.0
        if caf > config.forcing_anisotropy_warning:
            print(f"warning: cumulative forcing anisotropy is high (A_F={caf:.3f})")
        if nfxy > 0.1:
            print("warning: cumulative forcing cross-correlation is high "
                  f"(|Fxy|/(Fxx+Fyy)={nfxy:.3f})")
    if diagnostics["A_K"] > config.flow_anisotropy_warning:
        print(f"warning: flow component anisotropy is high (A_K={diagnostics['A_K']:.3f})")
    if len(history) >= 3:
        r = [h["A_K"] for h in history[-3:]]
        if r[0] < r[1] < r[2] and r[-1] > 0.2:
            print("warning: flow component anisotropy has increased over the last three "
                  "diagnostic samples")
    if diagnostics["weno_fraction"] > config.weno_fraction_warning:
        print(f"warning: WENO is active over a large domain fraction ({diagnostics['weno_fraction']:.3f})")
    if diagnostics["large_scale_kinetic_fraction"] > 0.35 and config.large_scale_drag <= 0.0:
        print("warning: a large fraction of kinetic energy is in low-k modes "
              f"(K_low={diagnostics['large_scale_kinetic_fraction']:.3f}); "
              "consider enabling --large-scale-drag")


def _forcing_info(s, config) -> dict:
    target = s[_lib.S_POWER]
    return {"alpha": s[_lib.S_F_ALPHA], "alpha_target": s[_lib.S_F_ALPHA_TARGET],
            "target_power": target, "power_before_rescale": s[_lib.S_F_POWER_BEFORE],
            "injected_power": s[_lib.S_F_INJECTED], "Fxx": s[_lib.S_F_FXX],
            "Fyy": s[_lib.S_F_FYY], "Fxy": s[_lib.S_F_FXY], "A_F": s[_lib.S_F_AF],
            "ou_decay": s[_lib.S_F_DECAY], "mach_control_mach": s[_lib.S_MACH],
            "mach_control_target": float(config.target_mach if config.mach_control_target is None
                                         else config.mach_control_target),
            "mach_control_power_desired": s[_lib.S_POWER_DESIRED]}


class HITSolver:
    """A resident HIT solve: state on the device, steps advanced natively."""

    def __init__(self, config: HIT2DConfig):
        if config.hyperviscosity_interval <= 0 and config.hyperviscosity_mn > 0.0:
            raise ValueError("hyperviscosity_interval must be positive when mn > 0")
        select_array_module(config.backend)
        precision_code(config.precision)
        if config.forcing_noise not in NOISE_MODES:
            raise ValueError(f"forcing_noise must be one of {NOISE_MODES}")
        if config.initial_condition not in ("host", "device"):
            raise ValueError("initial_condition must be 'host' or 'device'")
        self.config = config
        self.domain = create_grid(config)[0]
        self.equation = _make_equation(config)
        self.plan = core.Plan(hit_descriptor(config, self.domain))
        rng = np.random.default_rng(config.forcing_seed)
        self.noise_rng = np.random.default_rng(config.forcing_seed + 1)
        init = initialize_hit_2d_device if config.initial_condition == "device" else initialize_hit_2d
        q = init(config, self.domain, self.equation, rng)
        self.q = self.equation.enforce_physical_state(q)
        self.plan.set_time(0.0, 0, 0.0, -1 if config.max_steps is None else config.max_steps)
        if config.forcing_noise == "numpy":
            # the reference's stream (default_rng(seed + 1), OOP/hit2d.py:791-803),
            # continued on the device draw for draw
            self.plan.set_noise_stream(self.noise_rng.bit_generator.state)
        if config.forcing_noise == "numpy-host":
            self._noise_dev = torch.empty((config.ny, config.nx), dtype=torch.float64, device="cuda")
            self._noise_host = torch.empty((config.ny, config.nx), dtype=torch.float64).pin_memory()

    def advance(self, nsteps: int) -> None:
        """Issue nsteps steps; steps past tfinal / max_steps are device no-ops."""
        if self.config.forcing_noise == "numpy-host":
            for _ in range(nsteps):
                self._noise_host.numpy()[...] = self.noise_rng.standard_normal(
                    (self.config.ny, self.config.nx))
                self._noise_dev.copy_(self._noise_host, non_blocking=True)
                self.plan.step(self.q, self._noise_dev)
                torch.cuda.current_stream().synchronize()  # host buffer reused next step
        else:
            self.plan.run(self.q, nsteps)

    def scalars(self) -> list[float]:
        return self.plan.scalars()

    def checkpoint(self) -> dict:
        """Everything the solve carries from one step to the next: the state,
        the plan's scalar block (time, step, Mach-control and forcing state,
        OU potential) and, with the reference's noise stream, that stream's
        position.  ``restore`` on a solver of the same configuration resumes
        the run bit for bit."""
        torch.cuda.synchronize()
        ck = {"q": self.q.detach().cpu().clone(), "block": self.plan.save_state_block()}
        if self.config.forcing_noise == "numpy-host":
            ck["noise_rng"] = self.noise_rng.bit_generator.state
        return ck

    def restore(self, ck: dict) -> None:
        if tuple(ck["q"].shape) != tuple(self.q.shape):
            raise ValueError("checkpoint state does not match the solver's grid")
        self.q.copy_(ck["q"])
        self.plan.load_state_block(ck["block"])
        if "noise_rng" in ck:
            self.noise_rng.bit_generator.state = ck["noise_rng"]


def as_config(config) -> HIT2DConfig:
    """The mirror's HIT2DConfig for a configuration object of the reference
    (``OOP.hit2d.HIT2DConfig`` with ``backend="b200"``, handed over by the
    reference's run_simulation): its fields copied, the mirror's own fields at
    their defaults."""
    if isinstance(config, HIT2DConfig):
        return config
    from dataclasses import fields

    names = {f.name for f in fields(HIT2DConfig)}
    return HIT2DConfig(**{k: getattr(config, k) for k in names if hasattr(config, k)})


def run_simulation(config: HIT2DConfig):
    """Driver of OOP/hit2d.py:764-918 on the B200 backend.  Returns (q, t, steps)."""
    config = as_config(config)
    select_array_module(config.backend)
    print("Using array backend: b200")
    if config.hyperviscosity_interval <= 0 and config.hyperviscosity_mn > 0.0:
        raise ValueError("hyperviscosity_interval must be positive when mn > 0")
    config_path = save_run_config(config.output_dir, config)
    print(f"saved run configuration: {config_path}")
    solver = HITSolver(config)
    domain, equation, plan = solver.domain, solver.equation, solver.plan
    sensor = PeriodicEulerShockSensor2D(domain, equation, width=config.sensor_width,
                                        compression_threshold=config.compression_threshold,
                                        jump_threshold=config.jump_threshold,
                                        shear_threshold=config.shear_threshold)
    q = solver.q
    weno0 = float(sensor.detect(q).double().mean())
    diag0 = compute_diagnostics(q, equation, domain, large_scale_fraction=large_scale_kinetic_fraction(
        q, equation, domain, config.large_scale_drag_kmax), weno_fraction=weno0, plan=plan)
    initial_mass = diag0["mass"]
    history = [{"step": 0.0, "time": 0.0, "dt": 0.0, **diag0}]
    save_snapshot(config.output_dir, 0, 0.0, q, equation, domain)
    save_diagnostic_history(config.output_dir, history, config)
    _print_diagnostics(0, 0.0, 0.0, diag0)
    every = math.gcd(max(config.diagnostics_every, 1), max(config.snapshot_every, 1))
    chunk = max(1, min(every, 64))
    step, time = 0, 0.0
    while True:
        solver.advance(chunk)
        s = solver.scalars()
        _lib.check_step_status(s[_lib.S_STATUS], "HIT2D state")
        new_step, time, dt = int(s[_lib.S_STEP]), s[_lib.S_TIME], s[_lib.S_DT]
        progressed = new_step > step
        step = new_step
        finished = time >= config.tfinal or (config.max_steps is not None and step >= config.max_steps)
        if progressed and (step % config.diagnostics_every == 0 or finished):
            weno = float(sensor.detect(q).double().mean())
            drag = large_scale_drag_source(q, equation, domain, config.large_scale_drag,
                                           config.large_scale_drag_kmax)
            cool = cooling_source(q, equation, config.cooling_time, config.cooling_target_pressure)
            d = compute_diagnostics(q, equation, domain, initial_mass=initial_mass,
                                    forcing_info=_forcing_info(s, config),
                                    drag_power=source_power(drag), cooling_power=source_power(cool),
                                    large_scale_fraction=large_scale_kinetic_fraction(
                                        q, equation, domain, config.large_scale_drag_kmax),
                                    weno_fraction=weno, plan=plan)
            history.append({"step": float(step), "time": time, "dt": dt, **d})
            _warn_diagnostic_state(d, history[1:], config)
            save_diagnostic_history(config.output_dir, history, config)
            _print_diagnostics(step, time, dt, d)
        if progressed and (step % config.snapshot_every == 0 or finished):
            path = save_snapshot(config.output_dir, step, time, q, equation, domain)
            print(f"saved snapshot: {path}")
        if finished or not progressed:
            break
    return q, time, step


def parse_args(argv=None) -> argparse.Namespace:
    p = argparse.ArgumentParser(description="2D forced compressible HIT on the B200 backend.")
    p.add_argument("--nx", type=int, default=128)
    p.add_argument("--ny", type=int, default=128)
    p.add_argument("--tfinal", type=float, default=1.0)
    p.add_argument("--cfl", type=float, default=0.05)
    p.add_argument("--mach", type=float, default=0.1)
    p.add_argument("--initial-kmin", type=int, default=1)
    p.add_argument("--initial-kmax", type=int, default=3)
    p.add_argument("--gamma", type=float, default=1.4)
    p.add_argument("--viscosity", type=float, default=1.0e-3)
    p.add_argument("--kf", type=float, default=3.0)
    p.add_argument("--kf-min", type=float, default=None)
    p.add_argument("--kf-max", type=float, default=None)
    p.add_argument("--p-target", "--pget", dest="p_target", type=float, default=1.0e-3)
    p.add_argument("--force-rms", type=float, default=1.0)
    p.add_argument("--forcing-correlation-time", type=float, default=1.0)
    p.add_argument("--forcing-alpha-memory", type=float, default=0.2)
    p.add_argument("--min-forcing-power", type=float, default=1.0e-6)
    p.add_argument("--max-forcing-rescale", type=float, default=20.0)
    p.add_argument("--mach-control", action="store_true")
    p.add_argument("--mach-control-target", type=float, default=None)
    p.add_argument("--mach-control-memory", type=float, default=0.995)
    p.add_argument("--mach-control-exponent", type=float, default=2.0)
    p.add_argument("--mach-control-min-power", type=float, default=0.0)
    p.add_argument("--mach-control-max-power", type=float, default=0.0)
    p.add_argument("--seed", type=int, default=1234)
    p.add_argument("--mn", type=float, default=0.002)
    p.add_argument("--large-scale-drag", type=float, default=0.0)
    p.add_argument("--drag-kmax", type=float, default=2.0)
    p.add_argument("--cooling-time", type=float, default=0.0)
    p.add_argument("--cooling-target-pressure", type=float, default=None)
    p.add_argument("--diagnostics-every", type=int, default=25)
    p.add_argument("--snapshot-every", type=int, default=100)
    p.add_argument("--output-dir", type=Path, default=DEFAULT_SNAPSHOT_DIR)
    p.add_argument("--backend", choices=("auto", "numpy", "cupy", "b200"), default="b200")
    p.add_argument("--no-forcing", action="store_true")
    p.add_argument("--precision", choices=("fp64", "fp32-bulk"), default="fp64")
    p.add_argument("--forcing-noise", choices=NOISE_MODES, default="numpy")
    p.add_argument("--max-steps", type=int, default=None)
    return p.parse_args(argv)


def config_from_args(a: argparse.Namespace) -> HIT2DConfig:
    """CLI to config, with the reference's 0-means-off conventions
    (OOP/hit2d.py:1042-1082)."""
    return HIT2DConfig(
        nx=a.nx, ny=a.ny, tfinal=a.tfinal, cfl=a.cfl, target_mach=a.mach,
        initial_kmin=a.initial_kmin, initial_kmax=a.initial_kmax, gamma=a.gamma,
        viscosity=a.viscosity, forcing_kmin=a.kf_min,
        forcing_kmax=a.kf if a.kf_max is None else a.kf_max,
        forcing_rms=0.0 if a.no_forcing else a.force_rms,
        forcing_correlation_time=a.forcing_correlation_time,
        forcing_alpha_memory=a.forcing_alpha_memory,
        target_energy_injection=None if a.no_forcing else a.p_target,
        min_forcing_power=a.min_forcing_power,
        max_forcing_rescale=None if a.max_forcing_rescale == 0.0 else a.max_forcing_rescale,
        mach_control=False if a.no_forcing else a.mach_control,
        mach_control_target=a.mach_control_target, mach_control_memory=a.mach_control_memory,
        mach_control_exponent=a.mach_control_exponent,
        mach_control_min_power=None if a.mach_control_min_power == 0.0 else a.mach_control_min_power,
        mach_control_max_power=None if a.mach_control_max_power == 0.0 else a.mach_control_max_power,
        forcing_seed=a.seed, hyperviscosity_mn=a.mn, large_scale_drag=a.large_scale_drag,
        large_scale_drag_kmax=a.drag_kmax,
        cooling_time=None if a.cooling_time <= 0.0 else a.cooling_time,
        cooling_target_pressure=a.cooling_target_pressure, diagnostics_every=a.diagnostics_every,
        snapshot_every=a.snapshot_every, output_dir=a.output_dir, backend=a.backend,
        precision=a.precision, forcing_noise=a.forcing_noise, max_steps=a.max_steps)


def main(argv=None) -> None:
    config = config_from_args(parse_args(argv))
    _q, time, steps = run_simulation(config)
    print(f"completed 2D HIT run at t={time:.6f} in {steps} steps")


if __name__ == "__main__":
    main(sys.argv[1:])
