"""Generate golden vectors by running the reference HIT_Solver itself.

Run once, in a container where the reference source tree is available:

    python tests/golden/make_golden.py <reference-root>

It imports the reference package ``OOP`` (with a placeholder ``matplotlib``
from ``_stubs/``, since plotting is never exercised), evaluates the reference's
own hot-path functions on small seeded states, and writes the inputs and
outputs to ``tests/golden/*.npz``.  The fixtures are committed; neither the
tests nor the product read the reference tree at run time.
"""

from __future__ import annotations

import contextlib
import io
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _import_reference(root: str):
    sys.path.insert(0, str(HERE / "_stubs"))
    sys.path.insert(0, root)
    from OOP.domain import Domain2D
    from OOP.equations import CompressibleNavierStokes2D, EulerEquation2D
    from OOP.forcing import IsotropicShellOUForcing2D
    from OOP import hit2d
    from OOP.spatial_operator import (PeriodicEulerShockSensor2D,
                                      PeriodicHybridEuler2DOperator,
                                      PeriodicHyperviscosity2D)
    from OOP.time_operator import SSPRK3
    from OOP.problems import riemann_config3 as rc3
    from OOP.problems.riemann_config6 import RiemannConfig6
    from OOP.problems.riemann_config3_08 import RiemannConfig3Offset08
    return dict(Domain2D=Domain2D, NS=CompressibleNavierStokes2D, Euler=EulerEquation2D,
                OU=IsotropicShellOUForcing2D, hit2d=hit2d, PSensor=PeriodicEulerShockSensor2D,
                POp=PeriodicHybridEuler2DOperator, PHv=PeriodicHyperviscosity2D,
                SSPRK3=SSPRK3, rc3=rc3, RC6=RiemannConfig6, RC308=RiemannConfig3Offset08)


def periodic_cases(R):
    """Periodic (HIT) states: the reference's HIT initial condition on a
    non-square grid, and the same flow with a density/pressure blob so the jump
    part of the sensor fires."""
    hit2d = R["hit2d"]
    out = {}
    for name, nx, ny, blob in (("hit_32x24", 32, 24, False), ("blob_40x36", 40, 36, True)):
        cfg = hit2d.HIT2DConfig(nx=nx, ny=ny, target_mach=0.25, initial_kmin=3, initial_kmax=5,
                                backend="numpy", output_dir=Path(tempfile.mkdtemp()))
        domain, X, Y = hit2d.create_grid(cfg)
        eq = R["NS"](gamma=1.4, viscosity=1e-3, prandtl=0.72)
        rng = np.random.default_rng(1234)
        q = eq.enforce_physical_state(hit2d.initialize_hit_2d(cfg, domain, eq, rng))
        if blob:
            rho, u, v, p = eq.primitive_from_conservative(q)
            r2 = (X - 2.0) ** 2 + (Y - 3.5) ** 2
            inside = r2 < 1.0
            rho = np.where(inside, 1.6, rho)
            p = np.where(inside, 1.4, p)
            q = eq.enforce_physical_state(eq.conservative_from_primitive(rho, u, v, p))
        out[name] = (cfg, domain, eq, q)
    return out


def gen_periodic(R, name, cfg, domain, eq, q):
    hit2d = R["hit2d"]
    sensor = R["PSensor"](domain, eq, width=4, compression_threshold=2.5, jump_threshold=0.04,
                          shear_threshold=None)
    sensor_shear = R["PSensor"](domain, eq, width=3, compression_threshold=2.5,
                                jump_threshold=0.04, shear_threshold=1.5)
    op = R["POp"](domain, eq, sensor)
    hv = R["PHv"](domain, mn=0.002)
    qs = eq.enforce_physical_state(q)
    mask = sensor.detect(qs)
    d_x = op._axis_derivative(qs, eq.flux_x(qs), mask, op.compact_x, normal_velocity_index=1)
    qy = np.moveaxis(qs, -2, -1)
    d_y = np.moveaxis(op._axis_derivative(qy, np.moveaxis(eq.flux_y(qs), -2, -1), mask.T,
                                          op.compact_y, normal_velocity_index=2), -1, -2)
    rng = np.random.default_rng(7)
    fx = 0.3 * rng.standard_normal(q.shape[1:])
    fy = 0.3 * rng.standard_normal(q.shape[1:])
    visc = eq.viscous_rhs(q, domain.dx, domain.dy)
    drag = hit2d.large_scale_drag_source(q, eq, domain, 0.1, 2.0)
    cool = hit2d.cooling_source(q, eq, 5.0, None)
    fsrc = hit2d.forcing_source(q, eq, fx, fy)
    dt = op.stable_time_step(q, 0.05, 1.0)

    def rhs_full(s):
        r = op.rhs(s) + eq.viscous_rhs(s, domain.dx, domain.dy)
        r = r + hit2d.forcing_source(s, eq, fx, fy)
        r = r + hit2d.large_scale_drag_source(s, eq, domain, 0.1, 2.0)
        return r + hit2d.cooling_source(s, eq, 5.0, None)

    step = R["SSPRK3"]().step(q, rhs_full, dt, clean=eq.enforce_physical_state)
    hvq = hv.apply(q, eq, active_mask=~mask)
    # three consecutive OU forcing updates from the reference's own RNG
    forcing = R["OU"](domain=domain, k_min=3.0, k_max=5.0, correlation_time=0.5, force_rms=1.0,
                      target_power=1e-3, min_power=1e-6, max_rescale=20.0, alpha_memory=0.2,
                      seed=1235)
    rho, u, v, p = eq.primitive_from_conservative(q)
    f_out = {}
    for k in range(3):
        fxk, fyk, info = forcing.update(dt * (1.0 + 0.1 * k), rho, u, v)
        f_out[f"forcing{k}_fx"] = fxk
        f_out[f"forcing{k}_fy"] = fyk
        for key, val in info.items():
            f_out[f"forcing{k}_info_{key}"] = np.asarray(val)
    diag = hit2d.compute_diagnostics(q, eq, domain)
    klow = {f"klow_{k:g}": np.asarray(hit2d.large_scale_kinetic_fraction(q, eq, domain, k))
            for k in (1.0, 2.0, 3.5)}
    np.savez_compressed(
        HERE / f"periodic_{name}.npz",
        q=q, mask=mask, mask_shear=sensor_shear.detect(qs), d_x=d_x, d_y=d_y, rhs=op.rhs(q),
        dt=np.asarray(dt), fx=fx, fy=fy, viscous=visc, drag=drag, cooling=cool, forcing_src=fsrc,
        step=step, hv=hvq, dx=np.asarray(domain.dx), dy=np.asarray(domain.dy),
        **f_out, **klow, **{f"diag_{k}": np.asarray(v) for k, v in diag.items()})


def gen_hit_run(R):
    """A short complete HIT run through the reference's run_simulation."""
    hit2d = R["hit2d"]
    with tempfile.TemporaryDirectory() as tmp:
        cfg = hit2d.HIT2DConfig(nx=24, ny=24, tfinal=0.02, cfl=0.05, target_mach=0.25,
                                initial_kmin=3, initial_kmax=5, forcing_kmin=3.0,
                                forcing_kmax=5.0, forcing_correlation_time=0.5,
                                mach_control=True, mach_control_target=0.25, viscosity=7.5e-4,
                                large_scale_drag=0.1, cooling_time=5.0, hyperviscosity_mn=0.002,
                                diagnostics_every=1000, snapshot_every=1000,
                                output_dir=Path(tmp), backend="numpy")
        with contextlib.redirect_stdout(io.StringIO()):
            q, time, steps = hit2d.run_simulation(cfg)
    np.savez_compressed(HERE / "hit_run_24.npz", q=q, time=np.asarray(time),
                        steps=np.asarray(steps))


def gen_riemann(R):
    rc3 = R["rc3"]
    out = {}
    for tag, cfg in (
        ("c3_32", rc3.RiemannConfig3(nx=32, ny=32, backend="numpy", shear_threshold=None)),
        ("c6_24x28", R["RC6"](nx=24, ny=28, backend="numpy", shear_threshold=None)),
        ("c308_20", R["RC308"](nx=20, ny=20, backend="numpy", shear_threshold=2.0)),
    ):
        eq = cfg.equation
        q0 = rc3.apply_outflow_guard(eq.enforce_physical_state(cfg.initial_state()),
                                     cfg.guard_cells)
        sensor = rc3.NonPeriodicEulerShockSensor2D(
            cfg.domain, eq, width=cfg.sensor_width, compression_threshold=cfg.compression_threshold,
            jump_threshold=cfg.jump_threshold, shear_threshold=cfg.shear_threshold,
            boundary_guard=cfg.boundary_guard)
        op = rc3.NonPeriodicHybridEuler2DOperator(cfg.domain, eq, sensor, scheme=cfg.scheme)
        op_w = rc3.NonPeriodicHybridEuler2DOperator(cfg.domain, eq, sensor, scheme="weno")
        dt, n = op.fixed_time_step(q0, cfg.cfl, cfg.tfinal)
        hv = rc3.LocalHyperviscosity2D(cfg.domain, mn=cfg.mn)

        def clean(s):
            return rc3.apply_outflow_guard(eq.enforce_physical_state(s), cfg.guard_cells)

        q = q0
        for _ in range(6):  # develop some structure first
            q = R["SSPRK3"]().step(q, op.rhs, dt, clean=clean)
        qs = eq.enforce_physical_state(q)
        mask = sensor.detect(qs)
        step = R["SSPRK3"]().step(q, op.rhs, dt, clean=clean)
        hvq = rc3.apply_outflow_guard(hv.apply(q, ~mask, eq), cfg.guard_cells)
        with contextlib.redirect_stdout(io.StringIO()):
            import dataclasses
            cfg_run = dataclasses.replace(cfg, tfinal=0.02, progress_every=10**6)
            q_run, diag = rc3.run_riemann(cfg_run)
        np.savez_compressed(
            HERE / f"riemann_{tag}.npz",
            q0=q0, q=q, mask=mask, rhs=op.rhs(q), rhs_weno=op_w.rhs(q), dt=np.asarray(dt),
            n=np.asarray(n), step=step, hv=hvq, q_run=q_run, run_steps=np.asarray(diag.steps),
            run_hv_apps=np.asarray(diag.hyperviscosity_applications),
            run_sensor_fraction=np.asarray(diag.final_sensor_fraction),
            run_density_min=np.asarray(diag.density_min),
            run_density_max=np.asarray(diag.density_max),
            run_pressure_max=np.asarray(diag.pressure_max),
            run_max_abs_vorticity=np.asarray(diag.max_abs_vorticity),
            shear=np.asarray(-1.0 if cfg.shear_threshold is None else cfg.shear_threshold),
            number=np.asarray(cfg.configuration_number),
            x_split=np.asarray(cfg.x_split), y_split=np.asarray(cfg.y_split),
            tfinal=np.asarray(cfg.tfinal), mn=np.asarray(cfg.mn),
            hv_interval=np.asarray(cfg.hyperviscosity_interval))
        out[tag] = True
    return out


SPECTRA_SETTINGS = (  # (name, fluctuation type, start_time, end_time, stride)
    ("reynolds", "reynolds", None, None, 1),
    ("favre", "favre", None, None, 1),
    ("window", "reynolds", 0.02, 0.07, 2),
)


def gen_spectra(R):
    """HIT2DSpectra.compute (OOP/postprocess/spectra.py:48-149) over snapshots
    that the reference's run_simulation wrote: a non-square 32 x 24 grid (two
    fundamental wavenumbers) and an odd 25 x 20 one, Reynolds and Favre
    fluctuations, a time window with a stride.  The snapshot fields and the
    results (with the warnings raised) are stored."""
    import warnings

    from OOP.postprocess.spectra import HIT2DSpectra

    hit2d = R["hit2d"]
    for tag, nx, ny in (("32x24", 32, 24), ("25x20", 25, 20)):
        with tempfile.TemporaryDirectory() as tmp:
            cfg = hit2d.HIT2DConfig(nx=nx, ny=ny, tfinal=0.08, cfl=0.05, target_mach=0.3,
                                    initial_kmin=2, initial_kmax=6, forcing_kmin=3.0,
                                    forcing_kmax=5.0, viscosity=7.5e-4, large_scale_drag=0.1,
                                    cooling_time=5.0, diagnostics_every=1000, snapshot_every=2,
                                    output_dir=Path(tmp), backend="numpy")
            with contextlib.redirect_stdout(io.StringIO()):
                hit2d.run_simulation(cfg)
            paths = sorted(Path(tmp).glob("hit2d_step*.npz"))
            snaps = [dict(np.load(p)) for p in paths]
            out = {"time": np.array([float(d["time"]) for d in snaps]),
                   "step": np.array([int(d["step"]) for d in snaps]),
                   "x": snaps[0]["x"], "y": snaps[0]["y"],
                   "rho": np.stack([d["rho"] for d in snaps]),
                   "u": np.stack([d["u"] for d in snaps]),
                   "v": np.stack([d["v"] for d in snaps])}
            for name, kind, t0, t1, stride in SPECTRA_SETTINGS:
                with warnings.catch_warnings(record=True) as caught:
                    warnings.simplefilter("always")
                    r = HIT2DSpectra(tmp, fluctuation_type=kind, start_time=t0, end_time=t1,
                                     stride=stride).compute()
                out.update({f"{name}_k": r.k, f"{name}_energy_mean": r.energy_mean,
                            f"{name}_energy_std": r.energy_std,
                            f"{name}_enstrophy_mean": r.enstrophy_mean,
                            f"{name}_enstrophy_std": r.enstrophy_std,
                            f"{name}_n": np.asarray(r.number_of_snapshots),
                            f"{name}_interval": np.asarray(r.selected_time_interval),
                            f"{name}_hk_energy": np.asarray(r.high_k_energy_ratio),
                            f"{name}_hk_enstrophy": np.asarray(r.high_k_enstrophy_ratio),
                            f"{name}_warnings": np.asarray([str(w.message) for w in caught] or [""])})
        np.savez_compressed(HERE / f"spectra_{tag}.npz", **out)


def _collect(tmp: Path) -> dict:
    """Every file a run wrote, flattened into arrays: '<file>::<key>' for each
    .npz member (dtype and shape kept) and '<file>' for each .json (its text)."""
    out = {}
    for path in sorted(tmp.rglob("*")):
        if path.is_dir():
            continue
        rel = path.relative_to(tmp).as_posix()
        if path.suffix == ".npz":
            with np.load(path, allow_pickle=False) as d:
                for k in d.files:
                    out[f"{rel}::{k}"] = d[k]
        elif path.suffix == ".json":
            out[rel] = np.asarray(path.read_text())
    return out


def gen_formats(R):
    """Output files of the reference's own writers: run_simulation's
    config.json, diagnostic_history.npz and snapshots (OOP/hit2d.py:551-694,
    764-918) for a short 24^2 HIT run, and run_riemann plus save_run_outputs
    (OOP/problems/riemann_config3.py:486-519, 681-809; no figure) for a
    24^2 configuration-3 run."""
    hit2d, rc3 = R["hit2d"], R["rc3"]
    with tempfile.TemporaryDirectory() as t:
        tmp = Path(t)
        cfg = hit2d.HIT2DConfig(nx=24, ny=24, tfinal=0.006, cfl=0.05, target_mach=0.25,
                                initial_kmin=3, initial_kmax=5, forcing_kmin=3.0,
                                forcing_kmax=5.0, forcing_correlation_time=0.5,
                                mach_control=True, mach_control_target=0.25, viscosity=7.5e-4,
                                large_scale_drag=0.1, cooling_time=5.0, hyperviscosity_mn=0.002,
                                diagnostics_every=2, snapshot_every=3, output_dir=tmp / "hit",
                                backend="numpy")
        with contextlib.redirect_stdout(io.StringIO()):
            hit2d.run_simulation(cfg)
        out = _collect(tmp / "hit")
    np.savez_compressed(HERE / "formats_hit_24.npz", **out)
    with tempfile.TemporaryDirectory() as t:
        tmp = Path(t)
        cfg = rc3.RiemannConfig3(nx=24, ny=24, tfinal=0.02, backend="numpy", shear_threshold=None,
                                 progress_every=10**6)
        with contextlib.redirect_stdout(io.StringIO()):
            q, diag = rc3.run_riemann(cfg)
            rc3.save_run_outputs(q, cfg, diag, tmp, run_id="fixture", plot=False)
        out = _collect(tmp)
    np.savez_compressed(HERE / "formats_riemann_24.npz", **out)


def main(root: str) -> None:
    R = _import_reference(root)
    for name, (cfg, domain, eq, q) in periodic_cases(R).items():
        gen_periodic(R, name, cfg, domain, eq, q)
    gen_hit_run(R)
    gen_riemann(R)
    gen_spectra(R)
    gen_formats(R)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py <reference-root>")
    main(sys.argv[1])
