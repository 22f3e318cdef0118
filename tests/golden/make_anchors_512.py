"""Full-size (512^2) anchors of the reference HIT_Solver, for the GPU parity tests.

Usage, in a container where the reference source tree is available:

    python tests/golden/make_anchors_512.py <reference-root> published
    python tests/golden/make_anchors_512.py <reference-root> riemann <tag>
    python tests/golden/make_anchors_512.py <reference-root> hit

``published``
    Copies the summary statistics the reference publishes for its 512^2
    Riemann runs (``results/riemann_config*/<run>/{config,diagnostics}.json``,
    FP64 CuPy runs on an unstated GPU) into ``published_riemann_512.json``.

``riemann <tag>``
    Re-runs one of those configurations through the reference's own NumPy
    ``run_riemann`` (``OOP/problems/riemann_config3.py:681-749``) and stores
    its ``RiemannDiagnostics`` plus 16 x 16-cell block means of the final
    conserved state in ``rerun_riemann_<tag>.npz``.  About 1.1 h of one host
    core per 1000 steps.

``hit``
    Runs the production-physics 512^2 forced HIT (shells 3..5, Mach 0.25, OU
    correlation time 0.5, Mach control, viscosity 7.5e-4, hyperviscosity 0.002
    every 5 steps, drag 0.10 on |k| <= 2, cooling time 5.0, CFL 0.05, seed
    1234) for exactly 1000 steps with the reference's objects, in the order of
    the step loop of ``OOP/hit2d.py:815-916`` (that loop stops on a final time
    only, so the step count is imposed here), and stores the reference's
    ``compute_diagnostics`` at steps 0, 1, 10, 100 and 1000, the time, the
    forcing info of the last step and the block means of the final state in
    ``hit512_1000.npz``.  About 1 h of one host core.

The fixtures are committed; neither the tests nor the product read the
reference tree at run time.
"""

from __future__ import annotations

import contextlib
import dataclasses
import io
import json
import sys
import tempfile
import time as _time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BLOCK = 16

# (tag, configuration module, class, results directory under results/, overrides)
RIEMANN_RUNS = {
    "c3_mn0015": ("riemann_config3", "RiemannConfig3",
                  "riemann_config3/config3_centered_hybrid_mn0015_hv1_noContours_gpu_512_t03"),
    "c3_mn001_cfl025": ("riemann_config3", "RiemannConfig3",
                        "riemann_config3/config3_centered_hybrd_gpu_512_t03_mn0p01_CFL_0p4"),
    "c308_t03": ("riemann_config3_08", "RiemannConfig3Offset08",
                 "riemann_config3_08/config3_08_hybrid_mn0001_hv5_gpu_512_t03"),
    "c308_t085": ("riemann_config3_08", "RiemannConfig3Offset08",
                  "riemann_config3_08/config3_08_hybrid_hv5_gpu_512_t085"),
    "c6_t025": ("riemann_config6", "RiemannConfig6",
                "riemann_config6/config6_hybrid_mn001_hv5_gpu_512_t025_no_contours"),
}
CONFIG_KEYS = ("nx", "ny", "tfinal", "cfl", "gamma", "x_split", "y_split", "scheme",
               "sensor_width", "jump_threshold", "compression_threshold", "shear_threshold",
               "boundary_guard", "mn", "hyperviscosity_interval",
               "hyperviscosity_density_weight", "hyperviscosity_momentum_weight",
               "hyperviscosity_energy_weight", "guard_cells")


def block_means(q: np.ndarray, b: int = BLOCK) -> np.ndarray:
    c, ny, nx = q.shape
    return q.reshape(c, ny // b, b, nx // b, b).mean(axis=(2, 4))


def _import_reference(root: str):
    sys.path.insert(0, str(HERE / "_stubs"))
    sys.path.insert(0, root)


def published(root: str) -> None:
    out = {}
    for tag, (_mod, _cls, rel) in RIEMANN_RUNS.items():
        d = Path(root) / "results" / rel
        cfg = json.loads((d / "config.json").read_text())
        diag = json.loads((d / "diagnostics.json").read_text())
        out[tag] = {"source": f"results/{rel}/diagnostics.json",
                    "config": {k: cfg[k] for k in CONFIG_KEYS},
                    "diagnostics": diag}
    (HERE / "published_riemann_512.json").write_text(json.dumps(out, indent=1, sort_keys=True))
    print("wrote", HERE / "published_riemann_512.json")


def riemann(root: str, tag: str) -> None:
    import importlib

    _import_reference(root)
    mod_name, cls_name, rel = RIEMANN_RUNS[tag]
    cfg_json = json.loads((Path(root) / "results" / rel / "config.json").read_text())
    rc3 = importlib.import_module("OOP.problems.riemann_config3")
    cls = getattr(importlib.import_module(f"OOP.problems.{mod_name}"), cls_name)
    kw = {k: cfg_json[k] for k in CONFIG_KEYS}
    cfg = cls(backend="numpy", progress_every=10**9, **kw)
    t0 = _time.time()
    with contextlib.redirect_stdout(io.StringIO()):
        q, diag = rc3.run_riemann(cfg)
    wall = _time.time() - t0
    d = dataclasses.asdict(diag)
    np.savez_compressed(
        HERE / f"rerun_riemann_{tag}.npz", block_means=block_means(np.asarray(q)),
        wall_s=np.asarray(wall),
        **{f"diag_{k}": np.asarray(v) for k, v in d.items()})
    print(tag, "steps", d["steps"], "wall", round(wall, 1), "s")


def hit(root: str, steps: int = 1000) -> None:
    _import_reference(root)
    from OOP import hit2d
    from OOP.forcing import IsotropicShellOUForcing2D
    from OOP.spatial_operator import (PeriodicEulerShockSensor2D,
                                      PeriodicHybridEuler2DOperator,
                                      PeriodicHyperviscosity2D)
    from OOP.time_operator import SSPRK3

    cfg = hit2d.HIT2DConfig(
        nx=512, ny=512, tfinal=1e9, cfl=0.05, target_mach=0.25, initial_kmin=3, initial_kmax=5,
        forcing_kmin=3.0, forcing_kmax=5.0, forcing_correlation_time=0.5,
        forcing_alpha_memory=0.2, target_energy_injection=1e-3, mach_control=True,
        mach_control_target=0.25, mach_control_memory=0.995, mach_control_exponent=2.0,
        viscosity=7.5e-4, hyperviscosity_mn=0.002, hyperviscosity_interval=5,
        large_scale_drag=0.10, large_scale_drag_kmax=2.0, cooling_time=5.0, forcing_seed=1234,
        output_dir=Path(tempfile.mkdtemp()), backend="numpy")
    domain, _x, _y = hit2d.create_grid(cfg)
    eq = hit2d._make_equation(cfg)
    sensor = PeriodicEulerShockSensor2D(domain, eq, width=cfg.sensor_width,
                                        compression_threshold=cfg.compression_threshold,
                                        jump_threshold=cfg.jump_threshold,
                                        shear_threshold=cfg.shear_threshold)
    op = PeriodicHybridEuler2DOperator(domain, eq, sensor)
    hv = PeriodicHyperviscosity2D(domain, mn=cfg.hyperviscosity_mn)
    integ = SSPRK3()
    rng = np.random.default_rng(cfg.forcing_seed)
    forcing = IsotropicShellOUForcing2D(
        domain=domain, k_min=cfg.forcing_kmin, k_max=cfg.forcing_kmax,
        correlation_time=cfg.forcing_correlation_time, force_rms=cfg.forcing_rms,
        target_power=cfg.target_energy_injection, min_power=cfg.min_forcing_power,
        max_rescale=cfg.max_forcing_rescale, alpha_memory=cfg.forcing_alpha_memory,
        seed=cfg.forcing_seed + 1)
    q = eq.enforce_physical_state(hit2d.initialize_hit_2d(cfg, domain, eq, rng))
    d0 = hit2d.compute_diagnostics(q, eq, domain)
    mass0 = d0["mass"]
    record = {0: d0}
    t, power, info = 0.0, cfg.target_energy_injection, {}
    t0 = _time.time()
    for step in range(1, steps + 1):
        dt = op.stable_time_step(q, cfg.cfl, cfg.tfinal - t)
        h = min(domain.dx, domain.dy)
        dt = min(dt, 0.25 * h ** 2 / cfg.viscosity, cfg.tfinal - t)
        rho, u, v, p = eq.primitive_from_conservative(q)
        power, mach_info = hit2d.update_mach_controlled_power(cfg, power, rho, u, v, p)
        forcing.target_power = power
        fx, fy, info = forcing.update(dt, rho, u, v)
        info.update(mach_info)

        def rhs(s, fx=fx, fy=fy):
            r = op.rhs(s) + eq.viscous_rhs(s, domain.dx, domain.dy)
            r = r + hit2d.forcing_source(s, eq, fx, fy)
            r = r + hit2d.large_scale_drag_source(s, eq, domain, cfg.large_scale_drag,
                                                  cfg.large_scale_drag_kmax)
            return r + hit2d.cooling_source(s, eq, cfg.cooling_time, cfg.cooling_target_pressure)

        q = integ.step(q, rhs, dt, clean=eq.enforce_physical_state)
        t += dt
        if step % cfg.hyperviscosity_interval == 0:
            q = hv.apply(q, eq, active_mask=~sensor.detect(q))
        if step in (1, 10, 100, steps):
            drag = hit2d.large_scale_drag_source(q, eq, domain, cfg.large_scale_drag,
                                                 cfg.large_scale_drag_kmax)
            cool = hit2d.cooling_source(q, eq, cfg.cooling_time, cfg.cooling_target_pressure)
            record[step] = hit2d.compute_diagnostics(
                q, eq, domain, initial_mass=mass0, forcing_info=info,
                drag_power=hit2d.source_power(drag), cooling_power=hit2d.source_power(cool),
                large_scale_fraction=hit2d.large_scale_kinetic_fraction(
                    q, eq, domain, cfg.large_scale_drag_kmax),
                weno_fraction=float(np.mean(sensor.detect(q))))
            record[step]["time"] = t
            print(f"step {step} t={t:.9f} KE={record[step]['kinetic_energy']:.12e} "
                  f"wall={_time.time() - t0:.0f}s", flush=True)
    out = {"block_means": block_means(q), "time": np.asarray(t), "steps": np.asarray(steps),
           "wall_s": np.asarray(_time.time() - t0)}
    for s, d in record.items():
        out.update({f"diag{s}_{k}": np.asarray(v) for k, v in d.items()})
    out.update({f"info_{k}": np.asarray(v) for k, v in info.items()})
    np.savez_compressed(HERE / "hit512_1000.npz", **out)
    print("wrote", HERE / "hit512_1000.npz")


def main(argv) -> None:
    if len(argv) < 3:
        raise SystemExit(__doc__)
    root, what = argv[1], argv[2]
    if what == "published":
        published(root)
    elif what == "riemann":
        riemann(root, argv[3])
    elif what == "hit":
        hit(root)
    else:
        raise SystemExit(f"unknown anchor {what!r}")


if __name__ == "__main__":
    main(sys.argv)
