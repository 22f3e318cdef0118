"""GPU parity of the native kernels against the CPU oracle (pinned to the
reference's golden vectors in tests/test_oracle_golden.py).

Tolerances (relative to the largest magnitude of the compared field):
  FP64 plain form: RHS-type fields within 20x the oracle's own sensitivity to
  a one-ulp perturbation of its input (``gpu_util.ulp_floor``; 1e-11 at
  least), states after short runs within 1e-8; sensor masks equal exactly.
  FP32-bulk form: 2e-4 for RHS-type fields, 1e-5 for states after short
  runs; masks equal outside the dilated footprint of nodes within 1e-4
  (relative) of a sensor threshold.
"""

import numpy as np
import pytest
import torch

from oracle import hit_oracle as O
from tests.gpu_util import (dev, fp64_tol, host, near_threshold_footprint, periodic_state,
                            rel_err)

pytestmark = pytest.mark.gpu

from hit_solver_b200 import _lib, core  # noqa: E402
from hit_solver_b200.descs import grid_desc, set_sensor  # noqa: E402
from hit_solver_b200.domain import Domain2D  # noqa: E402

G = 1.4
TOL64 = 1e-9
TOL32 = 2e-4


def periodic_plan(nx, ny, precision="fp64", width=4, jump=0.04, shear=None, **kw):
    dom = Domain2D(0.0, 2 * np.pi, 0.0, 2 * np.pi, nx, ny)
    d = grid_desc(dom, G, True, precision)
    set_sensor(d, width, 2.5, jump, shear)
    for k, v in kw.items():
        setattr(d, k, v)
    return core.Plan(d), dom


def outflow_plan(nx, ny, precision="fp64", scheme=0, shear=None, **kw):
    dom = Domain2D(0.0, 1.0, 0.0, 1.0, nx, ny)
    d = grid_desc(dom, G, False, precision)
    set_sensor(d, 4, 2.5, 0.025, shear, 4)
    d.scheme = scheme
    d.guard_cells = 2
    for i in range(4):
        d.hv_weight[i] = 1.0  # LocalHyperviscosity2D default weights
    for k, v in kw.items():
        setattr(d, k, v)
    return core.Plan(d), dom


PERIODIC_CASES = [(32, 24, False), (40, 36, True), (128, 96, True), (10, 12, True), (37, 29, True)]


@pytest.mark.parametrize("nx,ny,blob", PERIODIC_CASES)
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_periodic_sensor(nx, ny, blob, precision):
    q = periodic_state(nx, ny, blob)
    plan, dom = periodic_plan(nx, ny, precision)
    prm = O.SensorParams(4, 2.5, 0.04, None)
    qs = O.enforce(q, G)
    want = O.sensor(qs, dom.dx, dom.dy, G, prm, True)
    got = host(plan.sensor(dev(qs), enforce_first=False))
    if precision == "fp64":
        np.testing.assert_array_equal(got, want)
    else:
        skip, _ = near_threshold_footprint(qs, dom.dx, dom.dy, G, prm, True, 1e-4)
        assert np.array_equal(got[~skip], want[~skip])
    # shear part and another width
    plan2, _ = periodic_plan(nx, ny, precision, width=3, shear=1.5)
    prm2 = O.SensorParams(3, 2.5, 0.04, 1.5)
    want2 = O.sensor(qs, dom.dx, dom.dy, G, prm2, True)
    got2 = host(plan2.sensor(dev(qs), enforce_first=False))
    skip2, _ = near_threshold_footprint(qs, dom.dx, dom.dy, G, prm2, True,
                                        1e-12 if precision == "fp64" else 1e-4)
    assert np.array_equal(got2[~skip2], want2[~skip2])


@pytest.mark.parametrize("nx,ny,blob", PERIODIC_CASES)
@pytest.mark.parametrize("precision,tol", [("fp64", TOL64), ("fp32", TOL32)])
def test_periodic_axis_derivatives_and_rhs(nx, ny, blob, precision, tol):
    q = periodic_state(nx, ny, blob)
    plan, dom = periodic_plan(nx, ny, precision)
    prm = O.SensorParams(4, 2.5, 0.04, None)
    want, parts = O.inviscid_rhs(q, dom.dx, dom.dy, G, prm, True, return_parts=True)
    mask = dev(parts["mask"].astype(np.uint8))
    d_x = host(plan.axis_derivative(dev(q), mask, 0))
    d_y = host(plan.axis_derivative(dev(q), mask, 1))
    for axis, h, got_d in ((-1, dom.dx, d_x), (-2, dom.dy, d_y)):
        ref = parts["d_x" if axis == -1 else "d_y"]
        if precision == "fp64":
            tol = fp64_tol(lambda a: O.axis_derivative(O.enforce(a, G), parts["mask"], h, G, axis,
                                                       True), q)
        assert rel_err(got_d, ref) < tol
    if precision == "fp64":
        got = host(plan.rhs(dev(q), _lib.TERM_INVISCID))
        assert rel_err(got, want) < fp64_tol(
            lambda a: O.inviscid_rhs(a, dom.dx, dom.dy, G, prm, True), q)


def test_weno_everywhere_and_all_smooth():
    """Faces flagged everywhere (mask all ones) and nowhere (all zeros)."""
    q = periodic_state(48, 40, True)
    plan, dom = periodic_plan(48, 40)
    qs = O.enforce(q, G)
    for fill in (0, 1):
        m = np.full((40, 48), bool(fill))
        for axis, ax in ((0, -1), (1, -2)):
            h = dom.dx if axis == 0 else dom.dy
            want = O.axis_derivative(qs, m, h, G, ax, True)
            got = host(plan.axis_derivative(dev(q), dev(m.astype(np.uint8)), axis))
            tol = fp64_tol(lambda a: O.axis_derivative(O.enforce(a, G), m, h, G, ax, True), q)
            assert rel_err(got, want) < tol


@pytest.mark.parametrize("nx,ny", [(64, 48), (37, 29)])
@pytest.mark.parametrize("precision,tol", [("fp64", TOL64), ("fp32", TOL32)])
def test_hit_full_rhs_and_sources(nx, ny, precision, tol):
    q = periodic_state(nx, ny, True)
    rng = np.random.default_rng(5)
    fx, fy = 0.3 * rng.standard_normal((ny, nx)), 0.3 * rng.standard_normal((ny, nx))
    plan, dom = periodic_plan(nx, ny, precision, viscosity=1e-3, drag_coefficient=0.1,
                              drag_kmax=2.0, cooling_time=5.0)
    prm = O.HITParams(nx=nx, ny=ny, viscosity=1e-3, large_scale_drag=0.1, cooling_time=5.0)
    want = O.hit_rhs(q, prm, fx, fy)
    got = host(plan.rhs(dev(q), _lib.TERM_ALL, dev(fx), dev(fy)))
    if precision == "fp64":
        tol = fp64_tol(lambda a: O.hit_rhs(a, prm, fx, fy), q)
    assert rel_err(got, want) < tol
    # individual source terms (no inviscid part)
    dx, dy = dom.dx, dom.dy
    checks = [
        (_lib.TERM_VISCOUS, O.viscous_rhs(q, dx, dy, G, 1e-3)),
        (_lib.TERM_DRAG, O.drag_source(q, dx, dy, G, 0.1, 2.0)),
        (_lib.TERM_COOLING, O.cooling_source(q, G, 5.0)),
        (_lib.TERM_FORCING, O.forcing_source(q, fx, fy, G)),
    ]
    for term, ref in checks:
        out = host(plan.rhs(dev(q), term, dev(fx), dev(fy)))
        assert rel_err(out, ref) < (1e-12 if precision == "fp64" else 1e-5), term


@pytest.mark.parametrize("name", ["periodic_hit_32x24", "periodic_blob_40x36"])
def test_golden_periodic_fixtures(name):
    """Native FP64 results against the reference's own outputs."""
    from pathlib import Path

    d = np.load(Path(__file__).parent / "golden" / f"{name}.npz")
    q = d["q"]
    ny, nx = q.shape[1:]
    plan, dom = periodic_plan(nx, ny, viscosity=1e-3, drag_coefficient=0.1, drag_kmax=2.0,
                              cooling_time=5.0)
    qs = host(plan.enforce(dev(q)))
    plan_sensor = host(plan.sensor(dev(qs), False))
    np.testing.assert_array_equal(plan_sensor, d["mask"])
    assert plan_sensor.dtype == bool
    prm = O.SensorParams(4, 2.5, 0.04, None)
    tol = fp64_tol(lambda a: O.inviscid_rhs(a, dom.dx, dom.dy, G, prm, True), q)
    assert rel_err(host(plan.rhs(dev(q), _lib.TERM_INVISCID)), d["rhs"]) < tol
    assert rel_err(host(plan.viscous_rhs(dev(q))), d["viscous"]) < 1e-12
    assert abs(plan.stable_time_step(dev(q), 0.05, 1.0) - float(d["dt"])) < 1e-15
    hv, _ = periodic_plan(nx, ny, hv_mn=0.002)
    out = host(hv.hyperviscosity(dev(q), dev((~d["mask"]).astype(np.uint8))))
    assert rel_err(out, d["hv"]) < 1e-14


@pytest.mark.parametrize("nx,ny", [(40, 36), (128, 96)])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("fp32", 1e-9)])
def test_hyperviscosity(nx, ny, precision, tol):
    q = periodic_state(nx, ny, True)
    plan, dom = periodic_plan(nx, ny, precision, hv_mn=0.002)
    m = O.sensor(q, dom.dx, dom.dy, G, O.SensorParams(), True)
    want = O.hyperviscosity(q, ~m, dom.dx, dom.dy, G, 0.002, (0.25, 1, 1, 0.25), True)
    got = host(plan.hyperviscosity(dev(q), dev((~m).astype(np.uint8))))
    assert rel_err(got, want) < tol
    # nodes outside the active mask are untouched up to the enforce filter
    np.testing.assert_allclose(got[:, m], O.enforce(q, G)[:, m], rtol=0, atol=1e-15)


RIEMANN_CASES = [("c3", 3, 64, 64, 0.5, None), ("c6", 6, 48, 56, 0.5, None),
                 ("c308", 3, 40, 40, 0.8, 2.0)]


def riemann_state(number, nx, ny, split, steps=8):
    prm = O.RiemannParams(number=number, nx=nx, ny=ny, x_split=split, y_split=split)
    q0, dt, n = O.riemann_setup(prm)
    q, _, _, _ = O.riemann_run(prm, max_steps=steps)
    return q, dt, prm


@pytest.mark.parametrize("tag,number,nx,ny,split,shear", RIEMANN_CASES)
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_riemann_sensor_rhs(tag, number, nx, ny, split, shear, precision):
    q, dt, prm = riemann_state(number, nx, ny, split)
    plan, dom = outflow_plan(nx, ny, precision, shear=shear)
    sp = O.SensorParams(4, 2.5, 0.025, shear, 4)
    qs = O.enforce(q, G)
    want = O.sensor(qs, dom.dx, dom.dy, G, sp, False)
    got = host(plan.sensor(dev(qs), False))
    if precision == "fp64":
        np.testing.assert_array_equal(got, want)
    else:
        skip, _ = near_threshold_footprint(qs, dom.dx, dom.dy, G, sp, False, 1e-4)
        assert np.array_equal(got[~skip], want[~skip])
    want_rhs, parts = O.inviscid_rhs(q, dom.dx, dom.dy, G, sp, False, return_parts=True)
    m = dev(parts["mask"].astype(np.uint8))
    for axis, ax, h, key in ((0, -1, dom.dx, "d_x"), (1, -2, dom.dy, "d_y")):
        tol = TOL32 if precision == "fp32" else fp64_tol(
            lambda a: O.axis_derivative(O.enforce(a, G), parts["mask"], h, G, ax, False), q)
        assert rel_err(host(plan.axis_derivative(dev(q), m, axis)), parts[key]) < tol
    if precision == "fp64":
        tol = fp64_tol(lambda a: O.inviscid_rhs(a, dom.dx, dom.dy, G, sp, False), q)
        assert rel_err(host(plan.rhs(dev(q), _lib.TERM_INVISCID)), want_rhs) < tol
        wplan, _ = outflow_plan(nx, ny, precision, scheme=1, shear=shear)
        want_w = O.inviscid_rhs(q, dom.dx, dom.dy, G, sp, False, "weno")
        tol = fp64_tol(lambda a: O.inviscid_rhs(a, dom.dx, dom.dy, G, sp, False, "weno"), q)
        assert rel_err(host(wplan.rhs(dev(q), _lib.TERM_INVISCID)), want_w) < tol


@pytest.mark.parametrize("tag", ["c3_32", "c6_24x28", "c308_20"])
def test_golden_riemann_fixtures(tag):
    from pathlib import Path

    d = np.load(Path(__file__).parent / "golden" / f"riemann_{tag}.npz")
    q = d["q"]
    ny, nx = q.shape[1:]
    sh = float(d["shear"])
    plan, dom = outflow_plan(nx, ny, shear=None if sh < 0 else sh, hv_mn=float(d["mn"]))
    qs = host(plan.enforce(dev(q)))
    np.testing.assert_array_equal(host(plan.sensor(dev(qs), False)), d["mask"])
    sp = O.SensorParams(4, 2.5, 0.025, None if sh < 0 else sh, 4)
    tol = fp64_tol(lambda a: O.inviscid_rhs(a, dom.dx, dom.dy, G, sp, False), q)
    assert rel_err(host(plan.rhs(dev(q), _lib.TERM_INVISCID)), d["rhs"]) < tol
    hv = host(plan.outflow_guard(plan.hyperviscosity(dev(q), dev((~d["mask"]).astype(np.uint8)))))
    assert rel_err(hv, d["hv"]) < 1e-14
    dt = plan.stable_time_step(dev(d["q0"]), 0.4, None)
    n = int(np.ceil(float(d["tfinal"]) / dt))
    assert n == int(d["n"]) and abs(float(d["tfinal"]) / n - float(d["dt"])) < 1e-17


def test_outflow_guard_and_validate():
    q, _, _ = riemann_state(3, 24, 20, 0.5, steps=2)
    plan, _ = outflow_plan(24, 20)
    qq = q.copy()
    qq[:, 5, 7] += 0.3
    want = O.outflow_guard(qq, 2)
    np.testing.assert_array_equal(host(plan.outflow_guard(dev(qq))), want)
    assert plan.validate(dev(q)) == _lib.OK
    bad = q.copy()
    bad[2, 3, 4] = np.nan
    assert plan.validate(dev(bad)) == _lib.ERR_NONFINITE
    bad = q.copy()
    bad[0, 3, 4] = -1.0
    assert plan.validate(dev(bad)) == _lib.ERR_NONPOSITIVE


@pytest.mark.parametrize("nx,ny", [(32, 24), (64, 64)])
def test_forcing_update_sequence(nx, ny):
    q = periodic_state(nx, ny, False)
    dom = Domain2D(0.0, 2 * np.pi, 0.0, 2 * np.pi, nx, ny)
    d = grid_desc(dom, G, True)
    d.forcing_on, d.forcing_kmin, d.forcing_kmax, d.forcing_correlation_time = 1, 3.0, 5.0, 0.5
    plan = core.Plan(d)
    ref = O.ShellOUForcing(nx, ny, dom.dx, dom.dy, 3.0, 5.0, 0.5, 1.0, 1e-3, 1e-6, 20.0, 0.2, 99)
    rho, u, v, _ = O.primitives(q, G)
    rng = np.random.default_rng(99)
    for k in range(3):
        noise = rng.standard_normal((ny, nx))
        dt = 0.004 * (1 + 0.1 * k)
        fx_w, fy_w, info = ref.update(dt, rho, u, v, noise=noise)
        fx, fy = plan.forcing_update(dev(q), dev(noise), dt, 1e-3)
        assert rel_err(host(fx), fx_w) < 1e-11
        assert rel_err(host(fy), fy_w) < 1e-11
        s = plan.scalars()
        assert s[_lib.S_F_ALPHA] == pytest.approx(info["alpha"], rel=1e-10)
        assert s[_lib.S_F_INJECTED] == pytest.approx(info["injected_power"], rel=1e-9)
        assert s[_lib.S_F_FXX] == pytest.approx(info["Fxx"], rel=1e-10)
        assert s[_lib.S_F_AF] == pytest.approx(info["A_F"], rel=1e-8, abs=1e-12)
        assert s[_lib.S_F_DECAY] == pytest.approx(info["ou_decay"], rel=1e-15)


def _hit_solver(nx, ny, precision="fp64", **kw):
    from hit_solver_b200.hit2d import HIT2DConfig, HITSolver

    cfg = HIT2DConfig(nx=nx, ny=ny, tfinal=kw.pop("tfinal", 1.0), cfl=0.05, target_mach=0.25,
                      initial_kmin=3, initial_kmax=5, forcing_kmin=3.0, forcing_kmax=5.0,
                      forcing_correlation_time=0.5, mach_control=True, mach_control_target=0.25,
                      viscosity=7.5e-4, large_scale_drag=0.1, cooling_time=5.0,
                      hyperviscosity_mn=0.002, precision=precision, **kw)
    prm = O.HITParams(nx=nx, ny=ny, tfinal=cfg.tfinal, cfl=0.05, target_mach=0.25,
                      forcing_correlation_time=0.5, mach_control=True, mach_control_target=0.25,
                      viscosity=7.5e-4, large_scale_drag=0.1, cooling_time=5.0)
    return HITSolver(cfg), prm


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("fp32", 1e-5)])
def test_hit_fused_steps_match_oracle(precision, tol):
    """hitb200_step (dt, Mach control, OU forcing with the reference's NumPy
    noise stream, SSP-RK3, hyperviscosity every 5 steps) against the oracle
    driver over 6 steps."""
    solver, prm = _hit_solver(48, 40, precision)
    want, t_w, steps_w, info_w = O.hit_run(prm, max_steps=6)
    solver.advance(6)
    s = solver.scalars()
    assert int(s[_lib.S_STEP]) == steps_w == 6
    # the CFL dt follows the state, so the FP32-bulk state moves it slightly
    assert s[_lib.S_TIME] == pytest.approx(t_w, rel=1e-12 if precision == "fp64" else 1e-6)
    assert rel_err(host(solver.q), want) < tol
    assert s[_lib.S_F_INJECTED] == pytest.approx(info_w["injected_power"], rel=1e-6)
    assert int(s[_lib.S_HV_APPLIED]) == 1


def test_hit_golden_run():
    """The reference's own run_simulation output (24x24, 5 steps to t=0.02)."""
    from pathlib import Path

    d = np.load(Path(__file__).parent / "golden" / "hit_run_24.npz")
    solver, _ = _hit_solver(24, 24, tfinal=0.02)
    solver.advance(int(d["steps"]) + 2)  # extra steps are no-ops after tfinal
    s = solver.scalars()
    assert int(s[_lib.S_STEP]) == int(d["steps"])
    assert s[_lib.S_TIME] == pytest.approx(float(d["time"]), rel=1e-14)
    assert rel_err(host(solver.q), d["q"]) < 1e-8


@pytest.mark.parametrize("tag,number,nx,ny,split,shear", RIEMANN_CASES)
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("fp32", 1e-5)])
def test_riemann_run_matches_oracle(tag, number, nx, ny, split, shear, precision, tol):
    from hit_solver_b200.problems.riemann import RiemannConfig3, RiemannConfig6, RiemannSolver

    cls = RiemannConfig6 if number == 6 else RiemannConfig3
    hv_interval = 5 if split == 0.8 else 1
    cfg = cls(nx=nx, ny=ny, x_split=split, y_split=split, shear_threshold=shear,
              hyperviscosity_interval=hv_interval, precision=precision)
    solver = RiemannSolver(cfg)
    prm = O.RiemannParams(number=number, nx=nx, ny=ny, x_split=split, y_split=split,
                          tfinal=cfg.tfinal, shear_threshold=shear, hyperviscosity_interval=hv_interval)
    want, dt, steps, apps = O.riemann_run(prm, max_steps=10)
    assert solver.dt == pytest.approx(dt, rel=1e-15)
    solver.advance(10)
    assert rel_err(host(solver.q), want) < tol
    assert int(solver.plan.scalars()[_lib.S_HV_APPLIED]) == apps


@pytest.mark.parametrize("tag", ["c3_32", "c6_24x28", "c308_20"])
def test_riemann_golden_runs(tag):
    """The reference's own run_riemann output to t = 0.02."""
    from pathlib import Path

    from hit_solver_b200.problems.riemann import (RiemannConfig3, RiemannConfig3Offset08,
                                                  RiemannConfig6, run_riemann)

    d = np.load(Path(__file__).parent / "golden" / f"riemann_{tag}.npz")
    ny, nx = d["q"].shape[1:]
    sh = float(d["shear"])
    cls = {"c3_32": RiemannConfig3, "c6_24x28": RiemannConfig6, "c308_20": RiemannConfig3Offset08}[tag]
    cfg = cls(nx=nx, ny=ny, tfinal=0.02, shear_threshold=None if sh < 0 else sh,
              progress_every=10 ** 6)
    q, diag = run_riemann(cfg)
    assert diag.steps == int(d["run_steps"])
    assert diag.hyperviscosity_applications == int(d["run_hv_apps"])
    assert rel_err(host(q), d["q_run"]) < 1e-8
    assert diag.density_max == pytest.approx(float(d["run_density_max"]), rel=1e-10)
    assert diag.max_abs_vorticity == pytest.approx(float(d["run_max_abs_vorticity"]), rel=1e-8)
    assert diag.final_sensor_fraction == pytest.approx(float(d["run_sensor_fraction"]), abs=1e-12)


@pytest.mark.parametrize("nx,ny", [(1024, 64), (64, 1024), (768, 96)])
def test_large_grid_steps_match_oracle(nx, ny):
    """Lines of 768 and 1024 nodes (8 nodes per sweep thread, in x and in y):
    2 FP64 steps of Riemann configuration 3 against the oracle, and the
    FP32-bulk form against the FP64 one."""
    from hit_solver_b200.problems.riemann import RiemannConfig3, RiemannSolver

    out = {}
    for precision in ("fp64", "fp32-bulk"):
        cfg = RiemannConfig3(nx=nx, ny=ny, x_split=0.45, y_split=0.55, shear_threshold=None,
                             precision=precision)
        solver = RiemannSolver(cfg)
        solver.advance(2)
        out[precision] = host(solver.q)
    prm = O.RiemannParams(number=3, nx=nx, ny=ny, x_split=0.45, y_split=0.55, shear_threshold=None)
    want, _, _, _ = O.riemann_run(prm, max_steps=2)
    assert rel_err(out["fp64"], want) < 1e-8
    assert rel_err(out["fp32-bulk"], out["fp64"]) < 1e-5


_DIAG_FROM_STATE = ("kinetic_energy", "Kx", "Ky", "A_K", "C_uv", "rms_velocity", "turbulent_mach",
                    "mean_density", "mean_pressure", "divergence_rms", "vorticity_rms", "mass",
                    "mass_error")


@pytest.mark.parametrize("name", ["periodic_hit_32x24", "periodic_blob_40x36"])
def test_golden_periodic_diagnostics(name):
    """compute_diagnostics (OOP/hit2d.py:471-548) of the fixture state: the
    native moment reduction plus the spectral divergence and vorticity,
    against the values the reference computed for the same state.  Values
    that are roundoff in the reference (A_K, C_uv and the divergence of the
    solenoidal initial state, about 1e-16) are compared on the scale of the
    quantity they are a difference of."""
    from pathlib import Path

    from hit_solver_b200.equations import EulerEquation2D
    from hit_solver_b200.hit2d import compute_diagnostics

    d = np.load(Path(__file__).parent / "golden" / f"{name}.npz")
    q = d["q"]
    ny, nx = q.shape[1:]
    dom = Domain2D(0.0, 2 * np.pi, 0.0, 2 * np.pi, nx, ny)
    got = compute_diagnostics(dev(q), EulerEquation2D(gamma=G), dom)
    scale = {"A_K": 1.0, "C_uv": 1.0, "divergence_rms": float(d["diag_vorticity_rms"]),
             "mass_error": 1.0}
    for key in _DIAG_FROM_STATE:
        want = float(d[f"diag_{key}"])
        ref = max(abs(want), scale.get(key, 0.0))
        assert abs(got[key] - want) <= 1e-12 * ref, (key, got[key], want)


@pytest.mark.parametrize("name", ["periodic_hit_32x24", "periodic_blob_40x36"])
def test_golden_large_scale_kinetic_fraction(name):
    """large_scale_kinetic_fraction (OOP/hit2d.py:429-449) through the
    library's line transforms, against the reference's values for the
    fixture state (the 1 and 2 bands hold only roundoff of this state)."""
    from pathlib import Path

    from hit_solver_b200.equations import EulerEquation2D
    from hit_solver_b200.hit2d import large_scale_kinetic_fraction

    d = np.load(Path(__file__).parent / "golden" / f"{name}.npz")
    q = d["q"]
    ny, nx = q.shape[1:]
    dom = Domain2D(0.0, 2 * np.pi, 0.0, 2 * np.pi, nx, ny)
    for k in (1.0, 2.0, 3.5):
        got = large_scale_kinetic_fraction(dev(q), EulerEquation2D(gamma=G), dom, k)
        want = float(d[f"klow_{k:g}"])
        assert abs(got - want) <= 1e-12 * max(abs(want), 1.0), (k, got, want)


@pytest.mark.parametrize("shape", [(24, 32), (20, 25), (97, 64), (63, 50), (1024, 6), (7, 1021), (384, 384),
                                   (512, 512), (33, 64), (256, 16), (8, 1024), (1024, 32), (128, 8)])
def test_rfft2_matches_numpy(shape):
    """The library's line transforms (hitb200_rfft2) against
    numpy.fft.rfft2: mixed radices 4, 2, 3, 5, 7 and prime lengths, and the
    radix-8 kernel of power-of-two lengths (rows packed in pairs, an odd
    row count included)."""
    ny, nx = shape
    lib = _lib.load()
    rng = np.random.default_rng(ny * 7 + nx)
    a = rng.standard_normal((3, ny, nx))
    out = torch.empty((3, ny, nx // 2 + 1), dtype=torch.complex128, device="cuda")
    ws = torch.empty(int(lib.hitb200_rfft2_workspace_bytes(nx, ny)), dtype=torch.uint8, device="cuda")
    _lib.check(lib.hitb200_rfft2(dev(a).data_ptr(), 3, nx, ny, out.data_ptr(), ws.data_ptr(), ws.numel(),
                                 core.stream_handle()))
    want = np.fft.rfft2(a)
    assert rel_err(out.cpu().numpy(), want) < 1e-13


def test_rfft2_unaligned_input_matches_numpy():
    """Rows that start 8 bytes past a 16-byte boundary take the radix-8
    kernel's one-value loads instead of its paired ones."""
    ny, nx = 64, 128
    lib = _lib.load()
    a = np.random.default_rng(11).standard_normal((2, ny, nx))
    buf = torch.empty(a.size + 1, dtype=torch.float64, device="cuda")
    src = buf[1:].view(2, ny, nx)
    src.copy_(dev(a))
    assert src.data_ptr() % 16 == 8
    out = torch.empty((2, ny, nx // 2 + 1), dtype=torch.complex128, device="cuda")
    ws = torch.empty(int(lib.hitb200_rfft2_workspace_bytes(nx, ny)), dtype=torch.uint8, device="cuda")
    _lib.check(lib.hitb200_rfft2(src.data_ptr(), 2, nx, ny, out.data_ptr(), ws.data_ptr(), ws.numel(),
                                 core.stream_handle()))
    assert rel_err(out.cpu().numpy(), np.fft.rfft2(a)) < 1e-13


@pytest.mark.parametrize("ny,nx", [(40, 27), (64, 128)])
def test_spectral_divergence_vorticity_fields(ny, nx):
    """divergence_and_vorticity (OOP/hit2d.py:146-155, 459-468) against the
    oracle's NumPy spectral derivatives on non-square grids with a Nyquist
    row (even ny): an odd nx (mixed radix) and power-of-two lengths."""
    from hit_solver_b200.hit2d import divergence_and_vorticity

    dom = Domain2D(0.0, 2 * np.pi, 0.0, 3.0, nx, ny)
    rng = np.random.default_rng(3)
    u, v = rng.standard_normal((ny, nx)), rng.standard_normal((ny, nx))
    kx, ky = O.wavenumbers(nx, ny, dom.dx, dom.dy)

    def d(a, k):
        return np.fft.ifft2(1j * k * np.fft.fft2(a)).real

    want_div = d(u, kx) + d(v, ky)
    want_vort = d(v, kx) - d(u, ky)
    div, vort = divergence_and_vorticity(dev(u), dev(v), dom)
    assert rel_err(host(div), want_div) < 1e-12
    assert rel_err(host(vort), want_vort) < 1e-12
