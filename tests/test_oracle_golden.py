"""Pins the CPU oracle against golden vectors the reference itself produced
(``tests/golden/make_golden.py``).  Every comparison here is bit-exact: the
oracle restates the reference's arithmetic in the same operation order."""

import dataclasses
from pathlib import Path

import numpy as np
import pytest

from oracle import hit_oracle as O

G = Path(__file__).resolve().parent / "golden"
PERIODIC = ["periodic_hit_32x24", "periodic_blob_40x36"]
RIEMANN = ["riemann_c3_32", "riemann_c6_24x28", "riemann_c308_20"]
GAMMA = 1.4


def load(name):
    return np.load(G / f"{name}.npz")


@pytest.mark.parametrize("name", PERIODIC)
def test_periodic_sensor_rhs_sources(name):
    d = load(name)
    q, dx, dy = d["q"], float(d["dx"]), float(d["dy"])
    qs = O.enforce(q, GAMMA)
    sp = O.SensorParams(4, 2.5, 0.04, None)
    np.testing.assert_array_equal(O.sensor(qs, dx, dy, GAMMA, sp, True), d["mask"])
    np.testing.assert_array_equal(
        O.sensor(qs, dx, dy, GAMMA, O.SensorParams(3, 2.5, 0.04, 1.5), True), d["mask_shear"])
    rhs, parts = O.inviscid_rhs(q, dx, dy, GAMMA, sp, True, return_parts=True)
    np.testing.assert_array_equal(rhs, d["rhs"])
    np.testing.assert_array_equal(parts["d_x"], d["d_x"])
    np.testing.assert_array_equal(parts["d_y"], d["d_y"])
    np.testing.assert_array_equal(O.viscous_rhs(q, dx, dy, GAMMA, 1e-3), d["viscous"])
    np.testing.assert_array_equal(O.drag_source(q, dx, dy, GAMMA, 0.1, 2.0), d["drag"])
    np.testing.assert_array_equal(O.cooling_source(q, GAMMA, 5.0), d["cooling"])
    np.testing.assert_array_equal(O.forcing_source(q, d["fx"], d["fy"], GAMMA), d["forcing_src"])
    assert O.spectral_radius_dt(q, 0.05, dx, dy, GAMMA, 1.0) == float(d["dt"])
    hv = O.hyperviscosity(q, ~d["mask"], dx, dy, GAMMA, 0.002, (0.25, 1, 1, 0.25), True)
    np.testing.assert_array_equal(hv, d["hv"])
    with pytest.raises(ValueError):
        O.hyperviscosity(q, None, dx, dy, GAMMA, 0.002, (0.25, 1, 1, 0.25), True)


@pytest.mark.parametrize("name", PERIODIC)
def test_large_scale_kinetic_fraction(name):
    d = load(name)
    q, dx, dy = d["q"], float(d["dx"]), float(d["dy"])
    for k in (1.0, 2.0, 3.5):
        assert O.large_scale_kinetic_fraction(q, dx, dy, GAMMA, k) == float(d[f"klow_{k:g}"])


@pytest.mark.parametrize("name", PERIODIC)
def test_periodic_rk3_step(name):
    d = load(name)
    q, dx, dy = d["q"], float(d["dx"]), float(d["dy"])
    prm = O.HITParams(nx=q.shape[2], ny=q.shape[1], viscosity=1e-3, large_scale_drag=0.1,
                      cooling_time=5.0)
    fx, fy = d["fx"], d["fy"]
    step = O.ssprk3(q, lambda s: O.hit_rhs(s, prm, fx, fy), float(d["dt"]),
                    lambda s: O.enforce(s, GAMMA))
    np.testing.assert_array_equal(step, d["step"])


@pytest.mark.parametrize("name", PERIODIC)
def test_ou_forcing_sequence(name):
    d = load(name)
    q, dx, dy, dt = d["q"], float(d["dx"]), float(d["dy"]), float(d["dt"])
    f = O.ShellOUForcing(q.shape[2], q.shape[1], dx, dy, 3.0, 5.0, 0.5, 1.0, 1e-3, 1e-6, 20.0,
                         0.2, 1235)
    rho, u, v, _ = O.primitives(q, GAMMA)
    for k in range(3):
        fx, fy, info = f.update(dt * (1.0 + 0.1 * k), rho, u, v)
        np.testing.assert_array_equal(fx, d[f"forcing{k}_fx"])
        np.testing.assert_array_equal(fy, d[f"forcing{k}_fy"])
        for key, val in info.items():
            assert val == float(d[f"forcing{k}_info_{key}"]), key


@pytest.mark.parametrize("name", PERIODIC)
def test_hit_diagnostics(name):
    d = load(name)
    dg = O.hit_diagnostics(d["q"], float(d["dx"]), float(d["dy"]), 2 * np.pi, GAMMA)
    for key, val in dg.items():
        if f"diag_{key}" in d:
            assert val == float(d[f"diag_{key}"]), key


def test_hit_run_simulation():
    d = load("hit_run_24")
    prm = O.HITParams(nx=24, ny=24, tfinal=0.02, cfl=0.05, target_mach=0.25,
                      forcing_correlation_time=0.5, mach_control=True, mach_control_target=0.25,
                      viscosity=7.5e-4, large_scale_drag=0.1, cooling_time=5.0)
    q, t, steps, _ = O.hit_run(prm)
    np.testing.assert_array_equal(q, d["q"])
    assert t == float(d["time"]) and steps == int(d["steps"])


def riemann_params(d):
    sh = float(d["shear"])
    return O.RiemannParams(number=int(d["number"]), nx=d["q"].shape[2], ny=d["q"].shape[1],
                           x_split=float(d["x_split"]), y_split=float(d["y_split"]),
                           tfinal=float(d["tfinal"]), mn=float(d["mn"]),
                           shear_threshold=None if sh < 0 else sh,
                           hyperviscosity_interval=int(d["hv_interval"]))


@pytest.mark.parametrize("name", RIEMANN)
def test_riemann_operators(name):
    d = load(name)
    prm = riemann_params(d)
    q0, dt, n = O.riemann_setup(prm)
    np.testing.assert_array_equal(q0, d["q0"])
    assert dt == float(d["dt"]) and n == int(d["n"])
    dx, dy = 1.0 / prm.nx, 1.0 / prm.ny
    sp = O.SensorParams(prm.sensor_width, prm.compression_threshold, prm.jump_threshold,
                        prm.shear_threshold, prm.boundary_guard)
    q = d["q"]
    m = O.sensor(O.enforce(q, GAMMA), dx, dy, GAMMA, sp, False)
    np.testing.assert_array_equal(m, d["mask"])
    np.testing.assert_array_equal(O.inviscid_rhs(q, dx, dy, GAMMA, sp, False), d["rhs"])
    np.testing.assert_array_equal(O.inviscid_rhs(q, dx, dy, GAMMA, sp, False, "weno"),
                                  d["rhs_weno"])

    def clean(s):
        return O.outflow_guard(O.enforce(s, GAMMA), prm.guard_cells)

    st = O.ssprk3(q, lambda s: O.inviscid_rhs(s, dx, dy, GAMMA, sp, False), dt, clean)
    np.testing.assert_array_equal(st, d["step"])
    hv = O.outflow_guard(O.hyperviscosity(q, ~m, dx, dy, GAMMA, prm.mn, prm.hv_weights, False),
                         prm.guard_cells)
    np.testing.assert_array_equal(hv, d["hv"])


@pytest.mark.parametrize("name", RIEMANN)
def test_riemann_run(name):
    d = load(name)
    prm = dataclasses.replace(riemann_params(d), tfinal=0.02)
    q, dt, steps, apps = O.riemann_run(prm)
    np.testing.assert_array_equal(q, d["q_run"])
    assert steps == int(d["run_steps"]) and apps == int(d["run_hv_apps"])
    diag = O.riemann_diagnostics(q, prm)
    assert diag["density_min"] == float(d["run_density_min"])
    assert diag["density_max"] == float(d["run_density_max"])
    assert diag["pressure_max"] == float(d["run_pressure_max"])
    assert diag["max_abs_vorticity"] == float(d["run_max_abs_vorticity"])


def test_reference_initial_states():
    """The quadrant fixtures of the reference's own tests
    (tests/test_riemann_config6.py:11-43, tests/test_riemann_config3_08.py:24-41)."""
    q = O.riemann_initial_state(6, 4, 4)
    rho, u, v, p = O.primitives(q, GAMMA)
    np.testing.assert_array_equal(rho, [[1, 1, 3, 3], [1, 1, 3, 3], [2, 2, 1, 1], [2, 2, 1, 1]])
    np.testing.assert_array_equal(u[:2], -0.75)
    np.testing.assert_array_equal(u[2:], 0.75)
    np.testing.assert_array_equal(v[:, :2], 0.5)
    np.testing.assert_array_equal(v[:, 2:], -0.5)
    np.testing.assert_array_equal(p, 1.0)
    q = O.riemann_initial_state(3, 10, 10, 0.8, 0.8)
    rho, u, v, p = O.primitives(q, GAMMA)
    for (j, i), st in {(0, 0): (0.138, 1.206, 1.206, 0.029), (0, 9): (0.5323, 0.0, 1.206, 0.3),
                       (9, 0): (0.5323, 1.206, 0.0, 0.3), (9, 9): (1.5, 0.0, 0.0, 1.5)}.items():
        np.testing.assert_allclose((rho[j, i], u[j, i], v[j, i], p[j, i]), st, rtol=0, atol=1e-14)
    assert np.count_nonzero(rho == 0.138) == 64
    assert np.count_nonzero(rho == 0.5323) == 32
    assert np.count_nonzero(rho == 1.5) == 4


SPECTRA_SETTINGS = (("reynolds", "reynolds", None, None, 1), ("favre", "favre", None, None, 1),
                    ("window", "reynolds", 0.02, 0.07, 2))


@pytest.mark.parametrize("tag", ["32x24", "25x20"])
def test_spectra_summary(tag):
    """HIT2DSpectra.compute over snapshots of the reference's own run."""
    from oracle import spectra_oracle as SO

    d = load(f"spectra_{tag}")
    for name, kind, t0, t1, stride in SPECTRA_SETTINGS:
        sel = [i for i, t in enumerate(d["time"])
               if (t0 is None or t >= t0) and (t1 is None or t <= t1)][::stride]
        r = SO.spectra_summary(((d["time"][i], d["x"], d["y"], d["rho"][i], d["u"][i], d["v"][i])
                                for i in sel), kind)
        assert r["number_of_snapshots"] == int(d[f"{name}_n"])
        np.testing.assert_array_equal(r["selected_time_interval"], d[f"{name}_interval"])
        for key in ("k", "energy_mean", "energy_std", "enstrophy_mean", "enstrophy_std"):
            np.testing.assert_array_equal(r[key], d[f"{name}_{key}"], err_msg=f"{name} {key}")
        assert r["high_k_energy_ratio"] == float(d[f"{name}_hk_energy"])
        assert r["high_k_enstrophy_ratio"] == float(d[f"{name}_hk_enstrophy"])
