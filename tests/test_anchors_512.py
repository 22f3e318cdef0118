"""Parity at the full 512^2 size of the benchmark configurations.

1. The reference publishes the summary statistics of five 512^2 Riemann runs
   (FP64 CuPy runs of its own ``run_riemann``: configuration 3 centred with
   mn 0.015 every step and with mn 0.01 at CFL 0.25, configuration 3 at
   x0 = y0 = 0.8 to t = 0.3 and to t = 0.85, configuration 6 to t = 0.25;
   ``results/riemann_config*/<run>/diagnostics.json``, copied into
   ``tests/golden/published_riemann_512.json`` by ``make_anchors_512.py``).
   Each run is repeated here through the mirror's ``run_riemann`` in the plain
   FP64 form and in the FP32-bulk form: the step count and the number of
   hyperviscosity applications must be equal, the density and pressure
   extrema, the largest |vorticity| and the final sensor fraction within the
   tolerances below.
2. Reruns of those configurations through the reference's NumPy
   ``run_riemann`` (``tests/golden/rerun_riemann_*.npz``): the same
   diagnostics plus 16 x 16-cell block means of the final state.
3. 1000 steps of the production 512^2 forced HIT with the reference's NumPy
   forcing-noise stream against the reference's own run of the same 1000
   steps (``tests/golden/hit512_1000.npz``): kinetic energy and enstrophy
   within 1e-4 relative in both precision forms, the other diagnostics and
   the block means of the final state within the stated tolerances.
4. A few 512^2 steps of both benchmark configurations against the oracle.
"""

import json
import math
from pathlib import Path

import numpy as np
import pytest
import torch

from hit_solver_b200 import _lib
from hit_solver_b200.problems import riemann as R

GOLD = Path(__file__).resolve().parent / "golden"
PUBLISHED = json.loads((GOLD / "published_riemann_512.json").read_text())
CLASSES = {3: R.RiemannConfig3, 6: R.RiemannConfig6}

BLOCK = 16
# Errors against the reference's NumPy reruns.  The problems amplify roundoff
# (see test_rerun_distance_is_the_problems_own_spread), so each limit is about
# 2.5x the largest error measured on a B200 over ten runs per configuration:
# both precision forms, each from the initial state and from four 1e-14
# perturbations of its density.  Largest measured (c3 / c308 / c6):
#   block_rms  rms over the 16 x 16 block means of (mirror - NumPy), relative
#              to the rms of NumPy's: 2.1e-3 / 5.1e-3 / 2.0e-3
#   block_means  largest block difference relative to the largest block
#              mean: 1.7e-2 / 3.5e-2 / 2.0e-2
#   density_min 2.3e-4 / 2.6e-4 / 8.7e-2; density_max 1.4e-3 / 2.4e-3 / 1.5e-3
#   pressure_max 1.8e-3 / 4.7e-3 / 1.2e-2; max_abs_vorticity 7.7e-3 / 1.7e-2 /
#   4.4e-2; sensor_fraction_abs 1.8e-4 / 2.2e-4 / 1.2e-3
RERUN_TOL = {
    "c3_mn0015": dict(block_rms=5e-3, block_means=4e-2, density_min=6e-4, density_max=4e-3,
                      pressure_max=5e-3, max_abs_vorticity=2e-2, sensor_fraction_abs=1e-3),
    "c308_t03": dict(block_rms=1.2e-2, block_means=8e-2, density_min=1e-3, density_max=6e-3,
                     pressure_max=1.2e-2, max_abs_vorticity=4e-2, sensor_fraction_abs=1e-3),
    "c6_t025": dict(block_rms=5e-3, block_means=5e-2, density_min=0.2, density_max=4e-3,
                    pressure_max=3e-2, max_abs_vorticity=0.1, sensor_fraction_abs=3e-3),
}
# a 1e-14 relative perturbation of the initial density alone moves the final
# block means of the mirror's own FP64 run by 1.0e-3 (c308), 1.6e-3 (c3),
# 1.0e-3 (c6) in block_rms; the distance to the NumPy run is 3.4x, 1.3x, 1.2x
# that spread
PERTURBATION = 1e-14
SPREAD_FACTOR = 8.0


def _config(tag, precision):
    c = PUBLISHED[tag]["config"]
    kw = {k: v for k, v in c.items()}
    number = 3 if tag.startswith("c3") else 6
    cls = CLASSES[number]
    if tag.startswith("c308"):
        cls = R.RiemannConfig3Offset08
    return cls(backend="b200", precision=precision, progress_every=10**9, **kw)


def _block_means(q):
    c, ny, nx = q.shape
    return q.reshape(c, ny // BLOCK, BLOCK, nx // BLOCK, BLOCK).mean(axis=(2, 4))


@pytest.fixture(scope="module")
def riemann_runs():
    out = {}
    for tag in sorted(PUBLISHED):
        for precision in ("fp64", "fp32-bulk"):
            q, diag = R.run_riemann(_config(tag, precision))
            torch.cuda.synchronize()
            out[tag, precision] = (q.double().cpu().numpy(), diag)
    return out


def _rel(a, b):
    return abs(a - b) / abs(b)


def _rms_rel(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))


def _errors(got, q, want_diag, want_blocks=None):
    e = {k: _rel(getattr(got, k), float(want_diag[k]))
         for k in ("density_min", "density_max", "pressure_max", "max_abs_vorticity")}
    e["sensor_fraction_abs"] = abs(got.final_sensor_fraction - float(want_diag["final_sensor_fraction"]))
    if want_blocks is not None:
        bm = _block_means(q)
        e["block_means"] = float(np.max(np.abs(bm - want_blocks)) / np.max(np.abs(want_blocks)))
        e["block_rms"] = _rms_rel(bm, want_blocks)
    return e


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32-bulk"])
@pytest.mark.parametrize("tag", sorted(PUBLISHED))
def test_published_riemann_512(riemann_runs, tag, precision):
    """The published runs' step and hyperviscosity counts are reproduced
    exactly.  Their field statistics are reported, not asserted: the
    reference's current code does not reproduce them itself (its NumPy rerun
    of these configurations, tests/golden/rerun_riemann_*.npz, differs from
    the published CuPy values by up to 26 % in the density minimum, and the
    published configuration-3 run hits the pressure floor where the rerun
    does not), so they come from an earlier version of the scheme."""
    want = PUBLISHED[tag]["diagnostics"]
    q, got = riemann_runs[tag, precision]
    e = _errors(got, q, want)
    print(f"\n[measured] published {tag} {precision}: " + " ".join(f"{k} {v:.2e}" for k, v in e.items()))
    assert got.steps == want["steps"]
    assert got.hyperviscosity_applications == want["hyperviscosity_applications"]
    assert abs(got.time - want["time"]) <= 1e-12
    assert not got.has_nonfinite and got.density_positive and got.pressure_positive


RERUNS = sorted(p.stem.replace("rerun_riemann_", "") for p in GOLD.glob("rerun_riemann_*.npz"))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32-bulk"])
@pytest.mark.parametrize("tag", RERUNS)
def test_numpy_rerun_riemann_512(riemann_runs, tag, precision):
    """Against the reference's NumPy run of the same configuration to its
    final time: step and hyperviscosity counts exact; 16 x 16 block means of
    the final state, the sensor fraction and the density / pressure extrema
    within the tolerances of RERUN_TOL.  The slip lines of these problems
    are Kelvin-Helmholtz unstable, so roundoff-level differences between two
    FP64 implementations grow over a thousand steps into visible differences
    of local extrema (measured: density minimum of configuration 6 within 9 %
    of the NumPy run's); smooth functionals of the field stay close, and
    test_rerun_distance_is_the_problems_own_spread shows the distance is
    of the size a 1e-14 perturbation of the initial state produces."""
    ref = np.load(GOLD / f"rerun_riemann_{tag}.npz")
    q, got = riemann_runs[tag, precision]
    want = {k[5:]: ref[k] for k in ref.files if k.startswith("diag_")}
    e = _errors(got, q, want, ref["block_means"])
    print(f"\n[measured] rerun {tag} {precision}: " + " ".join(f"{k} {v:.2e}" for k, v in e.items()))
    assert got.steps == int(want["steps"])
    assert got.hyperviscosity_applications == int(want["hyperviscosity_applications"])
    tol = RERUN_TOL[tag]
    for key, lim in tol.items():
        assert e[key] <= lim, (key, e[key], lim)


@pytest.mark.gpu
@pytest.mark.parametrize("tag", RERUNS)
def test_rerun_distance_is_the_problems_own_spread(riemann_runs, tag):
    """The mirror's FP64 run restarted from its initial state with the density
    multiplied by 1 + 1e-14 u (u uniform in [-1/2, 1/2), seeded) ends this far
    (block_rms) from the unperturbed run; the NumPy rerun must lie within
    SPREAD_FACTOR times that spread, and the spread itself must be far above
    the perturbation (the problem amplifies roundoff: two correct FP64
    implementations cannot agree more closely than this)."""
    cfg = _config(tag, "fp64")
    s = R.RiemannSolver(cfg)
    g = torch.Generator(device="cpu").manual_seed(1)
    u = (torch.rand(s.q.shape[1:], generator=g, dtype=torch.float64) - 0.5).to(s.q.device)
    s.q[0] *= 1 + PERTURBATION * u
    s.advance(s.n_steps)
    torch.cuda.synchronize()
    base = _block_means(riemann_runs[tag, "fp64"][0])
    spread = _rms_rel(_block_means(s.q.double().cpu().numpy()), base)
    dist = _rms_rel(base, np.load(GOLD / f"rerun_riemann_{tag}.npz")["block_means"])
    print(f"\n[measured] spread {tag}: perturbed {spread:.2e} NumPy {dist:.2e} ratio {dist / spread:.2f}")
    assert spread > 1e6 * PERTURBATION
    assert dist <= SPREAD_FACTOR * spread


# ---- 512^2 production HIT, 1000 steps, the reference's own noise stream ---------------------
HIT_STEPS = 1000
HIT_KW = dict(nx=512, ny=512, tfinal=1e9, cfl=0.05, target_mach=0.25, initial_kmin=3,
              initial_kmax=5, forcing_kmin=3.0, forcing_kmax=5.0, forcing_correlation_time=0.5,
              forcing_alpha_memory=0.2, target_energy_injection=1e-3, mach_control=True,
              mach_control_target=0.25, viscosity=7.5e-4, hyperviscosity_mn=0.002,
              hyperviscosity_interval=5, large_scale_drag=0.10, large_scale_drag_kmax=2.0,
              cooling_time=5.0, forcing_seed=1234, max_steps=HIT_STEPS)
# kinetic energy and enstrophy: the 1e-4 of the accuracy target; the other
# moments the same; block means of the state (relative to their largest)
HIT_TOL = {"fp64": dict(diag=1e-4, state=1e-6), "fp32-bulk": dict(diag=1e-4, state=1e-4)}


@pytest.mark.gpu
@pytest.mark.skipif(not (GOLD / "hit512_1000.npz").exists(), reason="reference HIT anchor not generated")
@pytest.mark.parametrize("precision", ["fp64", "fp32-bulk"])
def test_hit_512_1000_steps_match_reference(precision):
    from hit_solver_b200.hit2d import HIT2DConfig, HITSolver, compute_diagnostics

    ref = np.load(GOLD / "hit512_1000.npz")
    s = HITSolver(HIT2DConfig(precision=precision, forcing_noise="numpy", **HIT_KW))
    s.advance(HIT_STEPS)
    torch.cuda.synchronize()
    sc = s.plan.scalars()
    assert int(sc[_lib.S_STEP]) == HIT_STEPS and int(sc[_lib.S_STATUS]) == 0
    t_ref = float(ref["time"])
    d = compute_diagnostics(s.q, s.equation, s.domain)
    tol = HIT_TOL[precision]
    errs = {"time": _rel(sc[_lib.S_TIME], t_ref)}
    for key in ("kinetic_energy", "Kx", "Ky", "rms_velocity", "turbulent_mach", "mean_pressure"):
        errs[key] = _rel(d[key], float(ref[f"diag{HIT_STEPS}_{key}"]))
    errs["enstrophy"] = _rel(d["vorticity_rms"] ** 2, float(ref[f"diag{HIT_STEPS}_vorticity_rms"]) ** 2)
    errs["injected_power"] = _rel(sc[_lib.S_F_INJECTED], float(ref["info_injected_power"]))
    bm = _block_means(s.q.double().cpu().numpy())
    want = ref["block_means"]
    errs["state"] = float(np.max(np.abs(bm - want)) / np.max(np.abs(want)))
    print(f"\n[measured] HIT 512^2 x {HIT_STEPS} {precision}: " +
          " ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    for key, e in errs.items():
        if key == "state":
            assert e <= tol["state"], (key, e)
        else:
            assert e <= tol["diag"], (key, e)


# ---- a few 512^2 steps against the oracle ----------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("fp32-bulk", 1e-5)])
def test_riemann_c3_512_steps_match_oracle(precision, tol):
    """Benchmark configuration 2 (Riemann C3, 512^2, mn 0.001 every step,
    shear off, CFL 0.4): 3 steps against the oracle (about 12 s of one host
    core)."""
    from oracle import hit_oracle as O
    from tests.gpu_util import host, rel_err

    cfg = R.RiemannConfig3(nx=512, ny=512, shear_threshold=None, precision=precision)
    s = R.RiemannSolver(cfg)
    s.advance(3)
    torch.cuda.synchronize()
    want, _, steps, _ = O.riemann_run(O.RiemannParams(number=3, nx=512, ny=512), max_steps=3)
    assert steps == 3 and int(s.plan.scalars()[_lib.S_STEP]) == 3
    err = rel_err(host(s.q), want)
    print(f"\n[measured] Riemann C3 512^2 x 3 {precision}: state rel err {err:.2e}")
    assert err < tol


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("fp32-bulk", 1e-5)])
def test_hit_512_steps_match_oracle(precision, tol):
    """Benchmark configuration 3 (production HIT, 512^2) with the reference's
    noise stream: 2 steps against the oracle (about 10 s of one host core)."""
    from hit_solver_b200.hit2d import HIT2DConfig, HITSolver
    from oracle import hit_oracle as O
    from tests.gpu_util import host, rel_err

    kw = dict(HIT_KW, max_steps=2)
    s = HITSolver(HIT2DConfig(precision=precision, forcing_noise="numpy", **kw))
    s.advance(2)
    torch.cuda.synchronize()
    okw = {k: v for k, v in kw.items() if k in O.HITParams.__dataclass_fields__}
    want, _, steps, _ = O.hit_run(O.HITParams(**okw), max_steps=2)
    assert steps == 2
    err = rel_err(host(s.q), want)
    print(f"\n[measured] HIT 512^2 x 2 {precision}: state rel err {err:.2e}")
    assert err < tol
