"""Initial states built on the device (row: initial conditions on device).

The four-quadrant Riemann states are bit for bit the oracle's (the oracle is
pinned to the reference's own quadrant fixtures).  The HIT streamfunction
initial state uses the reference's phase stream and matches the oracle's to
roundoff (cos and the FFTs are CUDA's and cuFFT's, not NumPy's); a run from
it tracks the oracle's run.
"""

import ctypes
import math

import numpy as np
import pytest
import torch

from hit_solver_b200 import _lib
from oracle import hit_oracle as O

G = 1.4


@pytest.mark.gpu
@pytest.mark.parametrize("cls_name,number,nx,ny", [
    ("RiemannConfig3", 3, 64, 48), ("RiemannConfig6", 6, 33, 20),
    ("RiemannConfig3Offset08", 3, 40, 40), ("RiemannConfig3", 3, 1024, 1024)])
def test_riemann_quadrants_bit_exact(cls_name, number, nx, ny):
    from hit_solver_b200.problems import riemann as R

    cfg = getattr(R, cls_name)(nx=nx, ny=ny)
    got = cfg.initial_state().cpu().numpy()
    want = O.riemann_initial_state(number, nx, ny, cfg.x_split, cfg.y_split, G)
    np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny,kmin,kmax,length,mach,seed", [
    (64, 64, 3, 5, 2 * math.pi, 0.25, 1234), (96, 80, 1, 3, 2 * math.pi, 0.1, 7),
    (128, 128, 2, 6, 1.0, 0.3, 99), (512, 512, 3, 5, 2 * math.pi, 0.25, 5)])
def test_hit_streamfunction_state_matches_oracle(nx, ny, kmin, kmax, length, mach, seed):
    from hit_solver_b200.equations import EulerEquation2D
    from hit_solver_b200.hit2d import HIT2DConfig, create_grid, initialize_hit_2d_device

    cfg = HIT2DConfig(nx=nx, ny=ny, length=length, target_mach=mach, initial_kmin=kmin,
                      initial_kmax=kmax, forcing_seed=seed)
    dom = create_grid(cfg)[0]
    eq = EulerEquation2D(gamma=G)
    q = eq.enforce_physical_state(initialize_hit_2d_device(cfg, dom, eq, np.random.default_rng(seed)))
    want = O.hit_initial_state(nx, ny, length, G, mach, kmin, kmax, seed)
    got = q.cpu().numpy()
    for c in range(4):
        scale = max(float(np.max(np.abs(want[c]))), 1e-300)
        assert float(np.max(np.abs(got[c] - want[c]))) <= 1e-12 * scale, c


@pytest.mark.gpu
def test_hit_run_from_device_initial_state():
    """Six production-physics steps from the device-built initial state track
    the oracle's run from its own (host) initial state."""
    from hit_solver_b200.hit2d import HIT2DConfig, HITSolver

    kw = dict(cfl=0.05, target_mach=0.25, forcing_correlation_time=0.5, mach_control=True,
              mach_control_target=0.25, viscosity=7.5e-4, large_scale_drag=0.1, cooling_time=5.0)
    cfg = HIT2DConfig(nx=48, ny=40, tfinal=1.0, initial_kmin=3, initial_kmax=5, forcing_kmin=3.0,
                      forcing_kmax=5.0, hyperviscosity_mn=0.002, initial_condition="device", **kw)
    s = HITSolver(cfg)
    s.advance(6)
    want, _t, steps, _info = O.hit_run(O.HITParams(nx=48, ny=40, tfinal=1.0, **kw), max_steps=6)
    got = s.q.cpu().numpy()
    assert float(np.max(np.abs(got - want)) / np.max(np.abs(want))) < 1e-10


def test_initial_state_abi_rejects_bad_arguments():
    lib = _lib.load()
    buf = ctypes.create_string_buffer(256)
    p = ctypes.addressof(buf)
    states = (ctypes.c_double * 16)(*([1.0] * 16))
    assert lib.hitb200_hit_streamfunction(p, 1, 0, 8, 0.0, 0.1, 0.0, 0.1, p, None) == _lib.ERR_INVALID
    assert lib.hitb200_hit_streamfunction(None, 2, 8, 8, 0.0, 0.1, 0.0, 0.1, p, None) == _lib.ERR_INVALID
    assert lib.hitb200_hit_streamfunction(p, 1, 8, 8, 0.0, -0.1, 0.0, 0.1, p, None) == _lib.ERR_INVALID
    assert lib.hitb200_hit_compose(p, p, 8, 8, G, 0.1, 1.0, p, p, p, 8, None) == _lib.ERR_INVALID
    assert lib.hitb200_hit_compose(p, p, 8, 8, 1.0, 0.1, 1.0, p, p, p, 1 << 20, None) == _lib.ERR_INVALID
    assert lib.hitb200_riemann_initial_state(None, 8, 8, 0.0, 0.1, 0.0, 0.1, 0.5, 0.5, G, p,
                                             None) == _lib.ERR_INVALID
    assert lib.hitb200_riemann_initial_state(states, 8, 8, 0.0, 0.1, 0.0, 0.1, 0.5, 0.5, 0.9, p,
                                             None) == _lib.ERR_INVALID


def test_initial_modes_follow_the_reference_loop():
    """The host part of the device initial state: modes of the shell in the
    reference's loop order with one phase per mode from the same stream."""
    from hit_solver_b200.hit2d import HIT2DConfig, initial_modes

    cfg = HIT2DConfig(initial_kmin=3, initial_kmax=5)
    m = initial_modes(cfg, np.random.default_rng(1234))
    rng = np.random.default_rng(1234)
    want = []
    for kx in range(-5, 6):
        for ky in range(-5, 6):
            if ky < 0 or (ky == 0 and kx <= 0) or not 3 <= math.hypot(kx, ky) <= 5:
                continue
            want.append((kx, ky, 1.0 / (kx * kx + ky * ky), rng.uniform(0.0, 2 * math.pi)))
    np.testing.assert_array_equal(m, np.asarray(want))
