"""Helpers shared by the GPU parity tests (oracle side stays on the CPU)."""

import numpy as np
import torch

from oracle import hit_oracle as O


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.detach().cpu().numpy()


def rel_err(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def near_threshold_footprint(q, dx, dy, gamma, prm, periodic, rtol):
    """Nodes whose sensor metric lies within rtol (relative) of its threshold,
    dilated by the sensor width: outside this footprint the masks of two
    precisions must agree exactly."""
    div, vort, jumps = O.sensor_metrics(q, dx, dy, gamma, periodic)
    near = np.zeros(div.shape, dtype=bool)
    for j in jumps.values():
        near |= np.abs(j - prm.jump_threshold) <= rtol * prm.jump_threshold
    div_rms = float(np.sqrt(np.mean(div ** 2)))
    if div_rms > 1e-12:
        lim = -prm.compression_threshold * div_rms
        near |= np.abs(div - lim) <= rtol * abs(lim)
    if prm.shear_threshold is not None and (periodic or prm.shear_threshold > 0):
        vrms = float(np.sqrt(np.mean(vort ** 2)))
        if vrms > 1e-12:
            lim = prm.shear_threshold * vrms
            near |= np.abs(np.abs(vort) - lim) <= rtol * lim
    return O.dilate(near, prm.width, periodic), int(near.sum())


def periodic_state(nx, ny, blob=True, seed=1234, mach=0.25):
    """HIT initial condition (oracle) plus an optional density/pressure blob."""
    q = O.hit_initial_state(nx, ny, 2 * np.pi, 1.4, mach, 3, 5, seed)
    if blob:
        rho, u, v, p = O.primitives(q, 1.4)
        X, Y = np.meshgrid(O.cell_centres(0, 2 * np.pi, nx), O.cell_centres(0, 2 * np.pi, ny))
        inside = (X - 2.0) ** 2 + (Y - 3.5) ** 2 < 1.0
        rho = np.where(inside, 1.6, rho)
        p = np.where(inside, 1.4, p)
        q = O.enforce(O.conservative(rho, u, v, p, 1.4), 1.4)
    return q


def ulp_floor(fn, q, seed=0):
    """The oracle's own sensitivity to a one-ulp relative perturbation of its
    input: rel_err(fn(q (1 + 1e-16 xi)), fn(q)).  The reference's WENO
    smoothness indicators are quadratic forms of raw values whose roundoff
    (~1e-13 absolute on O(1) data) rivals eps = 1e-10 near constant states, so
    its nonlinear weights, and hence its fluxes, move at this level; FP64
    parity is asserted relative to this floor."""
    rng = np.random.default_rng(seed)
    qp = q * (1.0 + 1e-16 * rng.standard_normal(q.shape))
    return rel_err(fn(qp), fn(q))


def fp64_tol(fn, q):
    return max(20.0 * ulp_floor(fn, q), 1e-11)
