"""CPU oracle for the HIT_Solver RHS / SSP-RK3 hot path (NumPy, FP64).

TEST INFRASTRUCTURE ONLY.  Nothing under ``hit_solver_b200/`` imports this
module.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may call it, and there only as the checker (or as the
timed CPU baseline), never as the thing measured or shipped.

This is a restatement, in my own code, of the arithmetic that the reference
(FernandoAtienza/HIT_Solver) performs on the hot path.  Every function cites
the reference file:line it follows.  The restatement is pinned against golden
vectors that the reference itself produced (``tests/golden/make_golden.py``
imports the reference, runs it, and commits the results as ``.npz``
fixtures; ``tests/test_oracle_golden.py`` checks this module against them).

Boundary handling is expressed through one helper, :func:`shift`, that reads
``a[i + k]`` along an axis either with periodic wrap-around (HIT) or with the
index clamped to the edge (Riemann outflow, the reference's ``take_clipped``).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

RHO_FLOOR = 1e-10
P_FLOOR = 1e-10
COMPACT_ALPHA = 3.0 / 8.0


# --------------------------------------------------------------------------
# Index helpers
# --------------------------------------------------------------------------
def shift(a: np.ndarray, k: int, axis: int, periodic: bool) -> np.ndarray:
    """Return b with b[..., i, ...] = a[..., i + k, ...] along ``axis``.

    Periodic: index taken modulo n (same as ``np.roll(a, -k)``).
    Non-periodic: index clamped to [0, n-1]
    (``OOP/problems/riemann_config3.py:121-125`` ``take_clipped``).
    """
    n = a.shape[axis]
    idx = np.arange(n) + k
    idx = np.mod(idx, n) if periodic else np.clip(idx, 0, n - 1)
    return np.take(a, idx, axis=axis)


# --------------------------------------------------------------------------
# Thermodynamics  (OOP/equations.py:126-208, OOP/parallel/equations.py:11-73)
# --------------------------------------------------------------------------
def primitives(q: np.ndarray, gamma: float):
    """rho, u, v, p with the 1e-10 floors (``OOP/equations.py:136-145``)."""
    rho = np.maximum(q[0], RHO_FLOOR)
    u = q[1] / rho
    v = q[2] / rho
    kinetic = 0.5 * rho * (u ** 2 + v ** 2)
    p = (gamma - 1.0) * (q[3] - kinetic)
    return rho, u, v, np.maximum(p, P_FLOOR)


def conservative(rho, u, v, p, gamma: float) -> np.ndarray:
    """[rho, rho u, rho v, E] from primitives (``OOP/equations.py:147-163``)."""
    rho, u, v, p = np.broadcast_arrays(rho, u, v, p)
    rho = np.maximum(rho, RHO_FLOOR)
    p = np.maximum(p, P_FLOOR)
    out = np.zeros((4,) + rho.shape, dtype=np.result_type(rho, u, v, p))
    out[0] = rho
    out[1] = rho * u
    out[2] = rho * v
    out[3] = p / (gamma - 1.0) + 0.5 * rho * (u ** 2 + v ** 2)
    return out


def enforce(q: np.ndarray, gamma: float) -> np.ndarray:
    """Density floor, momentum rebuilt from the floored density, and E reset
    to floor pressure where p <= floor (``OOP/equations.py:165-181``)."""
    rho = np.maximum(q[0], RHO_FLOOR)
    u = q[1] / rho
    v = q[2] / rho
    kinetic = 0.5 * rho * (u ** 2 + v ** 2)
    p = (gamma - 1.0) * (q[3] - kinetic)
    out = np.empty_like(q)
    out[0] = rho
    out[1] = rho * u
    out[2] = rho * v
    out[3] = np.where(p > P_FLOOR, q[3], P_FLOOR / (gamma - 1.0) + kinetic)
    return out


def flux(q: np.ndarray, gamma: float, axis: int) -> np.ndarray:
    """Euler flux along x (axis=-1) or y (axis=-2) (``OOP/equations.py:183-199``)."""
    rho, u, v, p = primitives(q, gamma)
    out = np.zeros_like(q)
    if axis == -1:
        out[0] = q[1]
        out[1] = rho * u ** 2 + p
        out[2] = rho * u * v
        out[3] = (q[3] + p) * u
    else:
        out[0] = q[2]
        out[1] = rho * u * v
        out[2] = rho * v ** 2 + p
        out[3] = (q[3] + p) * v
    return out


def sound_speed(rho, p, gamma):
    return np.sqrt(gamma * p / rho)


# --------------------------------------------------------------------------
# Shock sensor
# --------------------------------------------------------------------------
def jump_metric(a: np.ndarray, axis: int, periodic: bool) -> np.ndarray:
    """max(left jump, right jump, curvature), each relative to local magnitude
    plus eps = 1e-14 + 1e-12 max|a| over the whole field.

    Periodic: ``OOP/spatial_operator.py:147-166``.  Non-periodic: one-sided
    pair jumps at the ends and clamped curvature
    (``OOP/problems/riemann_config3.py:128-146``); clamping the neighbour index
    makes the missing edge jump exactly 0, which is what the reference's
    zero-initialised ``jumps`` array gives.
    """
    eps = 1e-14 + 1e-12 * np.max(np.abs(a))
    ap = shift(a, 1, axis, periodic)
    am = shift(a, -1, axis, periodic)
    right = np.abs(ap - a) / (np.abs(ap) + np.abs(a) + eps)
    left = np.abs(a - am) / (np.abs(a) + np.abs(am) + eps)
    curv = np.abs(ap - 2.0 * a + am) / (np.abs(ap) + 2.0 * np.abs(a) + np.abs(am) + eps)
    return np.maximum(np.maximum(left, right), curv)


def central_diff(a: np.ndarray, h: float, axis: int, periodic: bool) -> np.ndarray:
    """Second-order central difference; one-sided first-order at the ends when
    not periodic (``OOP/spatial_operator.py:265-268``,
    ``OOP/problems/riemann_config3.py:268-275``)."""
    if periodic:
        return (shift(a, 1, axis, True) - shift(a, -1, axis, True)) / (2.0 * h)
    m = np.moveaxis(a, axis, -1)
    d = np.empty_like(m)
    d[..., 1:-1] = (m[..., 2:] - m[..., :-2]) / (2.0 * h)
    d[..., 0] = (m[..., 1] - m[..., 0]) / h
    d[..., -1] = (m[..., -1] - m[..., -2]) / h
    return np.moveaxis(d, -1, axis)


def dilate(mask: np.ndarray, width: int, periodic: bool) -> np.ndarray:
    """(2w+1)^2 box dilation, wrapped (``OOP/spatial_operator.py:169-176``) or
    clipped at the edges (``OOP/problems/riemann_config3.py:149-162``)."""
    ny, nx = mask.shape
    out = mask.copy()
    if periodic:
        for dy in range(-width, width + 1):
            rows = np.roll(mask, dy, axis=0)
            for dx in range(-width, width + 1):
                out |= np.roll(rows, dx, axis=1)
        return out
    for dy in range(-width, width + 1):
        for dx in range(-width, width + 1):
            ys, yd = slice(max(0, -dy), min(ny, ny - dy)), slice(max(0, dy), min(ny, ny + dy))
            xs, xd = slice(max(0, -dx), min(nx, nx - dx)), slice(max(0, dx), min(nx, nx + dx))
            out[yd, xd] |= mask[ys, xs]
    return out


@dataclass(frozen=True)
class SensorParams:
    width: int = 4
    compression_threshold: float = 2.5
    jump_threshold: float = 0.04
    shear_threshold: float | None = None
    boundary_guard: int = 0


def sensor_metrics(q, dx, dy, gamma, periodic):
    """Per-node quantities the sensor thresholds (used by tests to find nodes
    that sit within roundoff of a threshold)."""
    rho, u, v, p = primitives(q, gamma)
    du_dx = central_diff(u, dx, -1, periodic)
    du_dy = central_diff(u, dy, -2, periodic)
    dv_dx = central_diff(v, dx, -1, periodic)
    dv_dy = central_diff(v, dy, -2, periodic)
    div = du_dx + dv_dy
    vort = dv_dx - du_dy
    e = p / (rho * (gamma - 1.0))
    jumps = {
        "rho": np.maximum(jump_metric(rho, -1, periodic), jump_metric(rho, -2, periodic)),
        "p": np.maximum(jump_metric(p, -1, periodic), jump_metric(p, -2, periodic)),
        "e": np.maximum(jump_metric(e, -1, periodic), jump_metric(e, -2, periodic)),
    }
    return div, vort, jumps


def sensor(q: np.ndarray, dx: float, dy: float, gamma: float, prm: SensorParams,
           periodic: bool, raw: bool = False) -> np.ndarray:
    """Hybrid-switch node mask.

    Periodic: ``OOP/spatial_operator.py:263-304`` (shear only when the
    threshold is not None).  Non-periodic: ``OOP/problems/riemann_config3.py:
    288-326`` (shear only when the threshold is not None and > 0; a band of
    ``boundary_guard`` nodes along every edge is forced on before dilation).
    """
    div, vort, jumps = sensor_metrics(q, dx, dy, gamma, periodic)
    div_rms = float(np.sqrt(np.mean(div ** 2)))
    mask = np.zeros(div.shape, dtype=bool)
    if div_rms > 1e-12:
        mask |= div < -prm.compression_threshold * div_rms
    shear_on = prm.shear_threshold is not None and (periodic or prm.shear_threshold > 0.0)
    if shear_on:
        vort_rms = float(np.sqrt(np.mean(vort ** 2)))
        if vort_rms > 1e-12:
            mask |= np.abs(vort) > prm.shear_threshold * vort_rms
    for name in ("rho", "p", "e"):
        mask |= jumps[name] > prm.jump_threshold
    if not periodic and prm.boundary_guard:
        g = prm.boundary_guard
        mask[:g, :] = True
        mask[-g:, :] = True
        mask[:, :g] = True
        mask[:, -g:] = True
    if raw:
        return mask
    return dilate(mask, prm.width, periodic)


# --------------------------------------------------------------------------
# Interface fluxes
# --------------------------------------------------------------------------
# Candidate-polynomial weights of the four 4-point WENO7 stencils, and the
# reference's smoothness-indicator quadratic forms, written as upper-triangular
# coefficient tables: IS = sum_{a<=b} T[a][b] * w_a * w_b over the stencil's
# four values w.  Stencil k uses v_{k+1}..v_{k+4}
# (``OOP/spatial_operator.py:87-124``).  Note T0[0][0] = 544: the reference
# writes 544 where the Balsara-Shu coefficient is 547; it is kept as is.
_WENO_POLY = (
    (-1 / 4, 13 / 12, -23 / 12, 25 / 12),
    (1 / 12, -5 / 12, 13 / 12, 1 / 4),
    (-1 / 12, 7 / 12, 7 / 12, -1 / 12),
    (1 / 4, 13 / 12, -5 / 12, 1 / 12),
)
_WENO_IS = (
    ((544, -3882, 4642, -1854), (7043, -17246, 7042), (11003, -9402), (2107,)),
    ((267, -1642, 1602, -494), (2843, -5966, 1922), (3443, -2522), (547,)),
    ((547, -2522, 1922, -494), (3443, -5966, 1602), (2843, -1642), (267,)),
    ((2107, -9402, 7042, -1854), (11003, -17246, 4642), (7043, -3882), (547,)),
)
_WENO_D = (1 / 35, 12 / 35, 18 / 35, 4 / 35)
_WENO_EPS = 1e-10


def weno7(v):
    """Seventh-order WENO value at the right face of v[3] from v[0..6]
    (``OOP/spatial_operator.py:87-124``)."""
    num = 0.0
    den = 0.0
    for k in range(4):
        w = v[k:k + 4]
        cand = sum(c * x for c, x in zip(_WENO_POLY[k], w))
        smooth = 0.0
        for a in range(3):
            smooth = smooth + w[a] * sum(c * w[a + j] for j, c in enumerate(_WENO_IS[k][a]))
        smooth = smooth + _WENO_IS[k][3][0] * w[3] ** 2
        alpha = _WENO_D[k] / (_WENO_EPS + smooth) ** 2
        num = num + alpha * cand
        den = den + alpha
    return num / den


_A1, _B1, _C1 = 25 / 32, 1 / 20, -1 / 480


def interface_fluxes(qa, fa, node_mask, alpha, periodic, scheme="hybrid"):
    """Hybrid interface fluxes H along the last axis.

    Returns H with one entry per interface i+1/2 for i = -1 .. n-1 (n+1
    entries; entry 0 is the face left of node 0).  Periodic
    (``OOP/spatial_operator.py:179-211, 321-342``): the 6-point compact
    interface flux, WENO7 of the global Lax-Friedrichs split f+- =
    (F +- alpha q)/2, the compactised WENO flux (3/8 W_{i-1} + W_i + 3/8
    W_{i+1}), selected where node i or i+1 is flagged.  Non-periodic
    (``OOP/problems/riemann_config3.py:165-222, 344-357``): the same with
    clamped stencils and n+1 faces; ``scheme="weno"`` uses the WENO flux on
    every face.
    """
    n = qa.shape[-1]
    fp = 0.5 * (fa + alpha * qa)
    fm = 0.5 * (fa - alpha * qa)
    il = np.arange(-1, n)  # left node of each face

    def take(a, idx):
        idx = np.mod(idx, n) if periodic else np.clip(idx, 0, n - 1)
        return np.take(a, idx, axis=-1)

    smooth = (_C1 * (take(fa, il + 3) + take(fa, il - 2))
              + (_B1 + _C1) * (take(fa, il + 2) + take(fa, il - 1))
              + (_A1 + _B1 + _C1) * (take(fa, il + 1) + take(fa, il)))
    w = (weno7([take(fp, il + k) for k in range(-3, 4)])
         + weno7([take(fm, il + k) for k in range(4, -3, -1)]))
    # compactified WENO flux; neighbour faces wrap (periodic) or clamp.
    nf = n + 1
    f_idx = np.arange(nf)
    if periodic:
        # face -1/2 is face n-1/2: neighbours of face k are faces k+-1 with
        # the periodic identification of entries 0 and n.
        wn = w[..., 1:]                      # faces 1/2 .. n-1/2 (n unique faces)
        up = np.take(wn, np.mod(f_idx, n), axis=-1)        # W_{k+1}: entry k+1 -> wn[k]
        dn = np.take(wn, np.mod(f_idx - 2, n), axis=-1)    # W_{k-1}: entry k-1 -> wn[k-2]
    else:
        up = np.take(w, np.clip(f_idx + 1, 0, nf - 1), axis=-1)
        dn = np.take(w, np.clip(f_idx - 1, 0, nf - 1), axis=-1)
    what = COMPACT_ALPHA * up + w
    what = what + COMPACT_ALPHA * dn
    if scheme == "weno":
        return what
    flagged = take(node_mask, il) | take(node_mask, il + 1)
    return np.where(flagged[None, ...], what, smooth)


def compact_solve_periodic(raw: np.ndarray) -> np.ndarray:
    """Solve 3/8 d_{i-1} + d_i + 3/8 d_{i+1} = raw_i cyclically along the last
    axis; circulant, so diagonal in Fourier space
    (``OOP/spatial_operator.py:228-249``)."""
    n = raw.shape[-1]
    eig = 1.0 + 2.0 * COMPACT_ALPHA * np.cos(2.0 * np.pi * np.fft.fftfreq(n))
    return np.fft.ifft(np.fft.fft(raw, axis=-1) / eig, axis=-1).real


def compact_solve_dirichlet(raw: np.ndarray) -> np.ndarray:
    """Thomas solve of the same system with identity first and last rows
    (``OOP/problems/riemann_config3.py:226-265``)."""
    n = raw.shape[-1]
    a = COMPACT_ALPHA
    lower = np.full(n, a)
    upper = np.full(n, a)
    lower[0] = upper[0] = lower[-1] = upper[-1] = 0.0
    r = raw.reshape(-1, n)
    cp = np.zeros(n)
    dp = np.zeros_like(r)
    cp[0] = upper[0]
    dp[:, 0] = r[:, 0]
    for i in range(1, n):
        den = 1.0 - lower[i] * cp[i - 1]
        cp[i] = upper[i] / den if i < n - 1 else 0.0
        dp[:, i] = (r[:, i] - lower[i] * dp[:, i - 1]) / den
    out = np.zeros_like(dp)
    out[:, -1] = dp[:, -1]
    for i in range(n - 2, -1, -1):
        out[:, i] = dp[:, i] - cp[i] * out[:, i + 1]
    return out.reshape(raw.shape)


def lf_alpha(q, gamma, axis):
    """Global Lax-Friedrichs speed max(|u_n| + c) (``OOP/spatial_operator.py:
    329-332``)."""
    rho, u, v, p = primitives(q, gamma)
    un = u if axis == -1 else v
    return float(np.max(np.abs(un) + sound_speed(rho, p, gamma)))


def axis_derivative(q_safe, mask, h, gamma, axis, periodic, scheme="hybrid"):
    """d(F)/dx_axis by the hybrid compact/WENO scheme on q_safe
    (``OOP/spatial_operator.py:321-342``; non-periodic
    ``OOP/problems/riemann_config3.py:344-357``)."""
    alpha = lf_alpha(q_safe, gamma, axis)
    fa = flux(q_safe, gamma, axis)
    qa, m = q_safe, mask
    if axis == -2:
        qa, fa, m = np.swapaxes(qa, -1, -2), np.swapaxes(fa, -1, -2), m.T
    hf = interface_fluxes(qa, fa, m, alpha, periodic, scheme)
    raw = (hf[..., 1:] - hf[..., :-1]) / h
    d = compact_solve_periodic(raw) if periodic else compact_solve_dirichlet(raw)
    if axis == -2:
        d = np.swapaxes(d, -1, -2)
    return d


def inviscid_rhs(q, dx, dy, gamma, prm: SensorParams, periodic, scheme="hybrid",
                 return_parts=False):
    """-dF/dx - dG/dy (``OOP/spatial_operator.py:344-367``,
    ``OOP/problems/riemann_config3.py:359-369``)."""
    qs = enforce(q, gamma)
    mask = sensor(qs, dx, dy, gamma, prm, periodic)
    d_x = axis_derivative(qs, mask, dx, gamma, -1, periodic, scheme)
    d_y = axis_derivative(qs, mask, dy, gamma, -2, periodic, scheme)
    out = -d_x - d_y
    if return_parts:
        return out, {"mask": mask, "d_x": d_x, "d_y": d_y,
                     "alpha_x": lf_alpha(qs, gamma, -1), "alpha_y": lf_alpha(qs, gamma, -2)}
    return out


def spectral_radius_dt(q, cfl, dx, dy, gamma, remaining=None):
    """cfl / max((|u|+c)/dx + (|v|+c)/dy) (``OOP/spatial_operator.py:369-377``)."""
    rho, u, v, p = primitives(q, gamma)
    c = sound_speed(rho, p, gamma)
    sr = (np.abs(u) + c) / dx
    sr = sr + (np.abs(v) + c) / dy
    dt = cfl / float(np.max(sr))
    if remaining is not None:
        dt = min(dt, remaining)
    return dt


def fixed_time_step(q, cfl, t_end, dx, dy, gamma):
    """dt from the initial state, rounded so n steps land on t_end
    (``OOP/problems/riemann_config3.py:371-378``)."""
    dt = spectral_radius_dt(q, cfl, dx, dy, gamma)
    n = int(np.ceil(t_end / dt))
    return t_end / n, n


# --------------------------------------------------------------------------
# Viscous / thermal terms (OOP/equations.py:211-267)
# --------------------------------------------------------------------------
def viscous_rhs(q, dx, dy, gamma, mu, prandtl=0.72, gas_constant=1.0):
    """Central-difference Navier-Stokes stress and heat-flux divergence on a
    periodic grid (``OOP/equations.py:232-267``)."""
    if mu == 0.0:
        return np.zeros_like(q)
    rho, u, v, p = primitives(q, gamma)
    temp = p / (rho * gas_constant)
    cp = gamma * gas_constant / (gamma - 1.0)
    kappa = mu * cp / prandtl

    def ddx(a):
        return central_diff(a, dx, -1, True)

    def ddy(a):
        return central_diff(a, dy, -2, True)

    du_dx, du_dy, dv_dx, dv_dy = ddx(u), ddy(u), ddx(v), ddy(v)
    div = du_dx + dv_dy
    txx = 2.0 * mu * du_dx - (2.0 / 3.0) * mu * div
    tyy = 2.0 * mu * dv_dy - (2.0 / 3.0) * mu * div
    txy = mu * (du_dy + dv_dx)
    out = np.zeros_like(q)
    out[1] = ddx(txx) + ddy(txy)
    out[2] = ddx(txy) + ddy(tyy)
    efx = u * txx + v * txy + kappa * ddx(temp)
    efy = u * txy + v * tyy + kappa * ddy(temp)
    out[3] = ddx(efx) + ddy(efy)
    return out


# --------------------------------------------------------------------------
# HIT sources (OOP/hit2d.py:264-426)
# --------------------------------------------------------------------------
def wavenumbers(nx, ny, dx, dy):
    kx = 2.0 * np.pi * np.fft.fftfreq(nx, d=dx)
    ky = 2.0 * np.pi * np.fft.fftfreq(ny, d=dy)
    return np.meshgrid(kx, ky, indexing="xy")


def forcing_source(q, fx, fy, gamma):
    """[0, rho fx, rho fy, rho (u fx + v fy)] (``OOP/hit2d.py:264-276``)."""
    rho, u, v, _ = primitives(q, gamma)
    out = np.zeros_like(q)
    out[1] = rho * fx
    out[2] = rho * fy
    out[3] = rho * (u * fx + v * fy)
    return out


def band_filter(a, dx, dy, kmin, kmax):
    """Fourier content with kmin <= |k| <= kmax, k != 0 (``OOP/hit2d.py:352-367``)."""
    ny, nx = a.shape
    kx, ky = wavenumbers(nx, ny, dx, dy)
    k2 = kx ** 2 + ky ** 2
    mag = np.sqrt(k2)
    keep = (mag >= float(kmin)) & (k2 > 0.0)
    if kmax is not None:
        keep &= mag <= float(kmax)
    return np.fft.ifft2(np.where(keep, np.fft.fft2(a), 0.0)).real


def large_scale_kinetic_fraction(q, dx, dy, gamma, kmax):
    """Kinetic-energy fraction of the velocity fluctuations in 0 < |k| <= kmax
    (``OOP/hit2d.py:429-449``)."""
    if kmax <= 0.0:
        return 0.0
    rho, u, v, _ = primitives(q, gamma)
    uf, vf = u - np.mean(u), v - np.mean(v)
    total = float(np.mean(rho * (uf ** 2 + vf ** 2)))
    if total <= np.finfo(float).eps:
        return 0.0
    ul, vl = band_filter(uf, dx, dy, 0.0, kmax), band_filter(vf, dx, dy, 0.0, kmax)
    return float(np.mean(rho * (ul ** 2 + vl ** 2))) / total


def drag_source(q, dx, dy, gamma, coef, kmax):
    """Linear drag on the low-k momentum fluctuations (``OOP/hit2d.py:370-399``)."""
    out = np.zeros_like(q)
    if coef <= 0.0 or kmax <= 0.0:
        return out
    _, u, v, _ = primitives(q, gamma)
    lx = band_filter(q[1] - np.mean(q[1]), dx, dy, 0.0, kmax)
    ly = band_filter(q[2] - np.mean(q[2]), dx, dy, 0.0, kmax)
    out[1] = -coef * lx
    out[2] = -coef * ly
    out[3] = u * out[1] + v * out[2]
    return out


def cooling_source(q, gamma, cooling_time, p_target=None):
    """Uniform energy sink relaxing the mean pressure (``OOP/hit2d.py:402-426``)."""
    out = np.zeros_like(q)
    if cooling_time is None or cooling_time <= 0.0:
        return out
    _, _, _, p = primitives(q, gamma)
    p_ref = 1.0 / gamma if p_target is None else p_target
    out[3] = -((np.mean(p) - p_ref) / (gamma - 1.0)) / cooling_time
    return out


# --------------------------------------------------------------------------
# Hyperviscosity
# --------------------------------------------------------------------------
def _laplacian(a, dx, dy, periodic):
    ax = (shift(a, 1, -1, periodic) - 2.0 * a + shift(a, -1, -1, periodic)) / dx ** 2
    ay = (shift(a, 1, -2, periodic) - 2.0 * a + shift(a, -1, -2, periodic)) / dy ** 2
    return ax + ay


def hyperviscosity(q, active, dx, dy, gamma, mn, weights, periodic):
    """q - mn w h^4 active lap(lap(q)), then enforce.  Periodic Laplacian
    (``OOP/spatial_operator.py:394-435``) or edge-padded
    (``OOP/problems/riemann_config3.py:390-416``)."""
    if active is None:
        raise ValueError("active_mask is required")
    if active.shape != q.shape[-2:]:
        raise ValueError("active_mask shape does not match grid")
    h = min(dx, dy)
    bih = _laplacian(_laplacian(q, dx, dy, periodic), dx, dy, periodic)
    w = np.asarray(weights, dtype=q.dtype)[:, None, None]
    return enforce(q - mn * w * h ** 4 * active[None] * bih, gamma)


def outflow_guard(q, g):
    """Copy cell g (n-g-1) into the g guard cells at each edge, x first, then y
    (``OOP/problems/riemann_config3.py:419-429``)."""
    if g <= 0:
        return q
    out = q.copy()
    out[:, :, :g] = out[:, :, g:g + 1]
    out[:, :, -g:] = out[:, :, -g - 1:-g]
    out[:, :g, :] = out[:, g:g + 1, :]
    out[:, -g:, :] = out[:, -g - 1:-g, :]
    return out


def validate_raw(q, gamma, label="state"):
    """Raise FloatingPointError for non-finite or non-positive raw state
    (``OOP/problems/riemann_config3.py:432-452``)."""
    if not np.all(np.isfinite(q)):
        raise FloatingPointError(f"{label} contains NaN or Inf values")
    rho = q[0]
    u, v = q[1] / rho, q[2] / rho
    p = (gamma - 1.0) * (q[3] - 0.5 * rho * (u ** 2 + v ** 2))
    if not (np.all(np.isfinite(rho)) and np.all(np.isfinite(p))):
        raise FloatingPointError(f"{label} has non-finite density or pressure")
    if np.any(rho <= 0.0):
        raise FloatingPointError(f"{label} contains non-positive density")
    if np.any(p <= 0.0):
        raise FloatingPointError(f"{label} contains non-positive pressure")


# --------------------------------------------------------------------------
# Time integration (OOP/time_operator.py:17-26)
# --------------------------------------------------------------------------
def ssprk3(q0, rhs, dt, clean):
    """Shu-Osher SSP-RK3 with a clean filter after each stage
    (``OOP/time_operator.py:21-26``)."""
    q1 = clean(q0 + dt * rhs(q0))
    q2 = clean(0.75 * q0 + 0.25 * (q1 + dt * rhs(q1)))
    return clean((1.0 / 3.0) * q0 + (2.0 / 3.0) * (q2 + dt * rhs(q2)))


# --------------------------------------------------------------------------
# OU forcing (OOP/forcing.py:11-130) and Mach control (OOP/hit2d.py:279-349)
# --------------------------------------------------------------------------
@dataclass
class ShellOUForcing:
    """Solenoidal OU forcing on k_min <= |k| <= k_max (``OOP/forcing.py``).

    ``noise`` may be given to ``update`` (the real white-noise field); when it
    is None a NumPy ``default_rng(seed)`` draws it, as the reference's NumPy
    path does (``OOP/forcing.py:65-66, 77``).
    """

    nx: int
    ny: int
    dx: float
    dy: float
    k_min: float
    k_max: float
    correlation_time: float = 1.0
    force_rms: float = 1.0
    target_power: float | None = 1e-3
    min_power: float = 1e-6
    max_rescale: float | None = 20.0
    alpha_memory: float = 0.2
    seed: int = 1234
    potential_hat: np.ndarray = field(default=None, init=False, repr=False)
    alpha: float = field(default=1.0, init=False)

    def __post_init__(self):
        if self.k_min < 0.0 or self.k_max <= 0.0 or self.k_min > self.k_max:
            raise ValueError("forcing shell must satisfy 0 <= k_min <= k_max")
        if self.correlation_time <= 0.0:
            raise ValueError("forcing correlation time must be positive")
        if not 0.0 <= self.alpha_memory < 1.0:
            raise ValueError("alpha_memory must be in [0, 1)")
        self.kx, self.ky = wavenumbers(self.nx, self.ny, self.dx, self.dy)
        mag = np.sqrt(self.kx ** 2 + self.ky ** 2)
        self.shell = (mag >= float(self.k_min)) & (mag <= float(self.k_max)) & (mag > 0.0)
        if not np.any(self.shell):
            raise ValueError("forcing shell contains no Fourier modes on this grid")
        self.potential_hat = np.zeros((self.ny, self.nx), dtype=np.complex128)
        self.rng = np.random.default_rng(self.seed)

    def update(self, dt, rho, u, v, noise=None):
        """One OU step; returns fx, fy and the statistics dict
        (``OOP/forcing.py:70-130``)."""
        if dt <= 0.0:
            raise ValueError("forcing update requires dt > 0")
        decay = float(np.exp(-dt / self.correlation_time))
        inc = float(np.sqrt(max(1.0 - decay ** 2, 0.0)))
        if noise is None:
            noise = self.rng.standard_normal((self.ny, self.nx))
        xi_hat = np.where(self.shell, np.fft.fft2(noise), 0.0)
        self.potential_hat = decay * self.potential_hat + inc * xi_hat
        fx = np.fft.ifft2(1j * self.ky * self.potential_hat).real
        fy = np.fft.ifft2(-1j * self.kx * self.potential_hat).real
        rms = float(np.sqrt(np.mean(fx ** 2 + fy ** 2)))
        if self.force_rms <= 0.0:
            fx[...] = 0.0
            fy[...] = 0.0
        elif rms > np.finfo(float).eps:
            fx *= self.force_rms / rms
            fy *= self.force_rms / rms
        p_before = float(np.mean(rho * (fx * u + fy * v)))
        alpha_target = self.alpha
        if self.target_power is not None and abs(p_before) > self.min_power:
            alpha_target = self.target_power / p_before
            if self.max_rescale is not None:
                alpha_target = float(np.clip(alpha_target, -self.max_rescale, self.max_rescale))
            self.alpha = self.alpha_memory * self.alpha + (1.0 - self.alpha_memory) * alpha_target
        elif self.target_power is None:
            self.alpha = 1.0
        fx *= self.alpha
        fy *= self.alpha
        fxx = float(np.mean(fx ** 2))
        fyy = float(np.mean(fy ** 2))
        fxy = float(np.mean(fx * fy))
        den = fxx + fyy
        info = {
            "alpha": float(self.alpha),
            "alpha_target": float(alpha_target),
            "target_power": float("nan") if self.target_power is None else float(self.target_power),
            "power_before_rescale": p_before,
            "injected_power": float(np.mean(rho * (fx * u + fy * v))),
            "Fxx": fxx,
            "Fyy": fyy,
            "Fxy": fxy,
            "A_F": abs(fxx - fyy) / den if den > 0.0 else 0.0,
            "ou_decay": decay,
        }
        return fx, fy, info


def turbulent_mach(rho, u, v, p, gamma):
    """sqrt(mean(u^2+v^2)) / mean(c) (``OOP/hit2d.py:279-290``)."""
    return float(np.sqrt(np.mean(u ** 2 + v ** 2)) / np.mean(np.sqrt(gamma * p / rho)))


def mach_controlled_power(power, mach, target, enabled, memory, exponent,
                          pmin=None, pmax=None):
    """Slow feedback of the forcing power toward a target Mach
    (``OOP/hit2d.py:293-349``).  Returns (next_power, desired_power)."""
    if not enabled or power is None:
        return power, (np.nan if power is None else float(power))
    if target <= 0.0:
        raise ValueError("Mach control requires a positive target Mach number")
    if not 0.0 <= memory < 1.0:
        raise ValueError("mach_control_memory must be in [0, 1)")
    if exponent <= 0.0:
        raise ValueError("mach_control_exponent must be positive")
    desired = float(power * (target / max(mach, 1e-8)) ** exponent)
    if pmin is not None:
        desired = max(desired, pmin)
    if pmax is not None:
        desired = min(desired, pmax)
    return memory * power + (1.0 - memory) * desired, desired


# --------------------------------------------------------------------------
# Initial states
# --------------------------------------------------------------------------
def cell_centres(lo, hi, n):
    h = (hi - lo) / n
    return lo + h * (np.arange(n) + 0.5)


def hit_initial_state(nx, ny, length, gamma, target_mach, kmin, kmax, seed):
    """Streamfunction on the shell kmin <= |k| <= kmax with one uniform phase
    per +- pair, scaled to the target turbulent Mach
    (``OOP/hit2d.py:158-204``), followed by ``enforce`` as ``run_simulation``
    does (``OOP/hit2d.py:805``)."""
    rng = np.random.default_rng(seed)
    dx, dy = length / nx, length / ny
    X, Y = np.meshgrid(cell_centres(0.0, length, nx), cell_centres(0.0, length, ny), indexing="xy")
    psi = np.zeros_like(X)
    for kx in range(-kmax, kmax + 1):
        for ky in range(-kmax, kmax + 1):
            if ky < 0 or (ky == 0 and kx <= 0):
                continue
            mag = np.sqrt(kx ** 2 + ky ** 2)
            if mag < kmin or mag > kmax:
                continue
            phase = rng.uniform(0.0, 2.0 * np.pi)
            psi += (1.0 / max(kx ** 2 + ky ** 2, 1)) * np.cos(kx * X + ky * Y + phase)
    KX, KY = wavenumbers(nx, ny, dx, dy)
    ph = np.fft.fft2(psi)
    dpsi_dx = np.fft.ifft2(1j * KX * ph).real
    dpsi_dy = np.fft.ifft2(1j * KY * ph).real
    u = dpsi_dy - np.mean(dpsi_dy)
    v = -dpsi_dx
    v = v - np.mean(v)
    rho = np.ones_like(u)
    p = np.full_like(u, 1.0 / gamma)
    c = np.sqrt(gamma * p / rho)
    vrms = np.sqrt(np.mean(u ** 2 + v ** 2))
    if float(vrms) <= np.finfo(float).eps:
        raise ValueError("initial streamfunction produced zero velocity")
    scale = target_mach * float(np.mean(c)) / vrms
    return enforce(conservative(rho, u * scale, v * scale, p, gamma), gamma)


RIEMANN_STATES = {
    # quadrant -> (rho, u, v, p); quadrants: "ll" (x<xs,y<ys), "lr", "ul", "ur"
    3: {"ll": (0.138, 1.206, 1.206, 0.029), "ur": (1.5, 0.0, 0.0, 1.5),
        "ul": (0.5323, 1.206, 0.0, 0.3), "lr": (0.5323, 0.0, 1.206, 0.3)},
    6: {"ll": (1.0, -0.75, 0.5, 1.0), "ur": (1.0, 0.75, -0.5, 1.0),
        "ul": (2.0, 0.75, 0.5, 1.0), "lr": (3.0, -0.75, -0.5, 1.0)},
}


def riemann_initial_state(number, nx, ny, x_split=0.5, y_split=0.5, gamma=1.4,
                          extent=(0.0, 1.0, 0.0, 1.0)):
    """Piecewise-constant quadrant states (``OOP/problems/riemann_config3.py:
    60-99``, ``OOP/problems/riemann_config6.py:26-64``); a cell belongs to the
    upper/right side when its centre is >= the split."""
    X, Y = np.meshgrid(cell_centres(extent[0], extent[1], nx),
                       cell_centres(extent[2], extent[3], ny), indexing="xy")
    top, right = Y >= y_split, X >= x_split
    prim = np.zeros((4, ny, nx))
    for key, sel in (("ll", ~top & ~right), ("lr", ~top & right),
                     ("ul", top & ~right), ("ur", top & right)):
        for c in range(4):
            prim[c][sel] = RIEMANN_STATES[number][key][c]
    return conservative(prim[0], prim[1], prim[2], prim[3], gamma)


# --------------------------------------------------------------------------
# Drivers (the step loops of OOP/hit2d.py:764-918 and
# OOP/problems/riemann_config3.py:681-749), without file I/O.
# --------------------------------------------------------------------------
@dataclass
class HITParams:
    nx: int = 64
    ny: int = 64
    length: float = 2.0 * np.pi
    gamma: float = 1.4
    cfl: float = 0.05
    tfinal: float = 0.05
    target_mach: float = 0.25
    initial_kmin: int = 3
    initial_kmax: int = 5
    forcing_kmin: float = 3.0
    forcing_kmax: float = 5.0
    forcing_rms: float = 1.0
    forcing_correlation_time: float = 1.0
    forcing_alpha_memory: float = 0.2
    target_energy_injection: float | None = 1e-3
    min_forcing_power: float = 1e-6
    max_forcing_rescale: float | None = 20.0
    mach_control: bool = False
    mach_control_target: float | None = None
    mach_control_memory: float = 0.995
    mach_control_exponent: float = 2.0
    mach_control_min_power: float | None = None
    mach_control_max_power: float | None = None
    seed: int = 1234
    viscosity: float = 1e-3
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

    @classmethod
    def production_512(cls, **kw):
        """The 512^2 solenoidal production setup of the reference's README."""
        base = dict(nx=512, ny=512, target_mach=0.25, forcing_correlation_time=0.5,
                    mach_control=True, mach_control_target=0.25, viscosity=7.5e-4,
                    large_scale_drag=0.10, cooling_time=5.0, tfinal=110.0)
        base.update(kw)
        return cls(**base)


def hit_rhs(q, prm: HITParams, fx, fy):
    """``rhs_with_forcing`` of ``OOP/hit2d.py:847-867``."""
    dx, dy = prm.length / prm.nx, prm.length / prm.ny
    sp = SensorParams(prm.sensor_width, prm.compression_threshold, prm.jump_threshold,
                      prm.shear_threshold)
    r = inviscid_rhs(q, dx, dy, prm.gamma, sp, True)
    if prm.viscosity > 0.0:
        r = r + viscous_rhs(q, dx, dy, prm.gamma, prm.viscosity, prm.prandtl)
    s = r + forcing_source(q, fx, fy, prm.gamma)
    if prm.large_scale_drag > 0.0:
        s = s + drag_source(q, dx, dy, prm.gamma, prm.large_scale_drag, prm.large_scale_drag_kmax)
    if prm.cooling_time is not None and prm.cooling_time > 0.0:
        s = s + cooling_source(q, prm.gamma, prm.cooling_time, prm.cooling_target_pressure)
    return s


def hit_run(prm: HITParams, max_steps=None, noise_fn=None, q0=None, record=None):
    """Advance HIT until tfinal (or max_steps).  ``noise_fn(step)`` may supply
    the forcing white noise of each step; otherwise the forcing's own
    ``default_rng(seed + 1)`` stream is used exactly as the reference does.
    Returns (q, time, steps, last_info)."""
    dx, dy = prm.length / prm.nx, prm.length / prm.ny
    if prm.hyperviscosity_interval <= 0 and prm.hyperviscosity_mn > 0.0:
        raise ValueError("hyperviscosity_interval must be positive when mn > 0")
    sp = SensorParams(prm.sensor_width, prm.compression_threshold, prm.jump_threshold,
                      prm.shear_threshold)
    forcing = ShellOUForcing(prm.nx, prm.ny, dx, dy, prm.forcing_kmin or 0.0, prm.forcing_kmax,
                             prm.forcing_correlation_time, prm.forcing_rms,
                             prm.target_energy_injection, prm.min_forcing_power,
                             prm.max_forcing_rescale, prm.forcing_alpha_memory, prm.seed + 1)
    q = q0 if q0 is not None else hit_initial_state(
        prm.nx, prm.ny, prm.length, prm.gamma, prm.target_mach, prm.initial_kmin,
        prm.initial_kmax, prm.seed)
    time, step, info = 0.0, 0, None
    power = prm.target_energy_injection
    target_mach = prm.target_mach if prm.mach_control_target is None else prm.mach_control_target
    while time < prm.tfinal and (max_steps is None or step < max_steps):
        dt = spectral_radius_dt(q, prm.cfl, dx, dy, prm.gamma, prm.tfinal - time)
        if prm.viscosity > 0.0:
            dt = min(dt, 0.25 * min(dx, dy) ** 2 / prm.viscosity, prm.tfinal - time)
        rho, u, v, p = primitives(q, prm.gamma)
        mach = turbulent_mach(rho, u, v, p, prm.gamma)
        power, desired = mach_controlled_power(
            power, mach, target_mach, prm.mach_control, prm.mach_control_memory,
            prm.mach_control_exponent, prm.mach_control_min_power, prm.mach_control_max_power)
        forcing.target_power = power
        noise = None if noise_fn is None else noise_fn(step)
        fx, fy, info = forcing.update(dt, rho, u, v, noise=noise)
        info.update({"mach_control_mach": mach, "mach_control_target": float(target_mach),
                     "mach_control_power_desired": desired})
        q = ssprk3(q, lambda s: hit_rhs(s, prm, fx, fy), dt, lambda s: enforce(s, prm.gamma))
        step += 1
        time += dt
        if prm.hyperviscosity_mn > 0.0 and step % prm.hyperviscosity_interval == 0:
            m = sensor(q, dx, dy, prm.gamma, sp, True)
            q = hyperviscosity(q, ~m, dx, dy, prm.gamma, prm.hyperviscosity_mn,
                               (0.25, 1.0, 1.0, 0.25), True)
        if record is not None:
            record.append({"step": step, "time": time, "dt": dt, **info})
    return q, time, step, info


@dataclass
class RiemannParams:
    number: int = 3
    nx: int = 512
    ny: int = 512
    tfinal: float = 0.3
    cfl: float = 0.4
    gamma: float = 1.4
    x_split: float = 0.5
    y_split: float = 0.5
    scheme: str = "hybrid"
    sensor_width: int = 4
    jump_threshold: float = 0.025
    compression_threshold: float = 2.5
    shear_threshold: float | None = None
    boundary_guard: int = 4
    mn: float = 0.001
    hyperviscosity_interval: int = 1
    hv_weights: tuple = (1.0, 1.0, 1.0, 1.0)
    guard_cells: int = 2


def riemann_setup(prm: RiemannParams):
    q = riemann_initial_state(prm.number, prm.nx, prm.ny, prm.x_split, prm.y_split, prm.gamma)
    q = outflow_guard(enforce(q, prm.gamma), prm.guard_cells)
    dx, dy = 1.0 / prm.nx, 1.0 / prm.ny
    dt, n = fixed_time_step(q, prm.cfl, prm.tfinal, dx, dy, prm.gamma)
    return q, dt, n


def riemann_run(prm: RiemannParams, max_steps=None, q0=None, dt=None):
    """``run_riemann`` step loop (``OOP/problems/riemann_config3.py:681-749``).
    Returns (q, dt, steps, hyperviscosity applications)."""
    q, dt0, n = riemann_setup(prm)
    if q0 is not None:
        q = q0
    if dt is None:
        dt = dt0
    dx, dy = 1.0 / prm.nx, 1.0 / prm.ny
    sp = SensorParams(prm.sensor_width, prm.compression_threshold, prm.jump_threshold,
                      prm.shear_threshold, prm.boundary_guard)
    hv_on = prm.scheme == "hybrid" and prm.mn > 0.0 and prm.hyperviscosity_interval > 0

    def clean(s):
        return outflow_guard(enforce(s, prm.gamma), prm.guard_cells)

    def rhs(s):
        return inviscid_rhs(s, dx, dy, prm.gamma, sp, False, prm.scheme)

    steps = n if max_steps is None else min(n, max_steps)
    apps = 0
    for step in range(steps):
        q = ssprk3(q, rhs, dt, clean)
        if hv_on and (step + 1) % prm.hyperviscosity_interval == 0:
            m = sensor(q, dx, dy, prm.gamma, sp, False)
            q = hyperviscosity(q, ~m, dx, dy, prm.gamma, prm.mn, prm.hv_weights, False)
            q = outflow_guard(q, prm.guard_cells)
            apps += 1
    return q, dt, steps, apps


def riemann_diagnostics(q, prm: RiemannParams):
    """Summary statistics of ``OOP/problems/riemann_config3.py:629-650``
    (without the sensor fraction, which the caller adds)."""
    rho = q[0]
    u, v = q[1] / rho, q[2] / rho
    p = (prm.gamma - 1.0) * (q[3] - 0.5 * rho * (u ** 2 + v ** 2))
    _, uu, vv, _ = primitives(q, prm.gamma)
    omega = central_diff(vv, 1.0 / prm.nx, -1, False) - central_diff(uu, 1.0 / prm.ny, -2, False)
    return {
        "density_min": float(rho.min()), "density_max": float(rho.max()),
        "pressure_min": float(p.min()), "pressure_max": float(p.max()),
        "max_abs_vorticity": float(np.max(np.abs(omega))),
    }


def hit_diagnostics(q, dx, dy, length, gamma):
    """Scalar flow diagnostics of ``OOP/hit2d.py:471-514`` (spectral
    divergence and vorticity)."""
    rho, u, v, p = primitives(q, gamma)
    ny, nx = rho.shape
    KX, KY = wavenumbers(nx, ny, dx, dy)

    def sd(a):
        ah = np.fft.fft2(a)
        return np.fft.ifft2(1j * KX * ah).real, np.fft.ifft2(1j * KY * ah).real

    du_dx, du_dy = sd(u)
    dv_dx, dv_dy = sd(v)
    div = du_dx + dv_dy
    vort = dv_dx - du_dy
    c = np.sqrt(gamma * p / rho)
    uf, vf = u - np.mean(u), v - np.mean(v)
    uu = float(np.mean(rho * uf ** 2))
    vv = float(np.mean(rho * vf ** 2))
    uv = float(np.mean(rho * uf * vf))
    s = uu + vv
    cov = np.sqrt(max(uu * vv, 0.0))
    return {
        "kinetic_energy": 0.5 * s, "Kx": 0.5 * uu, "Ky": 0.5 * vv,
        "A_K": abs(uu - vv) / s if s > 0.0 else 0.0,
        "C_uv": uv / cov if cov > 0.0 else 0.0,
        "rms_velocity": float(np.sqrt(np.mean(u ** 2 + v ** 2))),
        "turbulent_mach": float(np.sqrt(np.mean(u ** 2 + v ** 2)) / np.mean(c)),
        "mean_density": float(np.mean(rho)),
        "mean_pressure": float(np.mean(p)),
        "divergence_rms": float(np.sqrt(np.mean(div ** 2))),
        "vorticity_rms": float(np.sqrt(np.mean(vort ** 2))),
        "enstrophy": float(0.5 * np.mean(vort ** 2)),
        "mass": float(np.mean(rho) * length * length),
    }
